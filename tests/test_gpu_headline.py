"""The headline configuration exactly as bench.py times it: the fused pipeline
rfft(4096) -> raised-cosine notch (mul-spectrum with H = the mask, bins 400-420
zeroed, 32-bin ramps) -> irfft, over all 8192 seeded signals (seed 1), built
by bench.py's own transform builder.  Every signal is checked against the
oracle's restatement of the reference pipeline (reference src/faf_pipeline.c:10-90,
src/chirp.c:1922-2055) and against FP64 numpy, at rel L2 <= 1e-5, and the
input ring's bounded waits must all have completed.  The R2C the bench times
beside it is checked the same way."""
import os
import sys

import numpy as np
import pytest

from conftest import REL_L2_TOL

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    return bench


def _rows_rel(got, want):
    """Per-row rel L2 (rows = signals)."""
    return np.linalg.norm(got - want, axis=-1) / np.linalg.norm(want, axis=-1)


def test_headline_pipeline_full_batch(cuda):
    import fastandfourier_b200 as F
    from oracle import orc
    torch = cuda
    bench = _bench()
    n, batch = 4096, 8192
    x = bench.make_inputs("pipeline", batch)[0]
    assert x.shape == (batch, n)
    t = bench.build_transform(F, "pipeline", torch)
    t.set_stream(torch.cuda.current_stream())
    out = torch.empty((batch, n), dtype=torch.float32, device="cuda")
    bench.run_step(F, t, "pipeline", [torch.from_numpy(x).cuda()], [out])
    torch.cuda.synchronize()
    assert t.wait_status() == 0
    y = out.cpu().numpy()
    m = bench.notch_mask(n)
    want = orc.pipeline(x, [(orc.OP_MUL, 0, 0)], m, np.zeros_like(m))
    r = _rows_rel(y.astype(np.float64), want.astype(np.float64))
    assert r.max() <= REL_L2_TOL, (int(r.argmax()), float(r.max()))
    y64 = np.fft.irfft(np.fft.rfft(x.astype(np.float64), axis=-1) * m, n=n, axis=-1)
    r64 = _rows_rel(y.astype(np.float64), y64)
    assert r64.max() <= REL_L2_TOL, (int(r64.argmax()), float(r64.max()))
    # the notch removed the bin-410 tone from every signal
    Y = np.abs(np.fft.rfft(y.astype(np.float64), axis=-1)[:, 410])
    assert Y.max() < 1e-2 * 5 * n / 2
    t.close()


def test_headline_r2c_full_batch(cuda):
    import fastandfourier_b200 as F
    from oracle import orc
    torch = cuda
    bench = _bench()
    n, batch = 4096, 8192
    x = bench.make_inputs("r2c", batch)[0]
    t = bench.build_transform(F, "r2c", torch)
    t.set_stream(torch.cuda.current_stream())
    outs = bench.alloc_outputs("r2c", batch, torch.empty(1, device="cuda"), torch)
    bench.run_step(F, t, "r2c", [torch.from_numpy(x).cuda()], outs)
    torch.cuda.synchronize()
    assert t.wait_status() == 0
    got = outs[0].cpu().numpy().astype(np.float64) + 1j * outs[1].cpu().numpy()
    wr, wi = orc.r2c(x)
    r = _rows_rel(got, wr.astype(np.float64) + 1j * wi)
    assert r.max() <= REL_L2_TOL, (int(r.argmax()), float(r.max()))
    r64 = _rows_rel(got, np.fft.rfft(x.astype(np.float64), axis=-1))
    assert r64.max() <= REL_L2_TOL
    t.close()


def test_bench_line_checks_its_output(cuda):
    """bench.py's own check of the timed output (first and last signals of
    the last step vs FP64) passes on the headline pipeline."""
    import fastandfourier_b200 as F
    torch = cuda
    bench = _bench()
    batch = 8192
    x = bench.make_inputs("pipeline", batch)
    t = bench.build_transform(F, "pipeline", torch)
    outs = bench.alloc_outputs("pipeline", batch, torch.empty(1, device="cuda"), torch)
    bench.run_step(F, t, "pipeline", [torch.from_numpy(x[0]).cuda()], outs)
    torch.cuda.synchronize()
    chk = bench.fp64_check("pipeline", x, outs, batch)
    assert chk["rel_l2_vs_fp64"] <= REL_L2_TOL
    t.close()
