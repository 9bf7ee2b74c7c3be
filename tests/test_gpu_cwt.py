"""CWT filter bank (faf_cuda_create_cwt): the device execute of the
reference's forward CWT (src/faf_cwt.c:769-847) against the reference's own
outputs for its default banks (golden fixtures), the oracle, and FP64 numpy,
over power-of-two and 5-smooth lengths, batches, host and device buffers, and
the create-time checks."""
import os
import sys

import numpy as np
import pytest

from conftest import REL_L2_TOL, ROOT, seeded
from oracle import orc

pytestmark = pytest.mark.gpu

GOLD = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLD)
import cases  # noqa: E402


def rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def bank(rows, n, seed):
    """Seeded smooth bandpass rows (positive, like analytic wavelet banks)."""
    nb = n // 2 + 1
    k = np.arange(nb)[None, :]
    c = np.geomspace(2.0, nb * 0.8, rows)[:, None]
    rng = seeded(seed)
    return (np.exp(-0.5 * ((k - c) / (0.25 * c + 1.0)) ** 2) * rng.uniform(0.5, 2, (rows, 1))).astype(np.float32)


@pytest.mark.parametrize("n", cases.CWT)
def test_cwt_matches_reference_golden(cuda, n):
    import fastandfourier_b200 as F
    torch = cuda
    g = np.load(os.path.join(GOLD, "golden.npz"))
    psi, want = g[f"cwt_psi_{n}"], g[f"cwt_{n}"]
    x = cases.real_input(n, batch=1, seed=9)
    t = F.Transform.cwt(n, psi)
    assert t.type == F.T_CWT and t.kind == "cwt" and t.cwt_rows == psi.shape[0]
    W = t.analyze(torch.from_numpy(x).cuda()).cpu().numpy()
    assert W.shape == want.shape
    assert rel(W, want) <= REL_L2_TOL
    assert rel(W, orc.fp64_cwt(x, psi)) <= REL_L2_TOL
    assert t.wait_status() == 0


@pytest.mark.parametrize("n", [16, 256, 1000, 4096, 6000, 32768])
def test_cwt_batches_match_oracle(cuda, n):
    import fastandfourier_b200 as F
    torch = cuda
    psi = bank(7, n, n)
    x = seeded(n + 1).standard_normal((3, n)).astype(np.float32)
    t = F.Transform.cwt(n, psi)
    W = t.analyze(torch.from_numpy(x).cuda()).cpu().numpy()
    assert W.shape == (3, 7, n)
    assert rel(W, orc.cwt(x, psi)) <= REL_L2_TOL
    assert rel(W, orc.fp64_cwt(x, psi)) <= REL_L2_TOL
    assert t.wait_status() == 0  # n >= 1024: the rows' spectra land in the C2R ring


def test_cwt_host_buffers_and_device_bank(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    n = 2048
    psi = bank(5, n, 3)
    x = seeded(5).standard_normal((4, n)).astype(np.float32)
    want = orc.fp64_cwt(x, psi)
    t_host = F.Transform.cwt(n, psi)                       # bank from host memory
    assert rel(t_host.analyze(x), want) <= REL_L2_TOL      # host signal and output
    t_dev = F.Transform.cwt(n, torch.from_numpy(psi).cuda())  # bank from device memory
    assert rel(t_dev.analyze(torch.from_numpy(x).cuda()).cpu().numpy(), want) <= REL_L2_TOL


def test_cwt_padded_bank_rows(cuda):
    """Rows `psi_stride` floats apart, as the reference bank pads them."""
    import fastandfourier_b200 as F
    torch = cuda
    n = 1000
    psi = bank(4, n, 8)
    padded = np.zeros((4, 512), np.float32)
    padded[:, :501] = psi
    padded[:, 501:] = 1e9  # the padding must never be read
    x = seeded(9).standard_normal((2, n)).astype(np.float32)
    W = F.Transform.cwt(n, padded).analyze(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel(W, orc.fp64_cwt(x, psi)) <= REL_L2_TOL


def test_cwt_large_batch_chunks(cuda):
    """More signals than one 32 MB chunk of spectra: two R2C / C2R rounds."""
    import fastandfourier_b200 as F
    torch = cuda
    n, rows, batch = 4096, 3, 2050
    psi = bank(rows, n, 11)
    x = seeded(12).standard_normal((batch, n)).astype(np.float32)
    t = F.Transform.cwt(n, psi)
    W = t.analyze(torch.from_numpy(x).cuda())
    assert F.lib().faf_cuda_last_launches() == 4
    pick = [0, 1, 2046, 2047, 2048, 2049]
    got = W[pick].cpu().numpy()
    assert rel(got, orc.fp64_cwt(x[pick], psi)) <= REL_L2_TOL


def test_cwt_create_errors(cuda):
    import fastandfourier_b200 as F
    psi = np.ones((2, 40000), np.float32)
    with pytest.raises(F.FafError, match="exceed one CTA"):
        F.Transform.cwt(65536, np.ones((2, 32769), np.float32))
    with pytest.raises(F.FafError, match="even and 5-smooth"):
        F.Transform.cwt(14, psi)
    t = F.Transform.cwt(64, psi[:, :33])
    with pytest.raises(F.FafError, match="buffer n mismatch"):
        t.execute(F._buf(np.zeros(2 * 64, np.float32), None, 2 * 64, F.L_REAL),
                  F._buf(np.zeros(32, np.float32), None, 32, F.L_REAL))


@pytest.mark.parametrize("n", cases.CWT)
def test_icwt_matches_reference_golden(cuda, n):
    """Both inverse forms on the reference's coefficients, against the
    reference's own inverse outputs."""
    import math
    import fastandfourier_b200 as F
    torch = cuda
    g = np.load(os.path.join(GOLD, "golden.npz"))
    W, psi = g[f"cwt_{n}"], g[f"cwt_psi_{n}"]
    C, voices = g[f"cwt_consts_{n}"]
    td = F.Transform.icwt_dual(n, F.Transform.cwt_dual_rows(psi))
    assert td.type == F.T_ICWT and td.kind == "icwt-dual"
    x = td.synthesize(torch.from_numpy(W).cuda()).cpu().numpy()
    assert rel(x, g[f"icwt_dual_{n}"]) <= REL_L2_TOL
    tl = F.Transform.icwt_l1(n, psi.shape[0], True, math.log(2) / voices, C)
    assert tl.kind == "icwt-l1"
    x = tl.synthesize(torch.from_numpy(W).cuda()).cpu().numpy()
    assert rel(x, g[f"icwt_l1_{n}"]) <= REL_L2_TOL


@pytest.mark.parametrize("n", [256, 1000, 4096, 6000])
def test_cwt_dual_round_trip(cuda, n):
    """analyze -> synthesize with the bank's dual rows returns the signal
    (a tight frame up to eps); batched, against the oracle too."""
    import fastandfourier_b200 as F
    torch = cuda
    psi = bank(24, n, n + 3)
    psi[0] = np.maximum(psi[0], 1.0 - psi[1:].max(axis=0))  # cover every bin
    x = seeded(n + 4).standard_normal((5, n)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    W = F.Transform.cwt(n, psi).analyze(xd)
    dual = F.Transform.cwt_dual_rows(psi)
    t = F.Transform.icwt_dual(n, dual)
    y = t.synthesize(W).cpu().numpy()
    assert rel(y, orc.icwt_dual(W.cpu().numpy(), dual)) <= REL_L2_TOL
    assert rel(y, x) <= 1e-4
    assert t.wait_status() == 0


def test_icwt_batches_and_host_buffers(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    n, rows = 2048, 9
    rng = seeded(21)
    W = rng.standard_normal((3, rows, n)).astype(np.float32)
    dual = bank(rows, n, 22)
    want = orc.icwt_dual(W, dual)
    t = F.Transform.icwt_dual(n, dual)
    assert rel(t.synthesize(W), want) <= REL_L2_TOL                      # host buffers
    assert rel(t.synthesize(torch.from_numpy(W).cuda()).cpu().numpy(), want) <= REL_L2_TOL
    tl = F.Transform.icwt_l1(n, rows, False, 0.0693, 0.5)
    assert rel(tl.synthesize(torch.from_numpy(W).cuda()).cpu().numpy(),
               orc.icwt_l1(W, False, 0.0693, 0.5)) <= REL_L2_TOL


def test_icwt_large_batch_chunks(cuda):
    """More coefficient sets than one 64 MB chunk of row spectra."""
    import fastandfourier_b200 as F
    torch = cuda
    n, rows, batch = 4096, 16, 260
    dual = bank(rows, n, 31)
    W = torch.randn(batch, rows, n, device="cuda")
    t = F.Transform.icwt_dual(n, dual)
    y = t.synthesize(W)
    assert F.lib().faf_cuda_last_launches() == 6
    pick = [0, 1, 255, 256, 259]
    assert rel(y[pick].cpu().numpy(), orc.icwt_dual(W[pick].cpu().numpy(), dual)) <= REL_L2_TOL
