"""Serving loop (include/faf_serve.h): results against the oracle, the same
alone and in a concurrent mix, streamed STFT continuity, the HBM budget,
host buffers and the arrival-time replay."""
import os
import sys

import numpy as np
import pytest

from conftest import REL_L2_TOL, ROOT, seeded
from oracle import orc

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import cases  # noqa: E402

pytestmark = pytest.mark.gpu

PIPE = "(pipeline (rfft :size 4096) (mul-spectrum) (irfft))"


def _mk_mix(torch, seed, count=48):
    """Mixed requests on the device: rfft of several sizes, the notch pipeline
    and whole-signal STFTs (some share a plan, so they can merge)."""
    import fastandfourier_b200 as F
    rng = seeded(seed)
    m = torch.from_numpy(cases.notch_mask(4096)).cuda()
    z = torch.zeros_like(m)
    h = (m, z, 2049)
    reqs, meta = [], []
    for i in range(count):
        kind = ("rfft", "pipe", "stft")[i % 3]
        if kind == "rfft":
            n = int(rng.choice([256, 1000, 4096, 65536]))
            units = int(rng.integers(1, 4))
            x = torch.from_numpy(rng.standard_normal(units * n).astype(np.float32)).cuda()
            o_re = torch.empty(units * (n // 2 + 1), device="cuda")
            o_im = torch.empty_like(o_re)
            reqs.append(F.Request(x, o_re, o_im, chirp=f"(rfft :size {n})"))
            meta.append(("rfft", n, x, (o_re, o_im)))
        elif kind == "pipe":
            units = int(rng.integers(1, 3))
            x = torch.from_numpy(rng.standard_normal(units * 4096).astype(np.float32)).cuda()
            o = torch.empty_like(x)
            reqs.append(F.Request(x, o, chirp=PIPE, h=h))
            meta.append(("pipe", 4096, x, (o,)))
        else:
            L = int(rng.choice([4096, 20000]))
            x = torch.from_numpy(rng.standard_normal(L).astype(np.float32)).cuda()
            Fr = 1 + (L - 1024) // 256
            o_re = torch.empty(Fr * 513, device="cuda")
            o_im = torch.empty_like(o_re)
            reqs.append(F.Request(x, o_re, o_im, stft=(1024, 1024, 256)))
            meta.append(("stft", L, x, (o_re, o_im)))
    return reqs, meta, h


def _check_oracle(meta, h):
    worst = 0.0
    for kind, n, x, outs in meta:
        xh = x.cpu().numpy()
        if kind == "rfft":
            Xr, Xi = orc.r2c(xh.reshape(-1, n))
            e = orc.rel_l2_complex(outs[0].cpu().numpy().reshape(Xr.shape),
                                   outs[1].cpu().numpy().reshape(Xr.shape), Xr + 1j * Xi)
        elif kind == "pipe":
            mh = h[0].cpu().numpy()
            y = orc.pipeline(xh.reshape(-1, 4096), [(orc.OP_MUL, 0, 0)], mh, np.zeros_like(mh))
            e = orc.rel_l2(outs[0].cpu().numpy().reshape(y.shape), y)
        else:
            Xr, Xi = orc.stft(xh[None], 1024, 1024, 256)
            e = orc.rel_l2_complex(outs[0].cpu().numpy().reshape(Xr.shape),
                                   outs[1].cpu().numpy().reshape(Xr.shape), Xr + 1j * Xi)
        worst = max(worst, e)
    return worst


def test_serve_mix_matches_oracle(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    reqs, meta, h = _mk_mix(torch, 11)
    srv = F.Server(hbm_budget=1 << 30, streams=4)
    ids = [srv.submit(r) for r in reqs]
    for i in ids:
        lat, _ = srv.wait(i)
        assert lat > 0
    assert _check_oracle(meta, h) <= REL_L2_TOL
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    srv.close()


def test_serve_alone_equals_in_mix(cuda):
    """Each result is the same when its request runs alone and when it runs
    merged and overlapped with the others."""
    import fastandfourier_b200 as F
    torch = cuda
    reqs, meta, h = _mk_mix(torch, 12)
    srv = F.Server(hbm_budget=1 << 30, streams=4, max_merge=64)
    alone = []
    for r in reqs:
        srv.wait(srv.submit(r))
        alone.append([o.clone() for o in r.keep[1:3] if o is not None])
    for r in reqs:
        for o in r.keep[1:3]:
            if o is not None:
                o.fill_(float("nan"))
    srv.reset_stats()
    ids = [srv.submit(r) for r in reqs]  # burst: merged and overlapped
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st["merged_requests"] > 0 and st["batches"] < len(reqs)
    for r, a in zip(reqs, alone):
        outs = [o for o in r.keep[1:3] if o is not None]
        for got, want in zip(outs, a):
            g, w = got.cpu().numpy(), want.cpu().numpy()
            assert np.isfinite(g).all()
            assert orc.rel_l2(g, w) <= REL_L2_TOL
    srv.close()


def test_serve_streamed_stft_continuity(cuda):
    """Chunks of one stream give the frames of the whole signal: the overlap
    stays on the device between requests."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(13)
    chunks = [50000, 70001, 255, 76352]
    total = sum(chunks)
    x = rng.standard_normal(total).astype(np.float32)
    srv = F.Server(hbm_budget=256 << 20, streams=3)
    key = 4242
    outs, off, ids = [], 0, []
    for c in chunks:
        fr = srv.stream_frames(key, 1024, 256, c)
        xc = torch.from_numpy(x[off:off + c].copy()).cuda()
        o_re = torch.empty(max(fr, 1) * 513, device="cuda")
        o_im = torch.empty_like(o_re)
        ids.append(srv.submit(F.Request(xc, o_re, o_im, stft=(1024, 1024, 256), stream_key=key)))
        outs.append((fr, o_re, o_im))
        off += c
    got_r, got_i = [], []
    for i, (fr, o_re, o_im) in zip(ids, outs):
        _, frames = srv.wait(i)
        assert frames == fr
        got_r.append(o_re.cpu().numpy()[:fr * 513])
        got_i.append(o_im.cpu().numpy()[:fr * 513])
    got_r, got_i = np.concatenate(got_r), np.concatenate(got_i)
    Xr, Xi = orc.stft(x[None], 1024, 1024, 256)
    assert got_r.size == Xr.size
    assert orc.rel_l2_complex(got_r.reshape(Xr.shape), got_i.reshape(Xr.shape),
                              Xr + 1j * Xi) <= REL_L2_TOL
    srv.close_stream(key)
    srv.close()


def test_serve_budget_admission(cuda):
    """A small arena still serves everything (requests wait for memory), the
    peak stays within it, and a request above it is rejected."""
    import fastandfourier_b200 as F
    torch = cuda
    budget = 4 << 20
    srv = F.Server(hbm_budget=budget, streams=8, max_merge=4)
    rng = seeded(14)
    reqs = []
    for _ in range(30):
        x = torch.from_numpy(rng.standard_normal(4 * 16384).astype(np.float32)).cuda()
        o_re = torch.empty(4 * 8193, device="cuda")
        o_im = torch.empty_like(o_re)
        reqs.append((x, o_re, o_im, F.Request(x, o_re, o_im, chirp="(rfft :size 16384)")))
    ids = [srv.submit(r[3]) for r in reqs]
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st["completed"] == 30 and st["arena_peak_bytes"] <= budget
    for x, o_re, o_im, _ in reqs[:3]:
        Xr, Xi = orc.r2c(x.cpu().numpy().reshape(4, 16384))
        assert orc.rel_l2_complex(o_re.cpu().numpy().reshape(Xr.shape),
                                  o_im.cpu().numpy().reshape(Xr.shape), Xr + 1j * Xi) <= REL_L2_TOL
    big = torch.zeros(1 << 20, device="cuda")
    ob = torch.empty(2 * ((1 << 20) // 2 + 1), device="cuda")
    with pytest.raises(F.FafError):
        srv.submit(F.Request(big, ob, ob, chirp="(rfft :size 65536)"))
    srv.close()


def test_serve_host_buffers(cuda):
    import fastandfourier_b200 as F
    rng = seeded(15)
    x = rng.standard_normal(3 * 4096).astype(np.float32)
    o_re = np.empty(3 * 2049, np.float32)
    o_im = np.empty_like(o_re)
    srv = F.Server(hbm_budget=64 << 20, streams=2)
    srv.wait(srv.submit(F.Request(x, o_re, o_im, chirp="(rfft :size 4096)")))
    Xr, Xi = orc.r2c(x.reshape(3, 4096))
    assert orc.rel_l2_complex(o_re.reshape(Xr.shape), o_im.reshape(Xr.shape),
                              Xr + 1j * Xi) <= REL_L2_TOL
    srv.close()


def test_serve_replay_latencies(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    reqs, meta, h = _mk_mix(torch, 16, count=120)
    srv = F.Server(hbm_budget=1 << 30, streams=8)
    for r in reqs[:6]:
        srv.prepare(r)
    rng = seeded(17)
    arrivals = np.cumsum(rng.exponential(1 / 20000.0, len(reqs)))
    lat = srv.replay(reqs, arrivals)
    assert all(v > 0 for v in lat)
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert 0 < st["p50_latency_s"] <= st["p99_latency_s"] <= st["max_latency_s"]
    assert _check_oracle(meta, h) <= REL_L2_TOL
    srv.close()
