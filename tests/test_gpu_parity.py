"""GPU parity: the CUDA path through the C ABI vs the oracle (CPU restatement
of the reference, oracle/faf_oracle.c) and vs the FP64 DFT, at rel L2 <= 1e-5.

Cases follow the reference's own known-answer tests (tests/test_mixed_radix.cpp,
tests/test_rader.cpp, tests/test_sizes.cpp, tests/test_rfft.cpp,
tests/test_spectral.cpp) plus the seeded configurations of the path.
"""
import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu

C2C_SIZES = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 15, 16, 20, 30, 32, 48, 60, 64, 100, 128, 192,
             240, 256, 360, 512, 1000, 1024, 1920, 2048, 3072, 4000, 4096, 4050, 6000, 8192,
             15360, 16384]
RADER_PRIMES = [11, 13, 17, 19, 29, 31, 37, 41, 43, 61, 97, 113, 257, 1009, 7681, 12289]
BLUESTEIN_SIZES = [23, 47, 53, 307, 1021, 4099]
REAL_SIZES = [2, 4, 6, 8, 10, 16, 30, 32, 64, 100, 1000, 1024, 4096, 6000, 8192, 16384, 30000,
              32768]


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    return t.cpu().numpy()


def _c2c_case(torch, F, n, inverse, norm=1, batch=3, flags=0, seed=0):
    rng = seeded(seed + n)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    t = F.Transform.fft(n, inverse=inverse, norm=norm, flags=flags)
    yr, yi = t.c2c(dev(torch, re), dev(torch, im))
    torch.cuda.synchronize()
    gr, gi = host(yr), host(yi)
    wr, wi = orc.c2c(re, im, inverse=inverse, norm=norm, flags=flags)
    e_orc = orc.rel_l2_complex(gr, gi, wr + 1j * wi)
    e_64 = orc.rel_l2_complex(gr, gi, orc.fp64_c2c(re, im, inverse=inverse, norm=norm))
    return t, e_orc, e_64


@pytest.mark.parametrize("n", C2C_SIZES)
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_matches_oracle(cuda, n, inverse):
    import fastandfourier_b200 as F
    t, e_orc, e_64 = _c2c_case(cuda, F, n, inverse)
    assert t.kind == "c2c"
    assert e_orc <= REL_L2_TOL, (n, inverse, e_orc)
    assert e_64 <= REL_L2_TOL, (n, inverse, e_64)


@pytest.mark.parametrize("norm", [2, 3])
@pytest.mark.parametrize("n", [60, 1024])
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_norms(cuda, n, norm, inverse):
    import fastandfourier_b200 as F
    _, e_orc, e_64 = _c2c_case(cuda, F, n, inverse, norm=norm)
    assert e_orc <= REL_L2_TOL and e_64 <= REL_L2_TOL


@pytest.mark.parametrize("p", RADER_PRIMES)
@pytest.mark.parametrize("inverse", [False, True])
def test_rader_matches_oracle(cuda, p, inverse):
    import fastandfourier_b200 as F
    t, e_orc, e_64 = _c2c_case(cuda, F, p, inverse)
    assert t.kind == "rader"
    assert e_orc <= REL_L2_TOL and e_64 <= REL_L2_TOL, (p, e_orc, e_64)


@pytest.mark.parametrize("n", BLUESTEIN_SIZES)
@pytest.mark.parametrize("inverse", [False, True])
def test_bluestein_matches_oracle(cuda, n, inverse):
    import fastandfourier_b200 as F
    t, e_orc, e_64 = _c2c_case(cuda, F, n, inverse, flags=F.FLAG_BLUESTEIN)
    assert t.kind == "bluestein"
    assert e_orc <= REL_L2_TOL and e_64 <= REL_L2_TOL, (n, e_orc, e_64)


@pytest.mark.parametrize("n", REAL_SIZES)
def test_r2c_c2r_match_oracle(cuda, n):
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(100 + n)
    x = rng.standard_normal((3, n)).astype(np.float32)
    fwd = F.Transform.rfft(n)
    Xr, Xi = fwd.r2c(dev(torch, x))
    torch.cuda.synchronize()
    gr, gi = host(Xr), host(Xi)
    wr, wi = orc.r2c(x)
    assert orc.rel_l2_complex(gr, gi, wr + 1j * wi) <= REL_L2_TOL
    assert orc.rel_l2_complex(gr, gi, orc.fp64_r2c(x)) <= REL_L2_TOL
    # DC and Nyquist are real
    assert np.all(gi[:, 0] == 0) and np.all(gi[:, -1] == 0)
    inv = fwd.inverse()
    assert inv.type == F.T_IRFFT
    y = host(inv.c2r(Xr, Xi))
    want = orc.c2r(gr, gi, n)
    assert orc.rel_l2(y, want) <= REL_L2_TOL
    assert orc.rel_l2(y, x) <= REL_L2_TOL


def notch_mask(n=4096, lo=400, hi=420, ramp=32):
    """Raised-cosine notch: 0 on [lo, hi], cosine ramps over `ramp` bins on
    each side, 1 elsewhere (the fused-pipeline configuration's mask)."""
    nb = n // 2 + 1
    k = np.arange(nb)
    m = np.ones(nb)
    m[(k >= lo) & (k <= hi)] = 0.0
    left = (k >= lo - ramp) & (k < lo)
    m[left] = 0.5 * (1 + np.cos(np.pi * (k[left] - (lo - ramp)) / ramp))
    right = (k > hi) & (k <= hi + ramp)
    m[right] = 0.5 * (1 - np.cos(np.pi * (k[right] - hi) / ramp))
    return m.astype(np.float32)


def notch_signal(batch, n=4096, seed=1):
    rng = seeded(seed)
    k = np.arange(n)
    return (rng.standard_normal((batch, n)) + 5 * np.cos(2 * np.pi * 410 * k / n)).astype(np.float32)


def test_pipeline_notch_matches_oracle(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    n, nb = 4096, 2049
    x = notch_signal(64)
    m = notch_mask()
    z = np.zeros(nb, np.float32)
    t = F.Transform.chirp("(pipeline (rfft :size 4096) (mul-spectrum) (irfft))")
    assert t.type == F.T_PIPELINE and t.kind == "pipeline"
    hm, hz = dev(torch, m), dev(torch, z)
    t.bind(hm, hz, nb)
    y = host(t.pipeline(dev(torch, x)))
    want = orc.pipeline(x, [(orc.OP_MUL, 0, 0)], m, z)
    assert orc.rel_l2(y, want) <= REL_L2_TOL
    # FP64: irfft(rfft(x) * mask)
    y64 = np.fft.irfft(np.fft.rfft(x.astype(np.float64)) * m, n=n)
    assert orc.rel_l2(y, y64) <= REL_L2_TOL
    # the 410-bin tone is gone
    assert np.abs(np.fft.rfft(y[0])[410]) < 1e-2 * np.abs(np.fft.rfft(x[0])[410])


def test_pipeline_host_bound_spectrum(cuda):
    """H bound in host memory is read at every execute (reference semantics)."""
    import fastandfourier_b200 as F
    torch = cuda
    n, nb = 256, 129
    x = notch_signal(4, n=n, seed=5)
    t = F.Transform.chirp("(pipeline (rfft :size 256) (mul-spectrum) (irfft))")
    hr = np.linspace(0, 1, nb).astype(np.float32)
    hi = np.linspace(1, -1, nb).astype(np.float32)
    t.bind(hr, hi, nb)
    y = host(t.pipeline(dev(torch, x)))
    assert orc.rel_l2(y, orc.pipeline(x, [(orc.OP_MUL, 0, 0)], hr, hi)) <= REL_L2_TOL
    hr[:] = 0.5
    y2 = host(t.pipeline(dev(torch, x)))
    assert orc.rel_l2(y2, orc.pipeline(x, [(orc.OP_MUL, 0, 0)], hr, hi)) <= REL_L2_TOL


@pytest.mark.parametrize("src,ops", [
    ("(pipeline (rfft :size 32) (bandpass :lo 4 :hi 4) (irfft))", [(3, 4, 4)]),
    ("(pipeline (rfft :size 16) conj (irfft))", [(1, 0, 0)]),
    ("(pipeline (rfft :size 6000) conj (bandpass :lo 10 :hi 2000) (irfft))",
     [(1, 0, 0), (3, 10, 2000)]),
    ("(pipeline (rfft :size 1024 :norm ortho) (bandpass :lo 0 :hi 100) (irfft))", [(3, 0, 100)]),
])
def test_pipeline_ops_match_oracle(cuda, src, ops):
    import fastandfourier_b200 as F
    torch = cuda
    t = F.Transform.chirp(src)
    n = t.n
    x = seeded(7).standard_normal((5, n)).astype(np.float32)
    y = host(t.pipeline(dev(torch, x)))
    norm = 2 if ":norm ortho" in src else 1
    assert orc.rel_l2(y, orc.pipeline(x, ops, norm=norm)) <= REL_L2_TOL


def test_pipeline_known_answers(cuda):
    """reference tests/test_spectral.cpp: bandpass keeps bin 4 and drops bin 7;
    conj is time reversal; identity kernel is the identity."""
    import fastandfourier_b200 as F
    torch = cuda
    n = 32
    i = np.arange(n)
    x = (np.cos(2 * np.pi * 4 * i / n) + np.cos(2 * np.pi * 7 * i / n)).astype(np.float32)[None]
    t = F.Transform.chirp("(pipeline (rfft :size 32) (bandpass :lo 4 :hi 4) (irfft))")
    y = host(t.pipeline(dev(torch, x)))[0]
    Y = np.fft.rfft(y)
    assert abs(Y[4]) > 8 and abs(Y[7]) < 1e-3
    t = F.Transform.chirp("(pipeline (rfft :size 16) conj (irfft))")
    x = (np.arange(16) - 8).astype(np.float32)[None]
    y = host(t.pipeline(dev(torch, x)))[0]
    assert abs(y[0] - x[0, 0]) < 1e-4
    assert np.allclose(y[1:], x[0, 1:][::-1], atol=1e-4)
    t = F.Transform.chirp("(pipeline (rfft :size 32) (mul-spectrum) (irfft))")
    h = np.zeros(32, np.float32)
    h[0] = 1
    Hr, Hi = orc.r2c(h)
    t.bind(dev(torch, Hr), dev(torch, Hi), 17)
    x = np.sin(2 * np.pi * 2 * np.arange(32) / 32).astype(np.float32)[None]
    y = host(t.pipeline(dev(torch, x)))
    assert np.allclose(y, x, atol=1e-4)


@pytest.mark.parametrize("n,win,hop,L", [(1024, 1024, 256, 5000), (512, 400, 160, 3000),
                                         (64, 64, 16, 64)])
def test_stft_framing_matches_oracle(cuda, n, win, hop, L):
    import fastandfourier_b200 as F
    torch = cuda
    x = seeded(4).standard_normal((3, L)).astype(np.float32)
    t = F.Transform.stft(n, win=win, hop=hop)
    assert t.type == F.T_STFT
    Xr, Xi = t.stft_frames(dev(torch, x))
    gr, gi = host(Xr), host(Xi)
    wr, wi = orc.stft(x, n, win, hop)
    assert gr.shape == wr.shape
    assert orc.rel_l2_complex(gr, gi, wr + 1j * wi) <= REL_L2_TOL


def test_c2c_interleaved_layout(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    n = 1000
    rng = seeded(11)
    z = rng.uniform(-1, 1, (4, n, 2)).astype(np.float32)
    t = F.Transform.fft(n, layout=F.L_INTERLEAVED)
    y = host(t.c2c(dev(torch, z.reshape(4, 2 * n)))).reshape(4, n, 2)
    want = orc.fp64_c2c(z[..., 0], z[..., 1])
    assert orc.rel_l2_complex(y[..., 0], y[..., 1], want) <= REL_L2_TOL


def test_host_buffers_roundtrip():
    """numpy (host) buffers: the library copies in and out around the kernel."""
    import fastandfourier_b200 as F
    n = 4096
    rng = seeded(12)
    re = rng.uniform(-1, 1, (8, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (8, n)).astype(np.float32)
    t = F.Transform.fft(n)
    yr, yi = t.c2c(re, im)
    assert orc.rel_l2_complex(yr, yi, orc.fp64_c2c(re, im)) <= REL_L2_TOL
    x = rng.standard_normal((5, n)).astype(np.float32)
    Xr, Xi = F.Transform.rfft(n).r2c(x)
    assert orc.rel_l2_complex(Xr, Xi, orc.fp64_r2c(x)) <= REL_L2_TOL



def test_in_place_c2c(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    for n in (16, 60, 1024, 6000, 17, 23):
        rng = seeded(13 + n)
        re = rng.uniform(-1, 1, (3, n)).astype(np.float32)
        im = rng.uniform(-1, 1, (3, n)).astype(np.float32)
        flags = F.FLAG_BLUESTEIN if n == 23 else 0
        t = F.Transform.fft(n, flags=flags)
        a, b = dev(torch, re), dev(torch, im)
        t.c2c(a, b, out_re=a, out_im=b)
        assert orc.rel_l2_complex(host(a), host(b), orc.fp64_c2c(re, im)) <= REL_L2_TOL, n


def test_batched_with_distance(cuda):
    """faf_execute_batched with strided transforms (dist > n)."""
    import fastandfourier_b200 as F
    torch = cuda
    n, dist, batch = 240, 256, 7
    rng = seeded(14)
    re = rng.uniform(-1, 1, (batch, dist)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, dist)).astype(np.float32)
    t = F.Transform.fft(n)
    a, b = dev(torch, re), dev(torch, im)
    oa, ob = torch.zeros_like(a), torch.zeros_like(b)
    t.execute_batched(F._buf(oa, ob, n, F.L_SPLIT), F._buf(a, b, n, F.L_SPLIT), batch, dist, dist)
    got = host(oa)[:, :n] + 1j * host(ob)[:, :n]
    want = orc.fp64_c2c(re[:, :n], im[:, :n])
    assert orc.rel_l2(got, want) <= REL_L2_TOL
    assert np.all(host(oa)[:, n:] == 0)


def test_user_stream_async(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    n = 2048
    s = torch.cuda.Stream()
    t = F.Transform.fft(n)
    t.set_stream(s)
    rng = seeded(15)
    re = rng.uniform(-1, 1, (64, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (64, n)).astype(np.float32)
    with torch.cuda.stream(s):
        a, b = dev(torch, re), dev(torch, im)
        yr, yi = t.c2c(a, b)
    s.synchronize()
    assert orc.rel_l2_complex(host(yr), host(yi), orc.fp64_c2c(re, im)) <= REL_L2_TOL


def test_default_torch_stream_is_asynchronous(cuda):
    """torch's default stream (handle 0) is set as cudaStreamLegacy: execute
    enqueues on it without synchronising, and stream order keeps results
    right for a consumer on the same stream."""
    import fastandfourier_b200 as F
    torch = cuda
    n = 4096
    t = F.Transform.rfft(n)
    t.set_stream(torch.cuda.current_stream())
    assert F.lib().faf_cuda_get_stream(t._p) == F.CUDA_STREAM_LEGACY
    x = seeded(16).standard_normal((256, n)).astype(np.float32)
    xd = dev(torch, x)
    Xr, Xi = t.r2c(xd)
    got = (Xr * 2).cpu().numpy() + 1j * (Xi * 2).cpu().numpy()  # same-stream consumer
    want = 2 * np.fft.rfft(x.astype(np.float64), axis=-1)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= REL_L2_TOL
    t.set_stream(None)
    assert F.lib().faf_cuda_get_stream(t._p) is None


def test_config1_c2c_forward_inverse(cuda):
    """C2C N=1024, batch 256, NumPy norm, forward then inverse, seed 0."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(0)
    re = rng.uniform(-1, 1, (256, 1024)).astype(np.float32)
    im = rng.uniform(-1, 1, (256, 1024)).astype(np.float32)
    fwd = F.Transform.fft(1024)
    inv = fwd.inverse()
    Yr, Yi = fwd.c2c(dev(torch, re), dev(torch, im))
    Zr, Zi = inv.c2c(Yr, Yi)
    wr, wi = orc.c2c(re, im)
    assert orc.rel_l2_complex(host(Yr), host(Yi), wr + 1j * wi) <= REL_L2_TOL
    assert orc.rel_l2_complex(host(Zr), host(Zi), re + 1j * im) <= REL_L2_TOL


@pytest.mark.parametrize("n", [16, 64, 1024, 2048, 16384])
def test_generic_engine_power_of_two(cuda, n, monkeypatch):
    """The runtime-radix engine on power-of-two sizes (normally served by the
    compile-time kernels) stays in parity too."""
    import fastandfourier_b200 as F
    monkeypatch.setenv("FAF_CUDA_GENERIC", "1")
    _, e_orc, e_64 = _c2c_case(cuda, F, n, False)
    assert e_orc <= REL_L2_TOL and e_64 <= REL_L2_TOL
    torch = cuda
    x = seeded(200 + n).standard_normal((3, 2 * n)).astype(np.float32)
    Xr, Xi = F.Transform.rfft(2 * n).r2c(dev(torch, x))
    assert orc.rel_l2_complex(host(Xr), host(Xi), orc.fp64_r2c(x)) <= REL_L2_TOL


# 15552 / 15625 / 16000 fit the single-CTA length limit but need more than
# 1024 threads at 16 values per thread (radix-3 / radix-5 stages), so they
# take the four-step path too.
LARGE_C2C = [15552, 15625, 16000, 20000, 24576, 32768, 40000, 65536]


@pytest.mark.parametrize("n", LARGE_C2C)
@pytest.mark.parametrize("inverse", [False, True])
def test_four_step_c2c(cuda, n, inverse):
    """Transforms longer than one CTA: the four-step path through per-CTA scratch."""
    import fastandfourier_b200 as F
    t, e_orc, e_64 = _c2c_case(cuda, F, n, inverse, batch=2)
    assert t.kind == "c2c-4step"
    assert e_orc <= REL_L2_TOL and e_64 <= REL_L2_TOL, (n, e_orc, e_64)


def test_four_step_persistent_batch(cuda):
    """More transforms than resident CTAs: every CTA loops over several."""
    import fastandfourier_b200 as F
    torch = cuda
    n, batch = 32768, 300
    rng = seeded(77)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    t = F.Transform.fft(n, norm=F.N_ORTHO)
    yr, yi = t.c2c(dev(torch, re), dev(torch, im))
    want = orc.fp64_c2c(re, im, norm=2)
    assert orc.rel_l2_complex(host(yr), host(yi), want) <= REL_L2_TOL


@pytest.mark.parametrize("n", [31250, 32000, 40000, 65536])
def test_four_step_real(cuda, n):
    import fastandfourier_b200 as F
    torch = cuda
    x = seeded(300 + n).standard_normal((3, n)).astype(np.float32)
    fwd = F.Transform.rfft(n)
    Xr, Xi = fwd.r2c(dev(torch, x))
    assert orc.rel_l2_complex(host(Xr), host(Xi), orc.fp64_r2c(x)) <= REL_L2_TOL
    y = host(fwd.inverse().c2r(Xr, Xi))
    assert orc.rel_l2(y, x) <= REL_L2_TOL
    p = F.Transform.chirp(f"(pipeline (rfft :size {n}) conj (bandpass :lo 5 :hi 9000) (irfft))")
    yp = host(p.pipeline(dev(torch, x)))
    assert orc.rel_l2(yp, orc.pipeline(x, [(1, 0, 0), (3, 5, 9000)])) <= REL_L2_TOL


def test_host_buffers_chunked_overlap(cuda):
    """Host buffers above the chunking threshold run through the overlapped
    copy / kernel / copy ring; results equal the device-buffer path."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(515)
    x = rng.standard_normal((3000, 4096)).astype(np.float32)  # 48 MB in
    t = F.Transform.rfft(4096)
    hr, hi = t.r2c(x)  # host numpy in and out
    dr, di = t.r2c(torch.from_numpy(x).cuda())
    assert np.array_equal(hr, dr.cpu().numpy()) and np.array_equal(hi, di.cpu().numpy())
    p = F.Transform.chirp("(pipeline (rfft :size 4096) conj (irfft))")
    y = p.pipeline(x)
    assert np.array_equal(y, p.pipeline(torch.from_numpy(x).cuda()).cpu().numpy())
    re = rng.uniform(-1, 1, (1500, 4096)).astype(np.float32)
    im = rng.uniform(-1, 1, (1500, 4096)).astype(np.float32)
    c = F.Transform.fft(4096)
    yr, yi = c.c2c(re, im)
    want = orc.fp64_c2c(re[:4], im[:4])
    assert orc.rel_l2_complex(yr[:4], yi[:4], want) <= REL_L2_TOL
    gr, gi = c.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    assert np.array_equal(yr, gr.cpu().numpy()) and np.array_equal(yi, gi.cpu().numpy())
    s = F.Transform.stft(1024, win=1024, hop=256)
    xs = rng.standard_normal((40, 1 << 17)).astype(np.float32)  # 20 MB in
    sr, si = s.stft_frames(xs)
    dr2, di2 = s.stft_frames(torch.from_numpy(xs).cuda())
    assert np.array_equal(sr, dr2.cpu().numpy()) and np.array_equal(si, di2.cpu().numpy())


def test_host_buffers_on_four_step_and_host_mask(cuda):
    """Host buffers through the paths that grow device scratch inside the
    execute (four-step scratch, a host-bound spectrum): results equal the
    device-buffer path."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(616)
    re = rng.uniform(-1, 1, (3, 32768)).astype(np.float32)
    im = rng.uniform(-1, 1, (3, 32768)).astype(np.float32)
    c = F.Transform.fft(32768)
    hr, hi = c.c2c(re, im)
    dr, di = c.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    assert np.array_equal(hr, dr.cpu().numpy()) and np.array_equal(hi, di.cpu().numpy())
    x = rng.standard_normal((2, 65536)).astype(np.float32)
    r = F.Transform.rfft(65536)
    Xr, Xi = r.r2c(x)
    assert orc.rel_l2_complex(Xr, Xi, orc.fp64_r2c(x)) <= REL_L2_TOL
    m = np.linspace(0, 1, 2049).astype(np.float32)
    p = F.Transform.chirp("(pipeline (rfft :size 4096) (mul-spectrum) (irfft))")
    p.bind(m, np.zeros_like(m), 2049)  # host H, host signal
    xs = rng.standard_normal((5, 4096)).astype(np.float32)
    y = p.pipeline(xs)
    assert orc.rel_l2(y, orc.pipeline(xs, [(orc.OP_MUL, 0, 0)], m, np.zeros_like(m))) <= REL_L2_TOL


@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_16384_two_pass_four_step(cuda, monkeypatch, inverse):
    """FAF_CUDA_FOURSTEP_16K=1 runs the 16384-point C2C as the multi-CTA
    128 x 128 two-pass four-step instead of one CTA per transform."""
    import fastandfourier_b200 as F
    monkeypatch.setenv("FAF_CUDA_FOURSTEP_16K", "1")
    torch = cuda
    n = 16384
    rng = seeded(161 + inverse)
    re = rng.uniform(-1, 1, (5, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (5, n)).astype(np.float32)
    t = F.Transform.fft(n, inverse=inverse)
    assert t.kind == "c2c-4step"
    yr, yi = t.c2c(dev(torch, re), dev(torch, im))
    want = orc.fp64_c2c(re, im, inverse=inverse)
    assert orc.rel_l2_complex(host(yr), host(yi), want) <= REL_L2_TOL


@pytest.mark.parametrize("n", [32768, 65536])
@pytest.mark.parametrize("threads", ["512", "1024"])
def test_four_step_cta_widths_agree(cuda, monkeypatch, n, threads):
    """The two-pass four-step gives the same values with CTAs of 256 (the
    standalone default), 512 (the uneven graph's) and 1024 threads: each
    column and row runs the same arithmetic."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(n)
    re = rng.uniform(-1, 1, (150, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (150, n)).astype(np.float32)
    t = F.Transform.fft(n)
    ar, ai = t.c2c(dev(torch, re), dev(torch, im))
    monkeypatch.setenv("FAF_CUDA_4STEP_THREADS", threads)
    br, bi = t.c2c(dev(torch, re), dev(torch, im))
    assert torch.equal(ar, br) and torch.equal(ai, bi)
    assert orc.rel_l2_complex(host(ar), host(ai), orc.fp64_c2c(re, im)) <= REL_L2_TOL
