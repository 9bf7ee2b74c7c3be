"""The input landing ring of the power-of-two R2C and pipeline kernels (inputs
land in shared-memory slots by bulk copy, a slot cycle ahead of use): parity
against FP64 numpy over ragged batches and input distances, the direct-load
path for distances the bulk copy cannot take, and a clean wait status."""
import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu


def rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


def _strided(torch, x, dist):
    """(batch, n) rows placed `dist` floats apart in one device buffer."""
    b, n = x.shape
    buf = torch.zeros(b * dist, dtype=torch.float32, device="cuda")
    buf.view(b, dist)[:, :n] = torch.from_numpy(x).cuda()
    return buf


@pytest.mark.parametrize("n", [64, 1024, 4096, 8192])
@pytest.mark.parametrize("batch", [1, 5, 1187, 8192 + 13])
def test_r2c_ring_batches(cuda, n, batch):
    import fastandfourier_b200 as F
    torch = cuda
    x = seeded(n + batch).standard_normal((batch, n)).astype(np.float32)
    t = F.Transform.rfft(n)
    Xr, Xi = t.r2c(torch.from_numpy(x).cuda())
    want = np.fft.rfft(x.astype(np.float64), axis=-1)
    assert rel(Xr.cpu().numpy() + 1j * Xi.cpu().numpy(), want) <= REL_L2_TOL
    assert t.wait_status() == 0


@pytest.mark.parametrize("dist_pad", [1, 2, 4, 12])
def test_r2c_ring_and_direct_distances(cuda, dist_pad):
    """dist % 4 == 0 takes the ring, other distances the direct loads."""
    import fastandfourier_b200 as F
    torch = cuda
    n, batch = 4096, 700
    dist = n + dist_pad
    x = seeded(dist).standard_normal((batch, n)).astype(np.float32)
    buf = _strided(torch, x, dist)
    nb = n // 2 + 1
    Xr = torch.empty(batch * nb, device="cuda")
    Xi = torch.empty(batch * nb, device="cuda")
    t = F.Transform.rfft(n)
    t.execute_batched(F._buf(Xr, Xi, nb, F.L_HERMITIAN), F._buf(buf, None, n, F.L_REAL), batch,
                      in_dist=dist, out_dist=nb)
    got = Xr.cpu().numpy().reshape(batch, nb) + 1j * Xi.cpu().numpy().reshape(batch, nb)
    assert rel(got, np.fft.rfft(x.astype(np.float64), axis=-1)) <= REL_L2_TOL
    assert t.wait_status() == 0


@pytest.mark.parametrize("n", [64, 128, 256, 512])
@pytest.mark.parametrize("batch", [1, 5, 1187, 20000 + 3])
@pytest.mark.parametrize("inter", [False, True])
def test_r2c_landed_short_lengths_match_direct_loads(cuda, monkeypatch, n, batch, inter):
    """Groups narrower than a warp: R2C of 512 samples lands each
    transform's samples in its group's workspace, and 64 to 256 samples stage
    their spectra in shared memory and write them row by row.  Both are
    bit-identical to k2_r2c's direct loads and stores and equal FP64 within
    the tolerance, for split and interleaved spectra."""
    import fastandfourier_b200 as F
    torch = cuda
    x = seeded(n + batch).standard_normal((batch, n)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    nb = n // 2 + 1

    def run():
        t = F.Transform.rfft(n, layout=F.L_INTERLEAVED if inter else F.L_DEFAULT)
        if inter:
            y = t.r2c(xd).cpu().numpy().reshape(batch, nb, 2)
            got = y[..., 0] + 1j * y[..., 1]
        else:
            Xr, Xi = t.r2c(xd)
            got = Xr.cpu().numpy() + 1j * Xi.cpu().numpy()
        assert t.wait_status() == 0
        return got

    got = run()
    assert rel(got, np.fft.rfft(x.astype(np.float64), axis=-1)) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    assert np.array_equal(got, run())


@pytest.mark.parametrize("n", [64, 128, 512])
@pytest.mark.parametrize("dist_pad,out_pad", [(1, 0), (2, 3), (3, 1)])
def test_r2c_short_odd_distances(cuda, n, dist_pad, out_pad):
    """Input distances of odd floats (transform starts 4-byte aligned) take
    the direct loads at 512 samples; even ones land.  The staged spectra of
    64 and 128 samples go to rows `nb + out_pad` apart.  All match FP64."""
    import fastandfourier_b200 as F
    torch = cuda
    batch = 999
    dist = n + dist_pad
    x = seeded(dist + n).standard_normal((batch, n)).astype(np.float32)
    buf = _strided(torch, x, dist)
    nb = n // 2 + 1
    od = nb + out_pad
    Xr = torch.full((batch * od,), 7.0, device="cuda")
    Xi = torch.full((batch * od,), 7.0, device="cuda")
    t = F.Transform.rfft(n)
    t.execute_batched(F._buf(Xr, Xi, nb, F.L_HERMITIAN), F._buf(buf, None, n, F.L_REAL), batch,
                      in_dist=dist, out_dist=od)
    yr = Xr.cpu().numpy().reshape(batch, od)
    yi = Xi.cpu().numpy().reshape(batch, od)
    got = yr[:, :nb] + 1j * yi[:, :nb]
    assert rel(got, np.fft.rfft(x.astype(np.float64), axis=-1)) <= REL_L2_TOL
    assert np.all(yr[:, nb:] == 7.0) and np.all(yi[:, nb:] == 7.0)  # gaps untouched
    assert t.wait_status() == 0


@pytest.mark.parametrize("batch", [3, 640, 8192 + 7])
def test_pipeline_ring_batches(cuda, batch):
    import fastandfourier_b200 as F
    torch = cuda
    n, nb = 4096, 2049
    rng = seeded(batch)
    x = rng.standard_normal((batch, n)).astype(np.float32)
    m = rng.uniform(0, 1, nb).astype(np.float32)
    t = F.Transform.chirp("(pipeline (rfft :size 4096) (mul-spectrum) (irfft))")
    hm = torch.from_numpy(m).cuda()
    hz = torch.zeros(nb, device="cuda")
    t.bind(hm, hz, nb)
    y = t.pipeline(torch.from_numpy(x).cuda()).cpu().numpy()
    want = np.fft.irfft(np.fft.rfft(x.astype(np.float64), axis=-1) * m, n=n, axis=-1)
    assert rel(y, want) <= REL_L2_TOL
    assert t.wait_status() == 0


def test_ring_off_matches_ring_on(cuda, monkeypatch):
    """FAF_CUDA_NO_STAGING=1 (direct loads) gives bit-identical results: the
    ring changes where the input comes from, not the arithmetic."""
    import fastandfourier_b200 as F
    torch = cuda
    x = torch.from_numpy(seeded(77).standard_normal((333, 4096)).astype(np.float32)).cuda()
    t = F.Transform.rfft(4096)
    a_re, a_im = t.r2c(x)
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    b_re, b_im = t.r2c(x)
    assert torch.equal(a_re, b_re) and torch.equal(a_im, b_im)


@pytest.mark.parametrize("n,win,hop", [(1024, 1024, 256), (512, 400, 100), (2048, 2048, 512),
                                       (1024, 1000, 250)])
def test_stft_ring_matches_direct(cuda, monkeypatch, n, win, hop):
    """STFT frames landed by bulk copy (aligned frame starts, win % 4 == 0)
    equal the direct loads bit for bit; hop 250 (frame starts not 16-byte
    aligned) takes the direct path both times.  Both match FP64 numpy."""
    import fastandfourier_b200 as F
    torch = cuda
    L = 40000
    x = seeded(n + win + hop).standard_normal((3, L)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    t = F.Transform.stft(n, win=win, hop=hop)
    a_re, a_im = t.stft_frames(xd)
    assert t.wait_status() == 0
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    b_re, b_im = t.stft_frames(xd)
    assert torch.equal(a_re, b_re) and torch.equal(a_im, b_im)
    frames = 1 + (L - win) // hop
    k = np.arange(win)
    w = 0.5 * (1 - np.cos(2 * np.pi * k / (win - 1)))
    idx = np.arange(frames)[:, None] * hop + k[None, :]
    fr = np.zeros((3, frames, n))
    fr[:, :, :win] = x.astype(np.float64)[:, idx] * w
    want = np.fft.rfft(fr, axis=-1)
    got = a_re.cpu().numpy() + 1j * a_im.cpu().numpy()
    assert rel(got, want) <= REL_L2_TOL


@pytest.mark.parametrize("n", [32, 64, 128, 256, 1024, 2048, 16384, 32768])
def test_pipeline_sizes_fused_middle(cuda, n):
    """The pipeline's bin-pair pass fused into the forward FFT's last stage
    at every length whose real-kind radix order ends in 8, and the unfused
    pass elsewhere, against FP64 numpy."""
    import fastandfourier_b200 as F
    torch = cuda
    nb = n // 2 + 1
    rng = seeded(n + 17)
    x = rng.standard_normal((9, n)).astype(np.float32)
    m = rng.uniform(0, 1, nb).astype(np.float32)
    t = F.Transform.chirp(f"(pipeline (rfft :size {n}) (mul-spectrum) (irfft))")
    t.bind(torch.from_numpy(m).cuda(), torch.zeros(nb, device="cuda"), nb)
    y = t.pipeline(torch.from_numpy(x).cuda()).cpu().numpy()
    want = np.fft.irfft(np.fft.rfft(x.astype(np.float64), axis=-1) * m, n=n, axis=-1)
    assert rel(y, want) <= REL_L2_TOL


def _c2c_pair(torch, F, n, batch, inverse, inter, seed):
    rng = seeded(seed)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    t = F.Transform.fft(n, inverse=inverse, layout=F.L_INTERLEAVED if inter else F.L_DEFAULT)
    if inter:
        z = np.stack([re, im], axis=-1).reshape(batch, 2 * n)
        y = t.c2c(torch.from_numpy(z).cuda()).cpu().numpy().reshape(batch, n, 2)
        got = y[..., 0] + 1j * y[..., 1]
    else:
        yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
        got = yr.cpu().numpy() + 1j * yi.cpu().numpy()
    assert t.wait_status() == 0
    return re, im, got


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384])
@pytest.mark.parametrize("batch", [1, 3, 149, 300, 1500])
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_landed_inputs_match_direct_loads(cuda, monkeypatch, n, batch, inverse):
    """Power-of-two C2C of 64 to 16384 points lands each transform's planes
    in the workspace by bulk copy; the result equals the direct loads bit for
    bit (same arithmetic) and FP64 within the tolerance."""
    import fastandfourier_b200 as F
    torch = cuda
    re, im, got = _c2c_pair(torch, F, n, batch, inverse, False, n + batch)
    want = orc.fp64_c2c(re, im, inverse=inverse)
    assert rel(got, want) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    _, _, direct = _c2c_pair(torch, F, n, batch, inverse, False, n + batch)
    assert np.array_equal(got, direct)


def test_c2c_landed_interleaved_and_unaligned(cuda):
    """Interleaved 16384-point inputs land as one copy per transform; plane
    distances that are not a multiple of 4 floats land from the 16-byte block
    at or below each plane's start."""
    import fastandfourier_b200 as F
    torch = cuda
    n = 16384
    re, im, got = _c2c_pair(torch, F, n, 5, False, True, 3)
    assert rel(got, orc.fp64_c2c(re, im)) <= REL_L2_TOL
    batch, dist = 7, n + 2
    rng = seeded(4)
    xr = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    xi = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    br, bi = _strided(torch, xr, dist), _strided(torch, xi, dist)
    yr = torch.empty(batch * n, device="cuda")
    yi = torch.empty(batch * n, device="cuda")
    t = F.Transform.fft(n)
    t.execute_batched(F._buf(yr, yi, n, F.L_SPLIT), F._buf(br, bi, n, F.L_SPLIT), batch,
                      in_dist=dist, out_dist=n)
    got = yr.cpu().numpy().reshape(batch, n) + 1j * yi.cpu().numpy().reshape(batch, n)
    assert rel(got, orc.fp64_c2c(xr, xi)) <= REL_L2_TOL
    assert t.wait_status() == 0


@pytest.mark.parametrize("n", [64, 128, 256])
@pytest.mark.parametrize("inverse,inter", [(False, False), (True, False), (False, True)])
def test_c2c_staged_outputs_match_unstaged(cuda, monkeypatch, n, inverse, inter):
    """C2C of 64 points stages its outputs in shared memory and writes them
    row by row: bit-identical to the landed kernel's direct stores
    (FAF_CUDA_STAGE_OUT=0) and equal to FP64 within the tolerance; 128 and
    256 points store directly both times."""
    import fastandfourier_b200 as F
    torch = cuda
    re, im, got = _c2c_pair(torch, F, n, 5003, inverse, inter, n + 5)
    assert rel(got, orc.fp64_c2c(re, im, inverse=inverse)) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_STAGE_OUT", "0")
    _, _, plain = _c2c_pair(torch, F, n, 5003, inverse, inter, n + 5)
    assert np.array_equal(got, plain)


def test_c2c_staged_outputs_row_distance(cuda):
    """Staged 64-point outputs go to rows `n + 5` apart; the gaps stay."""
    import fastandfourier_b200 as F
    torch = cuda
    n, batch, od = 64, 3001, 69
    rng = seeded(64)
    xr = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    xi = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    yr = torch.full((batch * od,), 7.0, device="cuda")
    yi = torch.full((batch * od,), 7.0, device="cuda")
    t = F.Transform.fft(n)
    t.execute_batched(F._buf(yr, yi, n, F.L_SPLIT),
                      F._buf(torch.from_numpy(xr).cuda(), torch.from_numpy(xi).cuda(), n,
                             F.L_SPLIT), batch, in_dist=n, out_dist=od)
    a = yr.cpu().numpy().reshape(batch, od)
    b = yi.cpu().numpy().reshape(batch, od)
    assert np.all(a[:, n:] == 7.0) and np.all(b[:, n:] == 7.0)
    assert rel(a[:, :n] + 1j * b[:, :n], orc.fp64_c2c(xr, xi)) <= REL_L2_TOL
    assert t.wait_status() == 0


@pytest.mark.parametrize("n", [64, 128, 512, 1024])
def test_c2c_landed_interleaved_matches_direct_loads(cuda, monkeypatch, n):
    """Interleaved inputs of sub-warp, one-warp (512-point) and two-warp
    transforms land as one copy per transform, bit-identical to the direct
    loads."""
    import fastandfourier_b200 as F
    torch = cuda
    re, im, got = _c2c_pair(torch, F, n, 1187, False, True, 9)
    assert rel(got, orc.fp64_c2c(re, im)) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    _, _, direct = _c2c_pair(torch, F, n, 1187, False, True, 9)
    assert np.array_equal(got, direct)


@pytest.mark.parametrize("n", [64, 256, 512, 1024, 4096, 16384])
@pytest.mark.parametrize("shift,extra", [(1, 1), (2, 3), (3, 0), (0, 2)])
def test_c2c_landed_unaligned_planes_match_direct_loads(cuda, monkeypatch, n, shift, extra):
    """Planes `shift` floats past a 16-byte boundary and `n + extra` floats
    apart land from the block at or below each start: bit-identical to the
    direct loads, and to FP64 within the tolerance."""
    import fastandfourier_b200 as F
    torch = cuda
    batch, dist = 300, n + extra
    rng = seeded(20 + shift + n)
    xr = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    xi = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    br = torch.zeros(batch * dist + 8, device="cuda")
    bi = torch.zeros(batch * dist + 8, device="cuda")
    br[shift:shift + batch * dist].view(batch, dist)[:, :n] = torch.from_numpy(xr).cuda()
    bi[3 - shift % 4:3 - shift % 4 + batch * dist].view(batch, dist)[:, :n] = \
        torch.from_numpy(xi).cuda()
    ir, ii = br[shift:], bi[3 - shift % 4:]

    def run():
        yr = torch.empty(batch * n, device="cuda")
        yi = torch.empty(batch * n, device="cuda")
        t = F.Transform.fft(n)
        t.execute_batched(F._buf(yr, yi, n, F.L_SPLIT), F._buf(ir, ii, n, F.L_SPLIT), batch,
                          in_dist=dist, out_dist=n)
        assert t.wait_status() == 0
        return yr.cpu().numpy().reshape(batch, n) + 1j * yi.cpu().numpy().reshape(batch, n)

    got = run()
    assert rel(got, orc.fp64_c2c(xr, xi)) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    assert np.array_equal(got, run())


def test_c2c_landed_inputs_unaligned_outputs(cuda):
    """Aligned inputs land by bulk copy while outputs 2 floats apart from
    alignment take the scalar stores: same values as the aligned case."""
    import fastandfourier_b200 as F
    torch = cuda
    n, batch = 16384, 5
    rng = seeded(8)
    xr = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    xi = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    dr, di = torch.from_numpy(xr).cuda(), torch.from_numpy(xi).cuda()
    odist = n + 2
    yr = torch.empty(batch * odist, device="cuda")
    yi = torch.empty(batch * odist, device="cuda")
    t = F.Transform.fft(n)
    t.execute_batched(F._buf(yr, yi, n, F.L_SPLIT), F._buf(dr, di, n, F.L_SPLIT), batch,
                      in_dist=n, out_dist=odist)
    got = (yr.cpu().numpy().reshape(batch, odist)[:, :n]
           + 1j * yi.cpu().numpy().reshape(batch, odist)[:, :n])
    ar, ai = t.c2c(dr, di)
    assert np.array_equal(got, ar.cpu().numpy() + 1j * ai.cpu().numpy())
    assert rel(got, orc.fp64_c2c(xr, xi)) <= REL_L2_TOL
    assert t.wait_status() == 0


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 4096, 32768])
@pytest.mark.parametrize("batch", [1, 5, 1187])
@pytest.mark.parametrize("shift,extra", [(0, 0), (1, 2), (3, 5)])
def test_c2r_landed_bins_match_direct_loads(cuda, monkeypatch, n, batch, shift, extra):
    """C2R bins (n/2 + 1 per plane, `n/2 + 1 + extra` apart, planes `shift`
    floats off a 16-byte boundary) land by bulk copy from the block at or
    below each plane's start: bit-identical to the direct loads, and equal to
    FP64 within the tolerance."""
    import fastandfourier_b200 as F
    torch = cuda
    nb = n // 2 + 1
    dist = nb + extra
    rng = seeded(30 + n + shift)
    x = rng.standard_normal((batch, n))
    X = np.fft.rfft(x, axis=1)
    br = torch.zeros(batch * dist + 8, device="cuda")
    bi = torch.zeros(batch * dist + 8, device="cuda")
    br[shift:shift + batch * dist].view(batch, dist)[:, :nb] = torch.from_numpy(
        X.real.astype(np.float32)).cuda()
    bi[(shift + 2) % 4:(shift + 2) % 4 + batch * dist].view(batch, dist)[:, :nb] = \
        torch.from_numpy(X.imag.astype(np.float32)).cuda()
    ir, ii = br[shift:], bi[(shift + 2) % 4:]

    def run():
        y = torch.empty(batch * n, device="cuda")
        t = F.Transform.rfft(n, inverse=True)
        t.execute_batched(F._buf(y, None, n, F.L_REAL), F._buf(ir, ii, nb, F.L_HERMITIAN),
                          batch, in_dist=dist, out_dist=n)
        assert t.wait_status() == 0
        return y.cpu().numpy().reshape(batch, n)

    got = run()
    assert rel(got, x) <= REL_L2_TOL  # the inverse real transform's default 1/n
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    assert np.array_equal(got, run())


@pytest.mark.parametrize("n", [64, 128, 512, 1024, 4096])
def test_c2r_landed_interleaved_bins(cuda, monkeypatch, n):
    """Interleaved Hermitian input lands as one copy per transform."""
    import fastandfourier_b200 as F
    torch = cuda
    batch, nb = 600, n // 2 + 1
    rng = seeded(40 + n)
    x = rng.standard_normal((batch, n))
    X = np.fft.rfft(x, axis=1)
    z = torch.from_numpy(np.stack([X.real, X.imag], axis=-1).astype(np.float32)).cuda()

    def run():
        t = F.Transform.rfft(n, inverse=True, layout=F.L_INTERLEAVED)
        y = t.c2r(z)
        assert t.wait_status() == 0
        return y.cpu().numpy().reshape(batch, n)

    got = run()
    assert rel(got, x) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    assert np.array_equal(got, run())
