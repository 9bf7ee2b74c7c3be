"""FP64 transforms (FAF_PREC_FP64): C2C, R2C and C2R on the FP64 engine
against numpy's FP64 FFT (rel L2 <= 1e-12), device and host buffers, and the
sizes / kinds that stay FP32-only refused at create."""
import numpy as np
import pytest

from conftest import seeded

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(got, want):
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


@pytest.mark.parametrize("n", [2, 12, 16, 60, 1000, 1024, 4096, 6000, 8192])
@pytest.mark.parametrize("inverse", [False, True])
def test_fp64_c2c(cuda, n, inverse):
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(900 + n)
    re = rng.uniform(-1, 1, (5, n))
    im = rng.uniform(-1, 1, (5, n))
    t = F.Transform.fft(n, inverse=inverse, precision=F.PREC_FP64)
    yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    z = re + 1j * im
    want = np.fft.ifft(z, axis=-1) if inverse else np.fft.fft(z, axis=-1)
    assert yr.dtype == torch.float64
    assert rel(yr.cpu().numpy() + 1j * yi.cpu().numpy(), want) <= TOL64
    hr, hi = t.c2c(re, im)  # host buffers
    assert rel(hr + 1j * hi, want) <= TOL64


@pytest.mark.parametrize("n", [60, 1024, 4096])
def test_fp64_c2c_vs_reference(cuda, n):
    """Against the reference's own FP64 C2C (src/faf_core.c:521, FAF_PREC_FP64),
    compiled from its sources into the oracle's reference library."""
    import fastandfourier_b200 as F
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference library not built")
    rng = seeded(980 + n)
    re = rng.uniform(-1, 1, (6, n))
    im = rng.uniform(-1, 1, (6, n))
    for inverse in (False, True):
        t = F.Transform.fft(n, inverse=inverse, precision=F.PREC_FP64)
        gr, gi = t.c2c(re, im)
        wr, wi = refimpl.c2c64(re, im, inverse=inverse)
        assert rel(gr + 1j * gi, wr + 1j * wi) <= TOL64


def test_fp64_c2c_interleaved(cuda):
    import fastandfourier_b200 as F
    rng = seeded(950)
    z = rng.standard_normal((3, 480)) + 1j * rng.standard_normal((3, 480))
    t = F.Transform.fft(480, layout=F.L_INTERLEAVED, precision=F.PREC_FP64)
    y = t.c2c(np.ascontiguousarray(z.view(np.float64).reshape(3, 960)))
    got = y.reshape(3, 480, 2)
    assert rel(got[..., 0] + 1j * got[..., 1], np.fft.fft(z, axis=-1)) <= TOL64


@pytest.mark.parametrize("n", [2, 64, 1000, 4096, 16384])
def test_fp64_real(cuda, n):
    import fastandfourier_b200 as F
    torch = cuda
    x = seeded(960 + n).standard_normal((4, n))
    fwd = F.Transform.rfft(n, precision=F.PREC_FP64)
    Xr, Xi = fwd.r2c(torch.from_numpy(x).cuda())
    want = np.fft.rfft(x, axis=-1)
    assert rel(Xr.cpu().numpy() + 1j * Xi.cpu().numpy(), want) <= TOL64
    inv = F.Transform.rfft(n, inverse=True, precision=F.PREC_FP64)
    y = inv.c2r(Xr, Xi).cpu().numpy()
    assert rel(y, x) <= TOL64


def test_fp64_host_chunked(cuda):
    """Host buffers above the chunking threshold (doubles: 8-byte values)."""
    import fastandfourier_b200 as F
    x = seeded(970).standard_normal((700, 4096))  # 22 MB in
    fwd = F.Transform.rfft(4096, precision=F.PREC_FP64)
    Xr, Xi = fwd.r2c(x)
    assert rel(Xr + 1j * Xi, np.fft.rfft(x, axis=-1)) <= TOL64


def test_fp64_refused_where_unavailable(cuda):
    import fastandfourier_b200 as F
    for n in (17, 32768):  # Rader prime; beyond one 512-thread CTA
        with pytest.raises(F.FafError):
            F.Transform.fft(n, precision=F.PREC_FP64)
    with pytest.raises(F.FafError):
        F.Transform.chirp("(pipeline (rfft :size 4096 :precision f64) conj (irfft))")
