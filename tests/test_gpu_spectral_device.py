"""Device spectral ops (chirp_register_spectral_device): (spectral NAME) ops
that run inside the fused pipeline kernel, against FP64 and against the same
ops applied through the host-callback round trip."""
import ctypes

import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded

pytestmark = pytest.mark.gpu

N = 4096


def fp64_pipeline(x, gain, delay, cutoff):
    X = np.fft.rfft(x.astype(np.float64), axis=-1)
    k = np.arange(X.shape[-1])
    X = X * gain * np.exp(-2j * np.pi * ((k * delay) % N) / N)
    X[..., k > cutoff] = 0
    return np.fft.irfft(X, n=N, axis=-1)


def test_device_ops_fused_and_match_fp64(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    C, L = F.C, F.lib()
    L.chirp_cleanup()
    assert L.chirp_register_spectral_device(b"dgain", C.CHIRP_DEVICE_GAIN, 0.5) >= 0
    assert L.chirp_register_spectral_device(b"ddelay", C.CHIRP_DEVICE_DELAY, 37.25) >= 0
    assert L.chirp_register_spectral_device(b"dlow", C.CHIRP_DEVICE_LOWPASS, 900.0) >= 0
    p = F.Transform.chirp(f"(pipeline (rfft :size {N}) (spectral dgain) (spectral ddelay) "
                          "(spectral dlow) (irfft))")
    x = seeded(31).standard_normal((64, N)).astype(np.float32)
    y = p.pipeline(torch.from_numpy(x).cuda())
    assert L.faf_cuda_last_launches() == 1  # one fused kernel, no host round trip
    want = fp64_pipeline(x, 0.5, 37.25, 900)
    got = y.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= REL_L2_TOL
    L.chirp_cleanup()


def test_device_ops_equal_host_callback_path(cuda):
    """The same ops as a host callback (R2C kernel -> host -> C2R kernel)."""
    import fastandfourier_b200 as F
    torch = cuda
    C, L = F.C, F.lib()
    L.chirp_cleanup()
    L.chirp_register_spectral_device(b"dphase", C.CHIRP_DEVICE_PHASE, 0.7)
    L.chirp_register_spectral_device(b"dhigh", C.CHIRP_DEVICE_HIGHPASS, 12.0)

    def host_op(re, im, n, ctx):
        r = np.ctypeslib.as_array(re, (n,))
        i = np.ctypeslib.as_array(im, (n,))
        z = (r.astype(np.float64) + 1j * i) * np.exp(0.7j)
        z[:12] = 0
        r[:] = z.real
        i[:] = z.imag

    cb = C.SPECTRAL_FN(host_op)
    L.chirp_register_spectral(b"hostop", cb, None)
    x = seeded(32).standard_normal((16, N)).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    pd = F.Transform.chirp(f"(pipeline (rfft :size {N}) (spectral dphase) (spectral dhigh) "
                           "(irfft))")
    ph = F.Transform.chirp(f"(pipeline (rfft :size {N}) (spectral hostop) (irfft))")
    yd = pd.pipeline(dx).cpu().numpy()
    yh = ph.pipeline(dx).cpu().numpy()
    assert np.linalg.norm(yd - yh) / np.linalg.norm(yh) <= REL_L2_TOL
    # a pipeline with a host callback runs its device ops on the host too
    pm = F.Transform.chirp(f"(pipeline (rfft :size {N}) (spectral dphase) (spectral hostop) "
                           "(irfft))")
    ym = pm.pipeline(dx).cpu().numpy()
    X = np.fft.rfft(x.astype(np.float64)) * np.exp(1.4j)
    X[:, :12] = 0
    want = np.fft.irfft(X, n=N)
    assert np.linalg.norm(ym - want) / np.linalg.norm(want) <= REL_L2_TOL
    L.chirp_cleanup()
    del cb
