"""Host-side behaviour of the C ABI that needs no GPU: size policy, create-time
validation and messages (against the reference's own answers, golden
policy.json), Chirp front-end errors, backend selection, and the loud
failure when no CUDA device is present."""
import ctypes
import json
import os

import pytest

from conftest import ROOT

import fastandfourier_b200 as F

POLICY = json.load(open(os.path.join(ROOT, "tests", "golden", "policy.json")))


@pytest.mark.parametrize("ttype", ["0", "2"])
def test_size_policy_matches_reference(ttype):
    L = F.lib()
    sup = [int(L.faf_is_size_supported(int(ttype), n)) for n in POLICY["n"]]
    rec = [int(L.faf_get_recommended_size(int(ttype), n)) for n in POLICY["n"]]
    assert sup == POLICY["supported"][ttype]
    assert rec == POLICY["recommended"][ttype]


@pytest.mark.parametrize("probe", [p for p in POLICY["create"] if not p["ok"]],
                         ids=lambda p: f"t{p['type']}n{p['n']}f{p['flags']}")
def test_create_errors_match_reference(probe):
    L = F.lib()
    c = F.config(probe["n"], flags=probe["flags"])
    L.faf_clear_error()
    t = L.faf_create(probe["type"], ctypes.byref(c))
    assert not t
    assert F.C.error() == probe["error"]


def test_layout_and_norm_rejections():
    L = F.lib()
    for lay in (F.L_REAL, F.L_HERMITIAN):
        c = F.config(64, layout=lay)
        assert not L.faf_create_fft(ctypes.byref(c))
        assert "does not support layout" in F.C.error()
    c = F.config(64, norm=4)
    assert not L.faf_create_fft(ctypes.byref(c))
    assert "does not support norm 'lazy'" in F.C.error()
    c = F.config(64, layout=F.L_SPLIT)
    assert not L.faf_create_rfft(ctypes.byref(c))
    assert "R2C layout must be hermitian or interleaved" in F.C.error()


def test_cpu_backends_are_refused():
    L = F.lib()
    for b, name in ((1, "VM"), (2, "JIT")):
        c = F.config(64, backend=b)
        assert not L.faf_create_fft(ctypes.byref(c))
        assert name in F.C.error() and "FAF_BACKEND_CUDA" in F.C.error()


def test_fp64_only_where_available():
    """FP64 runs C2C, R2C and C2R; STFT (and the fused pipeline) stay FP32
    and refuse FP64 at create with a message."""
    L = F.lib()
    c = F.config(1024, hop=256, win=1024, precision=F.C.PREC_FP64)
    assert not L.faf_create_stft(ctypes.byref(c))
    assert "FP32" in F.C.error() and "FP64" in F.C.error()
    c = F.config(64, precision=F.C.PREC_FP16)
    assert not L.faf_create_fft(ctypes.byref(c))
    assert "not available" in F.C.error()


def test_length_cap():
    L = F.lib()
    c = F.config(65536 * 2)
    assert not L.faf_create_fft(ctypes.byref(c))
    assert "2^16" in F.C.error()


def test_outside_path_types_are_refused():
    L = F.lib()
    c = F.config(64)
    assert not L.faf_create(5, ctypes.byref(c))  # DCT-II
    assert "outside the CUDA transform path" in F.C.error()


@pytest.mark.parametrize("src,msg", [
    ("(pipeline (rfft :size 64) (foo) (irfft))", "only accepts spectral"),
    ("(pipeline (rfft :size 64) (spectral nosuch) (irfft))", "unknown spectral builtin"),
    ("(rfft :size 64 :bluestein)", "does not support :bluestein"),
    ("(rfft :size 64 :norm lazy)", "jpeg2000/lazy is not valid"),
    ("(rfft :size 64 :layout diagonal)", "unknown :layout"),
    ("(pipeline (rfft :size 64) (inverse :size 64))", "inherits size"),
    ("(pipeline (rfft :size 64", "failed to parse"),
    ("(dwt :size 64)", "outside the CUDA transform path"),
    ("(rfft :size 63)", "even and >= 2"),
])
def test_chirp_front_end_errors(src, msg):
    L = F.lib()
    assert not L.chirp_compile(src.encode())
    assert msg in F.C.error(), F.C.error()


def test_chirp_bind_slots():
    L = F.lib()
    t = F.C.faf_transform()
    buf = (ctypes.c_float * 4)()
    assert L.chirp_bind(ctypes.byref(t), b"H", buf, buf, 4) == 0
    assert t.user_aux_n == 4
    assert L.chirp_bind(ctypes.byref(t), b"Q", buf, buf, 4) != 0
    assert "unknown slot" in F.C.error()


def test_spectral_registry():
    L = F.lib()
    L.chirp_cleanup()
    cb = F.C.SPECTRAL_FN(lambda re, im, n, ctx: None)
    assert L.chirp_register_spectral(b"notch", cb, None) == 0
    assert L.chirp_register_spectral(b"notch", cb, None) == 0  # re-register keeps index
    assert L.chirp_count() == 1
    L.chirp_cleanup()
    assert L.chirp_count() == 0


def test_device_spectral_registry():
    """chirp_register_spectral_device: valid ops register (a name replaces an
    earlier host registration in place), invalid ones fail with a message;
    the host application of a device op is its definition on host bins."""
    import numpy as np
    L = F.lib()
    C = F.C
    L.chirp_cleanup()
    cb = C.SPECTRAL_FN(lambda re, im, n, ctx: None)
    assert L.chirp_register_spectral(b"shape", cb, None) == 0
    assert L.chirp_register_spectral_device(b"shape", C.CHIRP_DEVICE_GAIN, 0.5) == 0
    assert L.chirp_register_spectral_device(b"late", C.CHIRP_DEVICE_DELAY, 3.25) == 1
    assert L.chirp_count() == 2
    assert L.chirp_register_spectral_device(b"bad", 9, 1.0) == -1
    assert "unknown op" in C.error()
    assert L.chirp_register_spectral_device(b"bad", C.CHIRP_DEVICE_LOWPASS, -1.0) == -1
    assert L.chirp_register_spectral_device(b"", C.CHIRP_DEVICE_GAIN, 1.0) == -1
    # host application: gain 0.5, then a 3.25-sample circular delay (n = 16)
    nb, n = 9, 16
    rng = np.random.default_rng(5)
    re = rng.standard_normal(nb).astype(np.float32)
    im = rng.standard_normal(nb).astype(np.float32)
    t = C.faf_transform()
    t.n = n
    r2, i2 = re.copy(), im.copy()
    for idx in (0, 1):
        L.chirp_apply_split_f32(ctypes.byref(t), idx, 0, 0, r2.ctypes.data, i2.ctypes.data, nb)
    k = np.arange(nb)
    want = 0.5 * (re + 1j * im) * np.exp(-2j * np.pi * ((k * 3.25) % n) / n)
    assert np.allclose(r2 + 1j * i2, want, atol=1e-6)
    L.chirp_cleanup()


def test_host_helpers():
    import numpy as np
    L = F.lib()
    nb = 9
    rng = np.random.default_rng(0)
    xr, xi, hr, hi = (rng.standard_normal(nb).astype(np.float32) for _ in range(4))
    yr, yi = np.empty_like(xr), np.empty_like(xi)
    L.faf_herm_mul_f32(yr.ctypes.data, yi.ctypes.data, xr.ctypes.data, xi.ctypes.data,
                       hr.ctypes.data, hi.ctypes.data, nb)
    z = (xr + 1j * xi) * (hr + 1j * hi)
    assert np.allclose(yr[1:-1], z.real[1:-1], atol=1e-6)
    assert np.allclose(yi[1:-1], z.imag[1:-1], atol=1e-6)
    assert yi[0] == 0 and yi[-1] == 0 and np.isclose(yr[0], xr[0] * hr[0])
    inter = np.empty(2 * nb, np.float32)
    assert L.faf_interleave_f32(inter.ctypes.data, xr.ctypes.data, xi.ctypes.data, nb) == 0
    a, b = np.empty_like(xr), np.empty_like(xi)
    assert L.faf_deinterleave_f32(a.ctypes.data, b.ctypes.data, inter.ctypes.data, nb) == 0
    assert np.array_equal(a, xr) and np.array_equal(b, xi)


def test_no_gpu_means_no_transform():
    """Without a CUDA device the library refuses to create a transform rather
    than falling back to a CPU engine."""
    L = F.lib()
    if L.faf_cuda_available():
        pytest.skip("a CUDA device is present")
    c = F.config(1024)
    assert not L.faf_create_fft(ctypes.byref(c))
    assert "CUDA" in F.C.error()
    assert not L.chirp_compile(b"(pipeline (rfft :size 64) conj (irfft))")
    assert "CUDA" in F.C.error()


def test_names_and_version():
    L = F.lib()
    assert L.faf_version() == b"1.2.0"
    assert L.faf_layout_name(F.L_HERMITIAN) == b"hermitian"
    assert L.faf_norm_name(F.N_ORTHO) == b"ortho"
    assert L.faf_transform_name(F.T_PIPELINE) == b"pipeline"
    assert L.faf_precision_size(3) == 4


def test_uneven_rejects_illegal_lengths():
    with pytest.raises(F.FafError, match="legal faf_create_fft size"):
        F.Uneven([60, 23])
    with pytest.raises(F.FafError, match="empty"):
        F.Uneven([])


def test_stream_handles():
    """None is the library's synchronous default; torch's default stream
    (handle 0, the legacy stream) becomes cudaStreamLegacy so execution stays
    asynchronous on it; other handles pass through."""
    import fastandfourier_b200 as F

    class S:  # stands in for torch.cuda.Stream
        def __init__(self, h):
            self.cuda_stream = h

    assert F._stream_handle(None) is None
    assert F._stream_handle(0) is None
    assert F._stream_handle(S(0)) == F.CUDA_STREAM_LEGACY == 1
    assert F._stream_handle(S(0x7f00deadbe00)) == 0x7f00deadbe00
    assert F._stream_handle(0x5000) == 0x5000


def test_cwt_create_checks():
    """faf_cuda_create_cwt validates n, the bank and its stride before any
    device work, with the reference's wording where it has one."""
    import numpy as np
    import fastandfourier_b200 as F
    L = F.lib()
    psi = np.ones((2, 64), np.float32)
    p = psi.ctypes.data
    for n, rows, ptr, stride, msg in [(15, 2, p, 64, "even and 5-smooth"),
                                     (14, 2, p, 64, "even and 5-smooth"),
                                     (64, 0, p, 64, "at least one row"),
                                     (64, 2, None, 64, "at least one row"),
                                     (120, 2, p, 60, "shorter than the 61 packed bins")]:
        assert not L.faf_cuda_create_cwt(n, rows, ptr, stride)
        assert msg in F.C.error()
