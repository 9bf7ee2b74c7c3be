"""ctypes bindings to the reference library itself (oracle/_ref/libfaf_ref_*.so),
compiled from the reference's own C sources by `make -C oracle ref`.

TEST / BASELINE INFRASTRUCTURE ONLY (see oracle/__init__.py).  Used to pin the
C restatement, to generate golden fixtures (in the container that has the
reference sources) and as the timed CPU baseline (`bench.py --impl
reference`).  The library is prebuilt; the GPU host only loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_DIR = os.path.join(_HERE, "_ref")
# Where the reference's sources are (needed only to compile oracle/_ref;
# the GPU host loads the prebuilt library).
REFERENCE_SRC = os.environ.get("FAF_REFERENCE_SRC", "")
_lib = None
_isa = None
_f32p = ctypes.POINTER(ctypes.c_float)


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = line.split()
                    return "avx512f" in fl and "avx512bw" in fl and "avx512vl" in fl
    except OSError:
        pass
    return False


def isa():
    return "v4" if _cpu_has_avx512() else "v3"


def lib_path():
    return os.path.join(_REF_DIR, f"libfaf_ref_{isa()}.so")


def available():
    return os.path.exists(lib_path())


def sources_present():
    return bool(REFERENCE_SRC) and os.path.isdir(os.path.join(REFERENCE_SRC, "src"))


def build():
    """Compile the reference library from its sources (needs the sources)."""
    if not REFERENCE_SRC:
        raise RuntimeError("FAF_REFERENCE_SRC is not set: point it at the reference's source "
                           "tree to compile oracle/_ref (the prebuilt library is used otherwise)")
    if not sources_present():
        raise RuntimeError(f"FAF_REFERENCE_SRC={REFERENCE_SRC!r} holds no reference sources")
    subprocess.run(["make", "-s", "-j8", "-C", _HERE, "ref", f"REF={REFERENCE_SRC}"],
                   check=True)


def lib():
    global _lib, _isa
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            build()
        # The pipeline JIT writes under $HOME/.cache/fastandfourier.
        os.environ.setdefault("HOME", "/tmp")
        L = ctypes.CDLL(path)
        sz, i, u32 = ctypes.c_size_t, ctypes.c_int, ctypes.c_uint32
        L.refdrv_error.restype = ctypes.c_char_p
        L.refdrv_c2c.argtypes = [sz, i, i, u32, sz, _f32p, _f32p, _f32p, _f32p, i]
        L.refdrv_r2c.argtypes = [sz, i, sz, _f32p, _f32p, _f32p, i]
        f64p = ctypes.POINTER(ctypes.c_double)
        L.refdrv_c2c64.argtypes = [sz, i, i, sz, f64p, f64p, f64p, f64p, i]
        L.refdrv_c2r.argtypes = [sz, i, sz, _f32p, _f32p, _f32p, i]
        L.refdrv_pipeline.argtypes = [ctypes.c_char_p, sz, _f32p, _f32p, sz, sz,
                                      _f32p, _f32p, i]
        L.refdrv_stft.argtypes = [sz, sz, sz, sz, sz, _f32p, _f32p, _f32p, i]
        szp = ctypes.POINTER(sz)
        L.refdrv_cwt_bank.argtypes = [sz, szp, szp, ctypes.POINTER(i), _f32p]
        L.refdrv_cwt.argtypes = [sz, sz, _f32p, _f32p, i]
        L.refdrv_cwt_consts.argtypes = [sz, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_uint)]
        L.refdrv_icwt.argtypes = [sz, i, sz, _f32p, _f32p, i]
        L.refdrv_is_size_supported.argtypes = [i, sz]
        L.refdrv_recommended_size.argtypes = [i, sz]
        L.refdrv_recommended_size.restype = sz
        L.refdrv_try_create.argtypes = [i, sz, u32, i, ctypes.c_char_p, sz]
        vp = ctypes.c_void_p
        for name, args in (("refdrv_open_c2c", [sz, i, i, u32, i, i]),
                           ("refdrv_open_r2c", [sz, i, i]),
                           ("refdrv_open_pipeline", [ctypes.c_char_p, sz, _f32p, _f32p, sz, i]),
                           ("refdrv_open_stft", [sz, sz, sz, sz, i]),
                           ("refdrv_open_cwt", [sz, i]),
                           ("refdrv_open_icwt", [sz, i, i])):
            f = getattr(L, name)
            f.argtypes, f.restype = args, vp
        L.refdrv_session_run.argtypes = [vp, sz, vp, vp, vp, vp]
        L.refdrv_session_threads.argtypes = [vp]
        L.refdrv_session_close.argtypes = [vp]
        _lib = L
        _isa = isa()
    return _lib


def _p(a):
    return a.ctypes.data_as(_f32p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + lib().refdrv_error().decode())


def c2c(re, im, inverse=False, norm=1, flags=0, threads=1):
    re, im = _f32(re), _f32(im)
    n = re.shape[-1]
    yr, yi = np.empty_like(re), np.empty_like(im)
    _check(lib().refdrv_c2c(n, int(inverse), norm, flags, re.size // n,
                            _p(re), _p(im), _p(yr), _p(yi), threads))
    return yr, yi


def c2c64(re, im, inverse=False, norm=1, threads=1):
    """The reference's FP64 C2C (FAF_PREC_FP64) on double split planes."""
    re = np.ascontiguousarray(re, dtype=np.float64)
    im = np.ascontiguousarray(im, dtype=np.float64)
    n = re.shape[-1]
    yr, yi = np.empty_like(re), np.empty_like(im)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    _check(lib().refdrv_c2c64(n, int(inverse), norm, re.size // n, p(re), p(im), p(yr), p(yi),
                              threads))
    return yr, yi


def r2c(x, norm=1, threads=1):
    x = _f32(x)
    n = x.shape[-1]
    shp = x.shape[:-1] + (n // 2 + 1,)
    Xr, Xi = np.empty(shp, np.float32), np.empty(shp, np.float32)
    _check(lib().refdrv_r2c(n, norm, x.size // n, _p(x), _p(Xr), _p(Xi), threads))
    return Xr, Xi


def c2r(Xr, Xi, n, norm=1, threads=1):
    Xr, Xi = _f32(Xr), _f32(Xi)
    y = np.empty(Xr.shape[:-1] + (n,), np.float32)
    _check(lib().refdrv_c2r(n, norm, Xr.size // (n // 2 + 1), _p(Xr), _p(Xi), _p(y),
                            threads))
    return y


def pipeline(src, x, hr=None, hi=None, threads=1):
    x = _f32(x)
    n = x.shape[-1]
    y = np.empty_like(x)
    hrp = hip = None
    hb = 0
    if hr is not None:
        hr, hi = _f32(hr), _f32(hi)
        hrp, hip, hb = _p(hr), _p(hi), hr.size
    _check(lib().refdrv_pipeline(src.encode(), n, hrp, hip, hb, x.size // n,
                                 _p(x), _p(y), threads))
    return y


def stft(x, n, win, hop, threads=1):
    x = _f32(np.atleast_2d(x))
    n_sig, L = x.shape
    F = 1 + (L - win) // hop
    shp = (n_sig, F, n // 2 + 1)
    Xr, Xi = np.empty(shp, np.float32), np.empty(shp, np.float32)
    _check(lib().refdrv_stft(n, win, hop, L, n_sig, _p(x), _p(Xr), _p(Xi), threads))
    return Xr, Xi


def cwt_bank(n):
    """The reference's default CWT bank for length n: (psi rows in execute
    order, (rows, n/2+1) float32; has_lowpass)."""
    rows, nb, lp = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int()
    _check(lib().refdrv_cwt_bank(n, ctypes.byref(rows), ctypes.byref(nb), ctypes.byref(lp), None))
    psi = np.empty((rows.value, nb.value), np.float32)
    _check(lib().refdrv_cwt_bank(n, None, None, None, _p(psi)))
    return psi, bool(lp.value)


def cwt(x, threads=1):
    """The reference's forward CWT (default bank) of signals x (batch, n):
    W (batch, rows, n)."""
    x = _f32(x)
    n = x.shape[-1]
    rows = cwt_bank(n)[0].shape[0]
    W = np.empty(x.shape[:-1] + (rows, n), np.float32)
    _check(lib().refdrv_cwt(n, x.size // n, _p(x), _p(W), threads))
    return W


def cwt_consts(n):
    """(admissibility C, voices) of the reference's default bank for n."""
    c, v = ctypes.c_double(), ctypes.c_uint()
    _check(lib().refdrv_cwt_consts(n, ctypes.byref(c), ctypes.byref(v)))
    return c.value, v.value


def icwt(W, kind=0, threads=1):
    """The reference's inverse CWT (kind 0 dual frame, 1 L1) of W (batch,
    rows, n) with its default bank: x (batch, n)."""
    W = _f32(W)
    n = W.shape[-1]
    x = np.empty(W.shape[:-2] + (n,), np.float32)
    _check(lib().refdrv_icwt(n, kind, x.size // n, _p(W), _p(x), threads))
    return x


def is_size_supported(ttype, n):
    return bool(lib().refdrv_is_size_supported(ttype, n))


def recommended_size(ttype, n):
    return int(lib().refdrv_recommended_size(ttype, n))


def try_create(ttype, n, flags=0, layout=0):
    buf = ctypes.create_string_buffer(512)
    ok = lib().refdrv_try_create(ttype, n, flags, layout, buf, 512)
    return bool(ok), buf.value.decode()


class Session:
    """Persistent reference workers for timing: `threads` threads, each with
    its own transform, created and warmed (pipeline JIT compiled) when the
    session opens.  run() executes a batch with nothing but faf_execute
    calls, split into contiguous slices over the threads.

    kind: "c2c", "c2c64", "r2c", "pipeline", "stft", "cwt", "icwt_dual".
    """

    def __init__(self, kind, n, threads=1, *, src=None, h=None, win=None, hop=None,
                 sig_len=None, inverse=False, norm=1, flags=0):
        L = lib()
        self.kind, self.n = kind, n
        self._keep = None
        if kind in ("c2c", "c2c64"):
            s = L.refdrv_open_c2c(n, int(inverse), norm, flags, int(kind == "c2c64"), threads)
        elif kind == "r2c":
            s = L.refdrv_open_r2c(n, norm, threads)
        elif kind == "pipeline":
            hr = hi = None
            hb = 0
            if h is not None:
                self._keep = (_f32(h[0]), _f32(h[1]), src.encode())
                hr, hi, hb = _p(self._keep[0]), _p(self._keep[1]), self._keep[0].size
            else:
                self._keep = (src.encode(),)
            s = L.refdrv_open_pipeline(self._keep[-1], n, hr, hi, hb, threads)
        elif kind == "stft":
            self.frames = 1 + (sig_len - win) // hop
            s = L.refdrv_open_stft(n, win, hop, sig_len, threads)
        elif kind == "cwt":
            s = L.refdrv_open_cwt(n, threads)
        elif kind == "icwt_dual":
            s = L.refdrv_open_icwt(n, 0, threads)
        else:
            raise ValueError(kind)
        if not s:
            raise RuntimeError("reference: " + L.refdrv_error().decode())
        self._s = s
        self.threads = L.refdrv_session_threads(s)

    def run(self, batch, in_re, in_im=None, out_re=None, out_im=None):
        """Execute `batch` transforms (STFT: signals) of C-contiguous arrays."""
        if self.kind == "stft":
            batch *= self.frames
        ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        _check(lib().refdrv_session_run(self._s, batch, ptr(in_re), ptr(in_im), ptr(out_re),
                                        ptr(out_im)))

    def close(self):
        if getattr(self, "_s", None):
            lib().refdrv_session_close(self._s)
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
