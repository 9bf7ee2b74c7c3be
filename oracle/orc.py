"""ctypes bindings to the oracle C restatement (oracle/faf_oracle.c) and FP64
numpy references.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  The C restatement follows
the reference's own algorithms (file:line citations in faf_oracle.c); the FP64
functions are the exact DFT every result is also reported against.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

# Norm / op codes shared with faf_oracle.c (norms equal faf_norm values).
NORM_DEFAULT, NORM_NONE, NORM_ORTHO, NORM_FORWARD = 0, 1, 2, 3
OP_CONJ, OP_MUL, OP_BANDPASS, OP_MUL_CONJ = 1, 2, 3, 4
FLAG_BLUESTEIN = 1 << 12

_f32p = ctypes.POINTER(ctypes.c_float)


def build():
    """Compile liboracle.so with gcc (oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        sz, i, u32 = ctypes.c_size_t, ctypes.c_int, ctypes.c_uint32
        L.orc_error.restype = ctypes.c_char_p
        L.orc_c2c.argtypes = [sz, i, i, u32, _f32p, _f32p, _f32p, _f32p]
        L.orc_c2c_batch.argtypes = [sz, i, i, u32, sz, _f32p, _f32p, _f32p, _f32p]
        L.orc_r2c_batch.argtypes = [sz, i, sz, _f32p, _f32p, _f32p]
        L.orc_c2r_batch.argtypes = [sz, i, sz, _f32p, _f32p, _f32p]
        L.orc_pipeline.argtypes = [sz, i, i, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(u32), ctypes.POINTER(u32),
                                   _f32p, _f32p, sz, sz, _f32p, _f32p]
        L.orc_stft.argtypes = [sz, sz, sz, sz, sz, _f32p, _f32p, _f32p]
        L.orc_hann.argtypes = [_f32p, sz]
        for nm in ("orc_is_5_smooth", "orc_is_7_smooth", "orc_is_prime",
                   "orc_rader_eligible", "orc_is_codelet"):
            getattr(L, nm).argtypes = [sz]
            getattr(L, nm).restype = i
        L.orc_primitive_root.argtypes = [sz]
        L.orc_primitive_root.restype = sz
        L.orc_next_5_smooth.argtypes = [sz]
        L.orc_next_5_smooth.restype = sz
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_f32p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_error().decode())


def c2c(re, im, inverse=False, norm=NORM_NONE, flags=0):
    """Batched split-plane C2C; re/im shaped (..., n)."""
    re, im = _f32(re), _f32(im)
    n = re.shape[-1]
    batch = re.size // n if n else 0
    yr, yi = np.empty_like(re), np.empty_like(im)
    _check(lib().orc_c2c_batch(n, int(inverse), norm, flags, batch,
                               _p(re), _p(im), _p(yr), _p(yi)))
    return yr, yi


def r2c(x, norm=NORM_NONE):
    x = _f32(x)
    n = x.shape[-1]
    batch = x.size // n
    shp = x.shape[:-1] + (n // 2 + 1,)
    Xr, Xi = np.empty(shp, np.float32), np.empty(shp, np.float32)
    _check(lib().orc_r2c_batch(n, norm, batch, _p(x), _p(Xr), _p(Xi)))
    return Xr, Xi


def c2r(Xr, Xi, n, norm=NORM_NONE):
    Xr, Xi = _f32(Xr), _f32(Xi)
    nb = n // 2 + 1
    batch = Xr.size // nb
    y = np.empty(Xr.shape[:-1] + (n,), np.float32)
    _check(lib().orc_c2r_batch(n, norm, batch, _p(Xr), _p(Xi), _p(y)))
    return y


def pipeline(x, ops, hr=None, hi=None, norm=NORM_NONE):
    """ops: list of (op_code, lo, hi) tuples applied between R2C and C2R."""
    x = _f32(x)
    n = x.shape[-1]
    batch = x.size // n
    k = len(ops)
    op_a = (ctypes.c_int * max(k, 1))(*[o[0] for o in ops])
    lo_a = (ctypes.c_uint32 * max(k, 1))(*[o[1] for o in ops])
    hi_a = (ctypes.c_uint32 * max(k, 1))(*[o[2] for o in ops])
    hrp = hip = None
    hb = 0
    if hr is not None:
        hr, hi = _f32(hr), _f32(hi)
        hrp, hip, hb = _p(hr), _p(hi), hr.size
    y = np.empty_like(x)
    _check(lib().orc_pipeline(n, norm, k, op_a, lo_a, hi_a, hrp, hip, hb, batch,
                              _p(x), _p(y)))
    return y


def stft(x, n, win, hop):
    """Framed real STFT; x shaped (n_sig, L) -> (n_sig, frames, n//2+1)."""
    x = _f32(np.atleast_2d(x))
    n_sig, L = x.shape
    F = 1 + (L - win) // hop
    shp = (n_sig, F, n // 2 + 1)
    Xr, Xi = np.empty(shp, np.float32), np.empty(shp, np.float32)
    _check(lib().orc_stft(n, win, hop, L, n_sig, _p(x), _p(Xr), _p(Xi)))
    return Xr, Xi


def istft(Xr, Xi, n, win, hop):
    """Inverse STFT by weighted overlap-add, in FP64 (the reference has no
    inverse STFT: its faf_create_inverse of an STFT returns a forward STFT,
    src/faf_core.c:1122-1123).  Frames (n_sig, F, n//2+1) -> signals
    (n_sig, (F-1) hop + win): irfft of each frame, times the symmetric Hann
    window of the forward STFT (src/faf_twiddles.c:159-163), overlap-added and
    divided by the summed squared window (0 where it is below 1e-10)."""
    X = np.asarray(Xr, np.float64) + 1j * np.asarray(Xi, np.float64)
    X = X.reshape((-1,) + X.shape[-2:])
    n_sig, F, _ = X.shape
    frames = np.fft.irfft(X, n=n, axis=-1)[..., :win]
    i = np.arange(win)
    w = 0.5 * (1 - np.cos(2 * np.pi * i / (win - 1))) if win > 1 else np.ones(1)
    L = (F - 1) * hop + win
    y = np.zeros((n_sig, L))
    env = np.zeros(L)
    for f in range(F):
        y[:, f * hop:f * hop + win] += w * frames[:, f]
        env[f * hop:f * hop + win] += w * w
    return np.where(env > 1e-10, y / np.where(env > 1e-10, env, 1.0), 0.0)


def cwt(x, psi):
    """Forward CWT filter bank (src/faf_cwt.c:769-847): R2C of each signal
    once, then per bank row Y = X * psi_row with the DC and Nyquist
    imaginary parts zeroed (src/faf_cwt_kernels.c:22-33), then the C2R with
    the reference's NONE norm (1/n on the inverse).  x (batch, n), psi (rows,
    n/2+1) -> W (batch, rows, n), on the oracle's own R2C / C2R."""
    x = _f32(x)
    psi = _f32(psi)
    n = x.shape[-1]
    Xr, Xi = r2c(x)
    Yr = Xr[..., None, :] * psi
    Yi = Xi[..., None, :] * psi
    Yi[..., 0] = 0.0
    Yi[..., -1] = 0.0
    return c2r(Yr, Yi, n)


def cwt_dual(psi, eps=1e-6):
    """Dual-frame rows of a bank (src/faf_cwt.c:440-482): psi_r / (sum_r
    psi_r^2 + eps), the sum in FP64, zero where it is 0."""
    p = np.asarray(psi, np.float64)
    s = np.sum(p * p, axis=0)
    return np.where(s > 0, p / (s + eps), 0.0).astype(np.float32)


def icwt_dual(W, dual):
    """Dual-frame inverse CWT (src/faf_cwt.c:935-985): the R2C of every row,
    acc = sum over rows (in order) of Y_r * dual_r, DC / Nyquist imaginary
    parts zeroed, then the C2R (1/n).  W (batch, rows, n) -> (batch, n)."""
    W = _f32(W)
    n = W.shape[-1]
    Yr, Yi = r2c(W)
    d = _f32(dual)
    ar = np.zeros(Yr.shape[:-2] + Yr.shape[-1:], np.float32)
    ai = np.zeros_like(ar)
    for r in range(W.shape[-2]):
        ar += Yr[..., r, :] * d[r]
        ai += Yi[..., r, :] * d[r]
    ai[..., 0] = 0.0
    ai[..., -1] = 0.0
    return c2r(ar, ai, n)


def icwt_l1(W, has_lowpass, dlog, C):
    """L1 one-integral inverse CWT (src/faf_cwt.c:879-930), FP32 in the
    reference's order."""
    W = _f32(W)
    lo = 1 if has_lowpass else 0
    acc = np.zeros(W.shape[:-2] + W.shape[-1:], np.float32)
    dl = np.float32(dlog)
    for r in range(lo, W.shape[-2]):
        acc += W[..., r, :] * dl
    acc /= np.float32(C if C > 0 else 1.0)
    if has_lowpass:
        acc += W[..., 0, :]
    return acc


def fp64_cwt(x, psi):
    """The same bank in FP64 numpy."""
    n = x.shape[-1]
    X = np.fft.rfft(np.asarray(x, np.float64), axis=-1)
    return np.fft.irfft(X[..., None, :] * np.asarray(psi, np.float64), n=n, axis=-1)


def hann(n):
    w = np.empty(n, np.float32)
    lib().orc_hann(_p(w), n)
    return w


# ---- FP64 references (exact DFT up to double rounding) ------------------

def norm_scale(norm, inverse, n):
    if norm == NORM_ORTHO:
        return 1.0 / np.sqrt(n)
    if norm == NORM_FORWARD:
        return 1.0 if inverse else 1.0 / n
    return 1.0 / n if inverse else 1.0


def fp64_c2c(re, im, inverse=False, norm=NORM_NONE):
    z = np.asarray(re, np.float64) + 1j * np.asarray(im, np.float64)
    n = z.shape[-1]
    Z = (np.fft.ifft(z, axis=-1) * n) if inverse else np.fft.fft(z, axis=-1)
    return Z * norm_scale(norm, inverse, n)


def fp64_r2c(x, norm=NORM_NONE):
    n = np.shape(x)[-1]
    return np.fft.rfft(np.asarray(x, np.float64), axis=-1) * norm_scale(norm, False, n)


def fp64_c2r(Xr, Xi, n, norm=NORM_NONE):
    # The reference C2R ignores the imaginary parts of DC and Nyquist
    # (src/faf_rfft.c:125-126), as does numpy's irfft.
    X = np.asarray(Xr, np.float64) + 1j * np.asarray(Xi, np.float64)
    return np.fft.irfft(X, n=n, axis=-1) * n * norm_scale(norm, True, n)


def rel_l2(got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    num = np.linalg.norm((got - want).ravel())
    den = np.linalg.norm(np.asarray(want).ravel())
    return float(num / den) if den > 0 else float(num)


def rel_l2_complex(gr, gi, want):
    return rel_l2(np.asarray(gr, np.float64) + 1j * np.asarray(gi, np.float64), want)
