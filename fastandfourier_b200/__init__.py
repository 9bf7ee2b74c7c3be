"""fastandfourier_b200 -- B200 (sm_100a) implementation of FastAndFourier's
batched split-plane transform path behind the reference's C API.

The product is the C-ABI library libfaf_b200.so (include/fastandfourier.h,
include/chirp.h, include/faf_cuda.h).  This package is its Python host
mirror: `Transform` wraps one faf_transform * and runs it on torch CUDA
tensors (device pointers, on the current torch stream) or on numpy arrays
(host pointers, copied in and out by the library).  The operation names
follow the reference API (faf_create_fft / faf_create_rfft /
faf_create_stft / chirp_compile / chirp_bind / faf_execute).
"""
from __future__ import annotations

import ctypes

from . import _lib as C
from ._lib import (B_CUDA, DIR_FORWARD, DIR_INVERSE, FLAG_BLUESTEIN, FLAG_MEASURE,
                   FLAG_TENSOR_CORE, PREC_FP32, PREC_FP64,
                   L_DEFAULT, L_HERMITIAN, L_INTERLEAVED, L_REAL, L_SPLIT, N_DEFAULT,
                   N_FORWARD, N_NONE, N_ORTHO, T_CWT, T_FFT, T_ICWT, T_IFFT, T_IRFFT,
                   T_PIPELINE, T_RFFT, T_STFT)

__all__ = ["FafError", "Transform", "Uneven", "Server", "Request", "config", "lib", "available",
           "B_CUDA", "DIR_FORWARD", "DIR_INVERSE", "FLAG_TENSOR_CORE", "FLAG_BLUESTEIN",
           "FLAG_MEASURE", "PREC_FP32", "PREC_FP64", "L_DEFAULT", "L_HERMITIAN",
           "L_INTERLEAVED", "L_REAL", "L_SPLIT", "N_DEFAULT", "N_FORWARD", "N_NONE", "N_ORTHO",
           "T_CWT", "T_ICWT", "T_FFT", "T_IFFT", "T_IRFFT", "T_PIPELINE", "T_RFFT", "T_STFT"]


class FafError(RuntimeError):
    """A create / execute call of libfaf_b200.so failed (message from
    faf_get_error())."""


def lib():
    return C.lib()


def available():
    return bool(C.lib().faf_cuda_available())


def config(n, *, dir=DIR_FORWARD, norm=N_DEFAULT, layout=L_DEFAULT, flags=0, hop=0, win=0,
           backend=0, precision=None):
    c = C.faf_config()
    c.n = n
    c.precision = C.PREC_FP32 if precision is None else precision
    c.dir = dir
    c.norm = norm
    c.layout = layout
    c.flags = flags
    c.hop_length = hop
    c.win_length = win
    c.backend = backend
    return c


def _ptr(a):
    """Raw data pointer of a torch tensor or numpy array (must be float32 and
    contiguous)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    if hasattr(a, "ctypes"):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    raise TypeError(f"unsupported buffer type {type(a)!r}")


def _buf(re, im, n, layout):
    return C.faf_buffer(_ptr(re), _ptr(im), n, layout)


CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy: the legacy default stream as an explicit handle


def _stream_handle(stream):
    """cudaStream_t for the C ABI.  None (or a raw 0) is NULL: the library's
    default, synchronous execute.  A torch stream whose handle is 0 is torch's
    default stream, the legacy stream; it is passed as cudaStreamLegacy so
    that work is enqueued there without a host synchronisation."""
    if stream is None:
        return None
    h = getattr(stream, "cuda_stream", None)
    if h is None:
        return int(stream) or None
    return int(h) or CUDA_STREAM_LEGACY


def _check(rc):
    if rc != 0:
        raise FafError(C.error())


def _empty_like_batch(ref, shape):
    """Output of `shape` beside `ref`: same device (torch) or host (numpy),
    same floating type (float32, or float64 for FP64 transforms)."""
    if hasattr(ref, "data_ptr"):
        import torch
        return torch.empty(shape, dtype=ref.dtype, device=ref.device)
    import numpy as np
    return np.empty(shape, ref.dtype)


class Request:
    """One faf_request of the serving loop.  `chirp` names a real transform or
    pipeline; without it, stft=(n, win, hop) asks for a framed STFT.  Buffers
    are torch tensors or numpy arrays (host or device); they must stay alive
    until the request completes (the object keeps references)."""

    def __init__(self, x, out_re, out_im=None, *, chirp=None, stft=None, h=None,
                 stream_key=0):
        r = C.faf_request()
        self._chirp = chirp.encode() if chirp else None
        r.chirp = self._chirp
        if stft is not None:
            r.stft_n, r.stft_win, r.stft_hop = (int(v) for v in stft)
        if h is not None:
            r.h_re, r.h_im, r.h_len = _ptr(h[0]), _ptr(h[1]), int(h[2])
        n = x.numel() if hasattr(x, "numel") else x.size
        r.in_, r.in_len = _ptr(x), int(n)
        r.out_re, r.out_im = _ptr(out_re), _ptr(out_im)
        r.stream_key = int(stream_key)
        self.struct = r
        self.keep = (x, out_re, out_im, h)


class Server:
    """faf_server: continuous-batching request loop on one GPU."""

    def __init__(self, hbm_budget=0, streams=0, max_merge=0):
        c = C.faf_server_config(int(hbm_budget), int(streams), int(max_merge))
        self._p = C.lib().faf_server_create(ctypes.byref(c))
        if not self._p:
            raise FafError(C.error())
        self._live = {}

    def submit(self, req):
        rid = C.lib().faf_server_submit(self._p, ctypes.byref(req.struct))
        if rid < 0:
            raise FafError(C.error())
        self._live[rid] = req
        return rid

    def wait(self, rid):
        """(latency seconds, frames) of request rid, once it has completed."""
        lat, fr = ctypes.c_double(), ctypes.c_size_t()
        rc = C.lib().faf_server_wait(self._p, rid, ctypes.byref(lat), ctypes.byref(fr))
        self._live.pop(rid, None)
        _check(rc)
        return lat.value, fr.value

    def drain(self):
        _check(C.lib().faf_server_drain(self._p))

    def prepare(self, req):
        _check(C.lib().faf_server_prepare(self._p, ctypes.byref(req.struct)))

    def stream_frames(self, key, win, hop, in_len):
        return C.lib().faf_server_stream_frames(self._p, key, win, hop, in_len)

    def close_stream(self, key):
        _check(C.lib().faf_server_close_stream(self._p, key))

    def replay(self, reqs, arrivals):
        """Submit reqs at arrival times (seconds from now) from the library's
        own client loop; returns the per-request latencies."""
        n = len(reqs)
        arr = (C.faf_request * n)(*[r.struct for r in reqs])
        t = (ctypes.c_double * n)(*[float(a) for a in arrivals])
        lat = (ctypes.c_double * n)()
        _check(C.lib().faf_server_replay(self._p, arr, t, n, lat))
        return list(lat)

    def stats(self):
        st = C.faf_server_stats()
        _check(C.lib().faf_server_stats_get(self._p, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def reset_stats(self):
        C.lib().faf_server_stats_reset(self._p)

    def close(self):
        if self._p:
            C.lib().faf_server_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Uneven:
    """faf_uneven: many C2C transforms of different lengths, one persistent
    launch.  Ragged packed split planes (transform i at offset sum of the
    previous lengths)."""

    def __init__(self, lengths, *, inverse=False, norm=N_DEFAULT, measure=False,
                 tensor_core=False):
        self.lengths = [int(n) for n in lengths]
        arr = (ctypes.c_size_t * len(self.lengths))(*self.lengths)
        flags = (FLAG_MEASURE if measure else 0) | (FLAG_TENSOR_CORE if tensor_core else 0)
        c = config(0, dir=DIR_INVERSE if inverse else DIR_FORWARD, norm=norm, flags=flags)
        self._p = C.lib().faf_uneven_create(arr, len(self.lengths), ctypes.byref(c))
        if not self._p:
            raise FafError(C.error())

    @property
    def total(self):
        return C.lib().faf_uneven_total(self._p)

    def set_stream(self, stream):
        _check(C.lib().faf_uneven_set_stream(self._p, _stream_handle(stream)))

    def execute(self, re, im, out_re, out_im, plain=False):
        f = C.lib().faf_uneven_execute_plain if plain else C.lib().faf_uneven_execute
        _check(f(self._p, _ptr(out_re), _ptr(out_im), _ptr(re), _ptr(im)))
        return out_re, out_im

    def close(self):
        if self._p:
            C.lib().faf_uneven_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Transform:
    """One faf_transform * of libfaf_b200.so."""

    def __init__(self, ptr, keep=()):
        if not ptr:
            raise FafError(C.error())
        self._p = ptr
        self._keep = list(keep)
        # fixed at create: read once, not through ctypes on every call
        self._n = ptr.contents.n
        self._inter = ptr.contents.cfg.layout == L_INTERLEAVED
        self._xb = C.lib().faf_execute_batched

    # ---- constructors (reference names) ----
    @classmethod
    def fft(cls, n, *, inverse=False, norm=N_DEFAULT, layout=L_DEFAULT, flags=0, precision=None):
        c = config(n, dir=DIR_INVERSE if inverse else DIR_FORWARD, norm=norm, layout=layout,
                   flags=flags, precision=precision)
        return cls(C.lib().faf_create_fft(ctypes.byref(c)))

    @classmethod
    def rfft(cls, n, *, inverse=False, norm=N_DEFAULT, layout=L_DEFAULT, precision=None):
        c = config(n, dir=DIR_INVERSE if inverse else DIR_FORWARD, norm=norm, layout=layout,
                   precision=precision)
        return cls(C.lib().faf_create_rfft(ctypes.byref(c)))

    @classmethod
    def stft(cls, n, *, win=0, hop=0):
        c = config(n, hop=hop, win=win)
        return cls(C.lib().faf_create_stft(ctypes.byref(c)))

    @classmethod
    def istft(cls, n, *, win=0, hop=0):
        """Inverse STFT (faf_cuda_create_istft): frames -> signal."""
        c = config(n, hop=hop, win=win)
        return cls(C.lib().faf_cuda_create_istft(ctypes.byref(c)))

    @classmethod
    def cwt(cls, n, psi):
        """CWT filter bank (faf_cuda_create_cwt): psi holds the bank's rows,
        (rows, >= n/2+1) real bin weights (numpy, or a torch tensor on the
        host or the device), row 0 the lowpass when the bank has one."""
        if hasattr(psi, "data_ptr"):
            if str(psi.dtype) != "torch.float32" or psi.stride(-1) != 1:
                raise FafError("cwt: psi must be float32 with contiguous rows")
            ptr, stride = psi.data_ptr(), psi.stride(0)
        else:
            import numpy as np
            psi = np.ascontiguousarray(psi, np.float32)
            ptr, stride = psi.ctypes.data, psi.shape[-1]
        return cls(C.lib().faf_cuda_create_cwt(n, psi.shape[0], ptr, stride))

    @classmethod
    def icwt_dual(cls, n, dual):
        """Dual-frame inverse CWT (faf_cuda_create_icwt_dual): dual rows
        (rows, >= n/2+1), numpy or torch."""
        if hasattr(dual, "data_ptr"):
            ptr, stride = dual.data_ptr(), dual.stride(0)
        else:
            import numpy as np
            dual = np.ascontiguousarray(dual, np.float32)
            ptr, stride = dual.ctypes.data, dual.shape[-1]
        return cls(C.lib().faf_cuda_create_icwt_dual(n, dual.shape[0], ptr, stride))

    @classmethod
    def icwt_l1(cls, n, rows, has_lowpass, dlog, c):
        """L1 one-integral inverse CWT (faf_cuda_create_icwt_l1)."""
        return cls(C.lib().faf_cuda_create_icwt_l1(n, rows, int(has_lowpass), dlog, c))

    @staticmethod
    def cwt_dual_rows(psi, eps=1e-6):
        """The dual-frame rows of a bank as the reference derives them
        (src/faf_cwt.c:440-482): psi_r / (sum_r psi_r^2 + eps), the sum over
        rows in FP64, zero where that sum is 0."""
        import numpy as np
        p = np.asarray(psi, np.float64)
        s = np.sum(p * p, axis=0)
        return np.where(s > 0, p / (s + eps), 0.0).astype(np.float32)

    @property
    def cwt_rows(self):
        return self.s.user_aux_n

    @classmethod
    def chirp(cls, source):
        return cls(C.lib().chirp_compile(source.encode()))

    def inverse(self):
        return Transform(C.lib().faf_create_inverse(self._p))

    # ---- fields ----
    @property
    def ptr(self):
        return self._p

    @property
    def s(self):
        return self._p.contents

    @property
    def n(self):
        return self._n

    @property
    def type(self):
        return self.s.type

    @property
    def kind(self):
        k = C.lib().faf_cuda_plan_kind(self._p)
        return k.decode() if k else None

    def spectrum_len(self):
        return C.lib().faf_spectrum_len(self._p)

    # ---- binding / streams ----
    def bind(self, hr, hi, n_bins=None, name="H"):
        n_bins = n_bins if n_bins is not None else len(hr)
        self._keep += [hr, hi]
        _check(C.lib().chirp_bind(self._p, name.encode(), _ptr(hr), _ptr(hi), n_bins))

    def set_stream(self, stream):
        """stream: torch.cuda.Stream, a raw cudaStream_t int, or None."""
        _check(C.lib().faf_cuda_set_stream(self._p, _stream_handle(stream)))

    def synchronize(self):
        _check(C.lib().faf_cuda_synchronize(self._p))

    def wait_status(self):
        """0: every bounded wait of this transform's kernels completed; 1: one
        ran out (that launch's results are invalid)."""
        rc = C.lib().faf_cuda_wait_status(self._p)
        if rc < 0:
            raise FafError(C.error())
        return rc

    def tc_status(self):
        """Tensor-core plans: 0 = every MMA wait completed, 1 = one ran out of
        its bound; -1 for other plans."""
        return C.lib().faf_cuda_tc_status(self._p)

    # ---- execute ----
    def execute(self, out, inp):
        """faf_execute with two faf_buffer descriptors."""
        _check(C.lib().faf_execute(self._p, ctypes.byref(out), ctypes.byref(inp)))

    def execute_batched(self, out, inp, batch, in_dist=0, out_dist=0):
        if self._xb(self._p, ctypes.byref(out), ctypes.byref(inp), batch, in_dist, out_dist):
            raise FafError(C.error())

    def c2c(self, re, im=None, out_re=None, out_im=None):
        """Batched C2C over the last axis.  Split planes (re, im) or one
        interleaved buffer (re only, shape (..., 2n)) for INTERLEAVED plans."""
        n = self.n
        inter = self._inter
        lay = L_INTERLEAVED if inter else L_SPLIT
        batch = (re.numel() if hasattr(re, "numel") else re.size) // (2 * n if inter else n)
        if out_re is None:
            out_re = _empty_like_batch(re, tuple(re.shape))
            out_im = None if inter else _empty_like_batch(re, tuple(re.shape))
        self.execute_batched(_buf(out_re, out_im, n, lay), _buf(re, im, n, lay), batch)
        return out_re if inter else (out_re, out_im)

    def r2c(self, x, out_re=None, out_im=None):
        n, nb = self.n, self.n // 2 + 1
        batch = (x.numel() if hasattr(x, "numel") else x.size) // n
        shp = tuple(x.shape[:-1]) + (nb,)
        inter = self._inter
        if out_re is None:
            out_re = _empty_like_batch(x, shp + (2,) if inter else shp)
            out_im = None if inter else _empty_like_batch(x, shp)
        lay = L_INTERLEAVED if inter else L_HERMITIAN
        self.execute_batched(_buf(out_re, out_im, nb, lay), _buf(x, None, n, L_REAL), batch)
        return out_re if inter else (out_re, out_im)

    def c2r(self, Xr, Xi=None, out=None):
        n, nb = self.n, self.n // 2 + 1
        inter = self._inter
        cnt = Xr.numel() if hasattr(Xr, "numel") else Xr.size
        batch = cnt // (2 * nb if inter else nb)
        shp = (tuple(Xr.shape[:-2]) if inter else tuple(Xr.shape[:-1])) + (n,)
        if out is None:
            out = _empty_like_batch(Xr, shp)
        lay = L_INTERLEAVED if inter else L_HERMITIAN
        self.execute_batched(_buf(out, None, n, L_REAL), _buf(Xr, Xi, nb, lay), batch)
        return out

    def pipeline(self, x, out=None):
        n = self.n
        batch = (x.numel() if hasattr(x, "numel") else x.size) // n
        if out is None:
            out = _empty_like_batch(x, tuple(x.shape))
        self.execute_batched(_buf(out, None, n, L_REAL), _buf(x, None, n, L_REAL), batch)
        return out

    def frames(self, sig_len):
        win, hop = self.s.win_length, self.s.hop_length
        return 1 + (sig_len - win) // hop

    def stft_frames(self, x, out_re=None, out_im=None):
        """Framed real STFT of signals x (n_sig, L) -> (n_sig, F, n/2+1)."""
        L = x.shape[-1]
        n_sig = (x.numel() if hasattr(x, "numel") else x.size) // L
        F, nb = self.frames(L), self.n // 2 + 1
        shp = tuple(x.shape[:-1]) + (F, nb)
        if out_re is None:
            out_re = _empty_like_batch(x, shp)
            out_im = _empty_like_batch(x, shp)
        self.execute_batched(_buf(out_re, out_im, F * nb, L_HERMITIAN),
                             _buf(x, None, L, L_REAL), n_sig)
        return out_re, out_im

    def istft_frames(self, Xr, Xi, out=None):
        """Inverse STFT of frames (n_sig, F, n/2+1) -> (n_sig, (F-1) hop + win)."""
        nb = self.n // 2 + 1
        F = Xr.shape[-2]
        L = (F - 1) * self.s.hop_length + self.s.win_length
        n_sig = (Xr.numel() if hasattr(Xr, "numel") else Xr.size) // (F * nb)
        if out is None:
            out = _empty_like_batch(Xr, tuple(Xr.shape[:-2]) + (L,))
        self.execute_batched(_buf(out, None, L, L_REAL), _buf(Xr, Xi, F * nb, L_HERMITIAN),
                             n_sig)
        return out

    def synthesize(self, W, out=None):
        """Inverse CWT of coefficients W (..., rows, n) -> x (..., n)."""
        n, rows = self.n, self.cwt_rows
        batch = (W.numel() if hasattr(W, "numel") else W.size) // (rows * n)
        if out is None:
            out = _empty_like_batch(W, tuple(W.shape[:-2]) + (n,))
        self.execute_batched(_buf(out, None, n, L_REAL), _buf(W, None, rows * n, L_REAL), batch)
        return out

    def analyze(self, x, out=None):
        """Forward CWT of signals x (..., n) -> W (..., rows, n)."""
        n, rows = self.n, self.cwt_rows
        batch = (x.numel() if hasattr(x, "numel") else x.size) // n
        if out is None:
            out = _empty_like_batch(x, tuple(x.shape[:-1]) + (rows, n))
        self.execute_batched(_buf(out, None, rows * n, L_REAL), _buf(x, None, n, L_REAL), batch)
        return out

    def close(self):
        if self._p:
            C.lib().faf_destroy_transform(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
