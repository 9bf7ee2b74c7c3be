"""ctypes binding of libfaf_b200.so -- the C ABI of include/fastandfourier.h,
include/chirp.h and include/faf_cuda.h.

The library is loaded from the package directory (built in-tree by
fastandfourier_b200.build).  There is no fallback: if the library cannot be
loaded, or a create/execute call fails, the error propagates.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfaf_b200.so")

# enum values (include/fastandfourier.h)
PREC_FP16, PREC_FP32, PREC_FP64 = 1, 3, 4
(T_FFT, T_IFFT, T_RFFT, T_IRFFT) = (0, 1, 2, 3)
T_STFT, T_PIPELINE, T_CWT, T_ICWT = 12, 20, 21, 22
L_DEFAULT, L_SPLIT, L_HERMITIAN, L_REAL, L_INTERLEAVED = 0, 1, 2, 3, 4
N_DEFAULT, N_NONE, N_ORTHO, N_FORWARD, N_LAZY, N_JPEG2000 = 0, 1, 2, 3, 4, 5
DIR_FORWARD, DIR_INVERSE = 0, 1
B_AUTO, B_VM, B_JIT, B_CUDA = 0, 1, 2, 3
FLAG_INVERSE, FLAG_REAL = 0x1, 0x8
FLAG_BLUESTEIN, FLAG_MEASURE = 1 << 12, 1 << 13
FLAG_TENSOR_CORE = 1 << 16
CHIRP_OP_CONJ, CHIRP_OP_MUL, CHIRP_OP_BANDPASS = 0x7FFFFFFD, 0x7FFFFFFE, 0x7FFFFFFF
(CHIRP_DEVICE_GAIN, CHIRP_DEVICE_PHASE, CHIRP_DEVICE_DELAY, CHIRP_DEVICE_LOWPASS,
 CHIRP_DEVICE_HIGHPASS) = range(5)
FAF_CALL_BUILTIN = 30


class faf_config(ctypes.Structure):
    _fields_ = [("n", ctypes.c_size_t), ("precision", ctypes.c_int), ("layout", ctypes.c_int),
                ("norm", ctypes.c_int), ("dir", ctypes.c_int), ("backend", ctypes.c_int),
                ("flags", ctypes.c_uint32), ("family", ctypes.c_int), ("levels", ctypes.c_size_t),
                ("conv", ctypes.c_int), ("dwt_backend", ctypes.c_int), ("dct_type", ctypes.c_int),
                ("hop_length", ctypes.c_size_t), ("win_length", ctypes.c_size_t)]


class faf_buffer(ctypes.Structure):
    _fields_ = [("re", ctypes.c_void_p), ("im", ctypes.c_void_p), ("n", ctypes.c_size_t),
                ("layout", ctypes.c_int)]


class faf_inst(ctypes.Structure):
    _fields_ = [("packed", ctypes.c_uint32), ("a0", ctypes.c_uint32), ("a1", ctypes.c_uint32),
                ("a2", ctypes.c_uint32)]


class faf_transform(ctypes.Structure):
    pass


faf_transform._fields_ = [
    ("n", ctypes.c_size_t), ("n_inst", ctypes.c_size_t), ("code", ctypes.POINTER(faf_inst)),
    ("twiddles", ctypes.c_void_p * 8), ("twiddle_sizes", ctypes.c_size_t * 8),
    ("precision", ctypes.c_int), ("type", ctypes.c_int), ("flags", ctypes.c_uint32),
    ("jit_cache", ctypes.c_void_p), ("hop_length", ctypes.c_size_t),
    ("win_length", ctypes.c_size_t), ("levels", ctypes.c_size_t), ("family", ctypes.c_int),
    ("cfg", faf_config), ("scratch", ctypes.c_void_p), ("scratch_size", ctypes.c_size_t),
    ("execute_func", ctypes.c_void_p), ("inner", ctypes.POINTER(faf_transform)),
    ("inner_inv", ctypes.POINTER(faf_transform)), ("user_aux", ctypes.c_void_p),
    ("user_aux_im", ctypes.c_void_p), ("user_aux_n", ctypes.c_size_t),
    ("custom_h", ctypes.c_void_p), ("custom_g", ctypes.c_void_p), ("custom_ht", ctypes.c_void_p),
    ("custom_gt", ctypes.c_void_p), ("custom_len_hg", ctypes.c_int),
    ("custom_len_syn", ctypes.c_int), ("device_plan", ctypes.c_void_p)]

class faf_server_config(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("streams", ctypes.c_int),
                ("max_merge", ctypes.c_int)]


class faf_request(ctypes.Structure):
    _fields_ = [("chirp", ctypes.c_char_p), ("stft_n", ctypes.c_size_t),
                ("stft_win", ctypes.c_size_t), ("stft_hop", ctypes.c_size_t),
                ("h_re", ctypes.c_void_p), ("h_im", ctypes.c_void_p), ("h_len", ctypes.c_size_t),
                ("in_", ctypes.c_void_p), ("in_len", ctypes.c_size_t),
                ("out_re", ctypes.c_void_p), ("out_im", ctypes.c_void_p),
                ("stream_key", ctypes.c_ulonglong)]


class faf_server_stats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("batches", ctypes.c_longlong), ("merged_requests", ctypes.c_longlong),
                ("p50_latency_s", ctypes.c_double), ("p99_latency_s", ctypes.c_double),
                ("mean_latency_s", ctypes.c_double), ("max_latency_s", ctypes.c_double),
                ("wall_s", ctypes.c_double), ("requests_per_s", ctypes.c_double),
                ("bytes_per_s", ctypes.c_double), ("arena_bytes", ctypes.c_size_t),
                ("arena_peak_bytes", ctypes.c_size_t)]


TP = ctypes.POINTER(faf_transform)
BP = ctypes.POINTER(faf_buffer)
SPECTRAL_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_float),
                               ctypes.POINTER(ctypes.c_float), ctypes.c_size_t, ctypes.c_void_p)

_lib = None
_lock = threading.Lock()

# (name, restype, argtypes) for every exported entry point.
_SIGS = [
    ("faf_init", ctypes.c_int, []),
    ("faf_cleanup", None, []),
    ("faf_version", ctypes.c_char_p, []),
    ("faf_arch_name", ctypes.c_char_p, []),
    ("faf_get_error", ctypes.c_char_p, []),
    ("faf_clear_error", None, []),
    ("faf_layout_name", ctypes.c_char_p, [ctypes.c_int]),
    ("faf_norm_name", ctypes.c_char_p, [ctypes.c_int]),
    ("faf_precision_name", ctypes.c_char_p, [ctypes.c_int]),
    ("faf_transform_name", ctypes.c_char_p, [ctypes.c_int]),
    ("faf_precision_size", ctypes.c_size_t, [ctypes.c_int]),
    ("faf_get_alignment", ctypes.c_size_t, []),
    ("faf_spectrum_len", ctypes.c_size_t, [TP]),
    ("faf_is_size_supported", ctypes.c_bool, [ctypes.c_int, ctypes.c_size_t]),
    ("faf_get_recommended_size", ctypes.c_size_t, [ctypes.c_int, ctypes.c_size_t]),
    ("faf_create", TP, [ctypes.c_int, ctypes.POINTER(faf_config)]),
    ("faf_create_fft", TP, [ctypes.POINTER(faf_config)]),
    ("faf_create_rfft", TP, [ctypes.POINTER(faf_config)]),
    ("faf_create_stft", TP, [ctypes.POINTER(faf_config)]),
    ("faf_create_inverse", TP, [TP]),
    ("faf_destroy_transform", None, [TP]),
    ("faf_execute", ctypes.c_int, [TP, BP, BP]),
    ("faf_execute_batched", ctypes.c_int, [TP, BP, BP, ctypes.c_size_t, ctypes.c_size_t,
                                           ctypes.c_size_t]),
    ("faf_cuda_available", ctypes.c_int, []),
    ("faf_cuda_plan_kind", ctypes.c_char_p, [TP]),
    ("faf_cuda_last_launches", ctypes.c_int, []),
    ("faf_cuda_tc_status", ctypes.c_int, [TP]),
    ("faf_cuda_create_istft", TP, [ctypes.POINTER(faf_config)]),
    ("faf_cuda_set_stream", ctypes.c_int, [TP, ctypes.c_void_p]),
    ("faf_cuda_get_stream", ctypes.c_void_p, [TP]),
    ("faf_cuda_wait_status", ctypes.c_int, [TP]),
    ("faf_cuda_create_cwt", TP, [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]),
    ("faf_cuda_create_icwt_dual", TP,
     [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]),
    ("faf_cuda_create_icwt_l1", TP,
     [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    ("faf_cuda_synchronize", ctypes.c_int, [TP]),
    ("faf_cuda_execute_c2c_noalloc", ctypes.c_int,
     [TP] + [ctypes.c_void_p] * 4 + [ctypes.c_size_t]),
    ("faf_uneven_create", ctypes.c_void_p, [ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t,
                                             ctypes.POINTER(faf_config)]),
    ("faf_uneven_execute", ctypes.c_int, [ctypes.c_void_p] * 5),
    ("faf_uneven_execute_plain", ctypes.c_int, [ctypes.c_void_p] * 5),
    ("faf_uneven_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("faf_uneven_total", ctypes.c_size_t, [ctypes.c_void_p]),
    ("faf_uneven_destroy", None, [ctypes.c_void_p]),
    ("faf_server_create", ctypes.c_void_p, [ctypes.POINTER(faf_server_config)]),
    ("faf_server_submit", ctypes.c_longlong, [ctypes.c_void_p, ctypes.POINTER(faf_request)]),
    ("faf_server_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong,
                                       ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_size_t)]),
    ("faf_server_drain", ctypes.c_int, [ctypes.c_void_p]),
    ("faf_server_stream_frames", ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_ulonglong]
     + [ctypes.c_size_t] * 3),
    ("faf_server_close_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_ulonglong]),
    ("faf_server_prepare", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(faf_request)]),
    ("faf_server_stats_get", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(faf_server_stats)]),
    ("faf_server_stats_reset", None, [ctypes.c_void_p]),
    ("faf_server_replay", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(faf_request),
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_size_t,
                                         ctypes.POINTER(ctypes.c_double)]),
    ("faf_server_destroy", None, [ctypes.c_void_p]),
    ("chirp_compile", TP, [ctypes.c_char_p]),
    ("chirp_bind", ctypes.c_int, [TP, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_size_t]),
    ("chirp_register_spectral", ctypes.c_int, [ctypes.c_char_p, SPECTRAL_FN, ctypes.c_void_p]),
    ("chirp_register_spectral_device", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int,
                                                      ctypes.c_double]),
    ("chirp_cleanup", None, []),
    ("chirp_apply_split_f32", None, [TP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    ("chirp_count", ctypes.c_int, []),
    ("faf_herm_mul_f32", None, [ctypes.c_void_p] * 6 + [ctypes.c_size_t]),
    ("faf_herm_mul_conj_f32", None, [ctypes.c_void_p] * 6 + [ctypes.c_size_t]),
    ("faf_deinterleave_f32", ctypes.c_int, [ctypes.c_void_p] * 3 + [ctypes.c_size_t]),
    ("faf_interleave_f32", ctypes.c_int, [ctypes.c_void_p] * 3 + [ctypes.c_size_t]),
]


def lib():
    """Load libfaf_b200.so (building it first when nvcc is present and the
    library is missing).  Raises if it cannot be loaded."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from . import build as _build
                _build.build()
            L = ctypes.CDLL(LIB_PATH)
            for name, res, args in _SIGS:
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def error():
    return lib().faf_get_error().decode(errors="replace")
