"""Seeded cases of the golden fixtures (shared by gen_golden.py and the tests).

Inputs are regenerated from their seeds (numpy PCG64); only the reference
library's outputs are stored in golden.npz.
"""
import numpy as np

C2C_SIZES = [2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 15, 16, 20, 30, 48, 60, 64, 192, 240, 1000,
             1024, 3072, 6000]
RADER = [11, 13, 17, 29, 31, 37, 97, 1009]
BLUESTEIN = [23, 47, 307]
BIG_C2C = [16384]
REAL_SIZES = [2, 16, 64, 4096, 6000]
STFT = (1024, 1024, 256, 4096)  # n, win, hop, signal length
CWT = [512, 1000]  # signal lengths; the reference's default bank (Morse 20/3, 10 voices, lowpass)
FLAG_BLUESTEIN = 1 << 12


def c2c_input(n, batch=2, seed=0):
    rng = np.random.default_rng(seed * 100003 + n)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    return re, im


def real_input(n, batch=2, seed=1):
    rng = np.random.default_rng(seed * 100003 + n)
    return rng.standard_normal((batch, n)).astype(np.float32)


def notch_mask(n=4096, lo=400, hi=420, ramp=32):
    nb = n // 2 + 1
    k = np.arange(nb)
    m = np.ones(nb)
    m[(k >= lo) & (k <= hi)] = 0.0
    left = (k >= lo - ramp) & (k < lo)
    m[left] = 0.5 * (1 + np.cos(np.pi * (k[left] - (lo - ramp)) / ramp))
    right = (k > hi) & (k <= hi + ramp)
    m[right] = 0.5 * (1 - np.cos(np.pi * (k[right] - hi) / ramp))
    return m.astype(np.float32)


def notch_signal(batch=2, n=4096, seed=1):
    rng = np.random.default_rng(seed)
    k = np.arange(n)
    return (rng.standard_normal((batch, n)) + 5 * np.cos(2 * np.pi * 410 * k / n)).astype(np.float32)


# (key, chirp source, oracle op list, n)
PIPELINES = [
    ("pipe_notch4096", "(pipeline (rfft :size 4096) (mul-spectrum) (irfft))", "mask", 4096),
    ("pipe_bandpass32", "(pipeline (rfft :size 32) (bandpass :lo 4 :hi 4) (irfft))",
     [(3, 4, 4)], 32),
    ("pipe_conj16", "(pipeline (rfft :size 16) conj (irfft))", [(1, 0, 0)], 16),
    ("pipe_conj_bp6000", "(pipeline (rfft :size 6000) conj (bandpass :lo 10 :hi 2000) (irfft))",
     [(1, 0, 0), (3, 10, 2000)], 6000),
]

# size-policy probe points
POLICY_N = list(range(0, 300)) + [1000, 1021, 1024, 3840, 4000, 4050, 4096, 4097, 6000, 7681,
                                  12289, 16384, 16385, 65536, 65537]
# (type, n, flags) create probes for error messages (reference tests/test_sizes.cpp)
CREATE_PROBES = [(0, 14, 0), (0, 23, 0), (0, 4097, 0), (2, 13, 0), (2, 14, 0), (2, 1002, 0),
                 (2, 64, FLAG_BLUESTEIN), (0, 23, FLAG_BLUESTEIN)]
