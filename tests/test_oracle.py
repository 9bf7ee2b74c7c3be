"""The oracle (C restatement of the reference, oracle/faf_oracle.c) pinned
against the golden fixtures made from the reference library itself, against
FP64, and against the reference's own known-answer tests.  CPU only."""
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import orc

GOLD = os.path.join(ROOT, "tests", "golden")
import sys  # noqa: E402
sys.path.insert(0, GOLD)
import cases  # noqa: E402

TOL = 1e-5


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "golden.npz"))


@pytest.mark.parametrize("n", cases.C2C_SIZES + cases.RADER)
@pytest.mark.parametrize("inv", [0, 1])
def test_oracle_c2c_vs_reference(gold, n, inv):
    re, im = cases.c2c_input(n)
    yr, yi = orc.c2c(re, im, inverse=inv)
    g = gold[f"c2c_{n}_{inv}"]
    assert orc.rel_l2_complex(yr, yi, g[0] + 1j * g[1]) <= TOL
    assert orc.rel_l2_complex(yr, yi, orc.fp64_c2c(re, im, inverse=inv)) <= TOL


@pytest.mark.parametrize("n", cases.BLUESTEIN)
@pytest.mark.parametrize("inv", [0, 1])
def test_oracle_bluestein_vs_reference(gold, n, inv):
    re, im = cases.c2c_input(n)
    yr, yi = orc.c2c(re, im, inverse=inv, flags=orc.FLAG_BLUESTEIN)
    g = gold[f"blue_{n}_{inv}"]
    assert orc.rel_l2_complex(yr, yi, g[0] + 1j * g[1]) <= TOL


def test_oracle_large_c2c_vs_reference(gold):
    re, im = cases.c2c_input(16384, batch=1)
    yr, yi = orc.c2c(re, im)
    g = gold["c2c_16384_0"]
    assert orc.rel_l2_complex(yr, yi, g[0] + 1j * g[1]) <= TOL


@pytest.mark.parametrize("n", cases.REAL_SIZES)
def test_oracle_real_vs_reference(gold, n):
    x = cases.real_input(n)
    Xr, Xi = orc.r2c(x)
    g = gold[f"r2c_{n}"]
    assert orc.rel_l2_complex(Xr, Xi, g[0] + 1j * g[1]) <= TOL
    y = orc.c2r(Xr, Xi, n)
    assert orc.rel_l2(y, gold[f"c2r_{n}"]) <= TOL
    assert orc.rel_l2(y, x) <= TOL


@pytest.mark.parametrize("key,src,ops,n", cases.PIPELINES)
def test_oracle_pipeline_vs_reference(gold, key, src, ops, n):
    x = cases.notch_signal(n=n) if key == "pipe_notch4096" else cases.real_input(n, seed=7)
    if ops == "mask":
        m = cases.notch_mask(n)
        y = orc.pipeline(x, [(orc.OP_MUL, 0, 0)], m, np.zeros_like(m))
    else:
        y = orc.pipeline(x, ops)
    assert orc.rel_l2(y, gold[key]) <= TOL


def test_oracle_stft_vs_reference(gold):
    n, win, hop, L = cases.STFT
    xs = cases.real_input(L, batch=2, seed=4)
    Xr, Xi = orc.stft(xs, n, win, hop)
    g = gold["stft"]
    assert Xr.shape == g[0].shape == (2, 1 + (L - win) // hop, n // 2 + 1)
    assert orc.rel_l2_complex(Xr, Xi, g[0] + 1j * g[1]) <= TOL


# ---- the reference's known answers, restated (tests/test_mixed_radix.cpp,
# tests/test_rader.cpp, tests/test_sizes.cpp, tests/test_rfft.cpp) ---------

@pytest.mark.parametrize("n", [12, 15, 20, 30, 48, 60, 192])
def test_kat_mixed_radix_vs_dft(n):
    i = np.arange(n)
    x = (np.sin(2 * np.pi * 2 * i / n) + 0.3 * ((i % 5) - 2)).astype(np.float32)
    yr, yi = orc.c2c(x[None], np.zeros((1, n), np.float32))
    want = np.fft.fft(x.astype(np.float64))
    tol = 2e-3 if n >= 100 else 5e-4
    assert np.max(np.abs(yr[0] + 1j * yi[0] - want)) <= tol


@pytest.mark.parametrize("n", [1000, 1920, 4000])
def test_kat_large_mixed_impulse(n):
    x = np.zeros((1, n), np.float32)
    x[0, 0] = 1
    yr, yi = orc.c2c(x, np.zeros_like(x))
    assert np.max(np.abs(yr - 1)) <= 2e-3 and np.max(np.abs(yi)) <= 2e-3


@pytest.mark.parametrize("p", [11, 13, 17, 19, 29, 31, 37])
def test_kat_rader_vs_dft(p):
    rng = np.random.default_rng(p)
    re = rng.uniform(-1, 1, (1, p)).astype(np.float32)
    im = rng.uniform(-1, 1, (1, p)).astype(np.float32)
    yr, yi = orc.c2c(re, im)
    assert orc.rel_l2_complex(yr, yi, orc.fp64_c2c(re, im)) <= 1e-5
    zr, zi = orc.c2c(yr, yi, inverse=True)
    assert np.allclose(zr, re, atol=1e-5) and np.allclose(zi, im, atol=1e-5)


@pytest.mark.parametrize("n", [23, 47, 307])
def test_kat_bluestein_vs_dft(n):
    x = np.cos(2 * np.pi * 3 * np.arange(n) / n).astype(np.float32)[None]
    yr, yi = orc.c2c(x, np.zeros_like(x), flags=orc.FLAG_BLUESTEIN)
    want = np.fft.fft(x[0].astype(np.float64))
    assert np.max(np.abs(yr[0] + 1j * yi[0] - want)) <= (5e-3 if n > 100 else 1e-3)


@pytest.mark.parametrize("n", [2, 4, 6, 8, 16, 30, 64, 128, 1000, 1024, 4096])
def test_kat_rfft_roundtrip(n):
    x = np.random.default_rng(n).standard_normal((1, n)).astype(np.float32)
    Xr, Xi = orc.r2c(x)
    assert Xi[0, 0] == 0 and Xi[0, -1] == 0
    y = orc.c2r(Xr, Xi, n)
    assert np.max(np.abs(y - x)) <= (2e-4 if n >= 1024 else 1e-4)


def test_kat_rfft_impulse_and_tone():
    n = 64
    x = np.zeros((1, n), np.float32)
    x[0, 0] = 1
    Xr, Xi = orc.r2c(x)
    assert np.allclose(Xr, 1, atol=1e-5) and np.allclose(Xi, 0, atol=1e-5)
    k = 5
    x = np.cos(2 * np.pi * k * np.arange(n) / n).astype(np.float32)[None]
    Xr, Xi = orc.r2c(x)
    assert abs(Xr[0, k] - n / 2) < 1e-3


def test_oracle_rejects_unsupported_size():
    with pytest.raises(RuntimeError):
        orc.c2c(np.zeros((1, 23), np.float32), np.zeros((1, 23), np.float32))


def test_hann_matches_definition():
    n = 1024
    w = orc.hann(n)
    i = np.arange(n)
    assert np.allclose(w, 0.5 * (1 - np.cos(2 * np.pi * i / (n - 1))), atol=1e-6)
    assert w[0] == 0 and abs(w[-1]) < 1e-6


@pytest.mark.parametrize("n", [60, 1024, 4096])
def test_reference_fp64_c2c_vs_numpy(n):
    """The reference's FP64 C2C path (src/faf_core.c:521) as the driver calls
    it agrees with numpy's FP64 FFT, so it can stand as the FP64 checker."""
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(n)
    re, im = rng.uniform(-1, 1, (3, n)), rng.uniform(-1, 1, (3, n))
    for inv in (False, True):
        yr, yi = refimpl.c2c64(re, im, inverse=inv)
        z = re + 1j * im
        want = np.fft.ifft(z, axis=-1) if inv else np.fft.fft(z, axis=-1)
        got = yr + 1j * yi
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-12


@pytest.mark.parametrize("n", cases.CWT)
def test_oracle_cwt_vs_reference(gold, n):
    """The oracle's CWT (its own R2C, bank multiply, C2R) against the
    reference's faf_cwt_execute on the reference's default bank."""
    x = cases.real_input(n, batch=1, seed=9)
    psi, want = gold[f"cwt_psi_{n}"], gold[f"cwt_{n}"]
    got = orc.cwt(x, psi)
    assert orc.rel_l2(got, want) <= TOL
    assert orc.rel_l2(got, orc.fp64_cwt(x, psi)) <= TOL


@pytest.mark.parametrize("n", cases.CWT)
def test_oracle_icwt_vs_reference(gold, n):
    """The oracle's dual-frame and L1 inverse CWT against the reference's
    faf_icwt_execute on the reference's own coefficients."""
    import math
    W, psi = gold[f"cwt_{n}"], gold[f"cwt_psi_{n}"]
    C, voices = gold[f"cwt_consts_{n}"]
    got = orc.icwt_dual(W, orc.cwt_dual(psi))
    assert orc.rel_l2(got, gold[f"icwt_dual_{n}"]) <= TOL
    got = orc.icwt_l1(W, True, math.log(2) / voices, C)
    assert orc.rel_l2(got, gold[f"icwt_l1_{n}"]) <= TOL
