"""Rader primes whose inner length p - 1 exceeds one CTA (16384), and
Bluestein lengths whose inner M = next 5-smooth >= 2n - 1 does: the inner
FFTs run on the four-step path between gather / x B / scatter (Rader,
reference src/faf_fft_rader.c:136-232) or chirp / x B / chirp (Bluestein,
reference src/faf_bluestein.c:165-223) passes.  Parity against the oracle
(the CPU restatement of the reference) and FP64 at rel L2 <= 1e-5, batches
past one scratch chunk, and the policy check: every length that
faf_is_size_supported(FFT, n) accepts creates a plan."""
import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _case(torch, F, n, inverse, flags=0, norm=1, batch=2):
    rng = seeded(n + int(inverse))
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    t = F.Transform.fft(n, inverse=inverse, norm=norm, flags=flags)
    yr, yi = t.c2c(dev(torch, re), dev(torch, im))
    torch.cuda.synchronize()
    gr, gi = yr.cpu().numpy(), yi.cpu().numpy()
    wr, wi = orc.c2c(re, im, inverse=inverse, norm=norm, flags=flags)
    e_orc = orc.rel_l2_complex(gr, gi, wr + 1j * wi)
    e_64 = orc.rel_l2_complex(gr, gi, orc.fp64_c2c(re, im, inverse=inverse, norm=norm))
    return t, e_orc, e_64


@pytest.mark.parametrize("p", [17011, 18433, 40961, 65537])
@pytest.mark.parametrize("inverse", [False, True])
def test_long_rader_matches_oracle(cuda, p, inverse):
    import fastandfourier_b200 as F
    t, e_orc, e_64 = _case(cuda, F, p, inverse)
    assert t.kind == "rader"
    assert e_orc <= REL_L2_TOL, (p, inverse, e_orc)
    assert e_64 <= REL_L2_TOL, (p, inverse, e_64)


@pytest.mark.parametrize("n", [10007, 30011, 65521])
@pytest.mark.parametrize("inverse", [False, True])
def test_long_bluestein_matches_oracle(cuda, n, inverse):
    import fastandfourier_b200 as F
    t, e_orc, e_64 = _case(cuda, F, n, inverse, flags=F.FLAG_BLUESTEIN)
    assert t.kind == "bluestein"
    assert e_orc <= REL_L2_TOL, (n, inverse, e_orc)
    assert e_64 <= REL_L2_TOL, (n, inverse, e_64)


def test_long_rader_norms(cuda):
    import fastandfourier_b200 as F
    for norm in (F.N_ORTHO, F.N_FORWARD):
        _, e_orc, e_64 = _case(cuda, F, 40961, False, norm=norm)
        assert e_orc <= REL_L2_TOL and e_64 <= REL_L2_TOL, (norm, e_orc, e_64)


@pytest.mark.parametrize("n,flags,batch", [(40961, 0, 103), (20011, "b", 200)])
def test_long_conv_batches_past_one_chunk(cuda, n, flags, batch):
    """The scratch holds 64 MB of inner transforms (102 of 40960 points, 103
    of Bluestein's 40500 for n = 20011): these batches take two chunks."""
    import fastandfourier_b200 as F
    torch = cuda
    fl = F.FLAG_BLUESTEIN if flags == "b" else 0
    rng = seeded(n + batch)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    t = F.Transform.fft(n, flags=fl)
    yr, yi = t.c2c(dev(torch, re), dev(torch, im))
    torch.cuda.synchronize()
    e_64 = orc.rel_l2_complex(yr.cpu().numpy(), yi.cpu().numpy(), orc.fp64_c2c(re, im))
    assert e_64 <= REL_L2_TOL, e_64
    assert F.lib().faf_cuda_last_launches() > 5  # two chunks of five-plus launches


def test_long_rader_host_buffers(cuda):
    """Host buffers (staged through the plan's device buffer) give the same
    result as device buffers."""
    import fastandfourier_b200 as F
    torch = cuda
    n, batch = 18433, 3
    rng = seeded(7)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    t = F.Transform.fft(n)
    hr, hi = t.c2c(re, im)
    dr, di = t.c2c(dev(torch, re), dev(torch, im))
    torch.cuda.synchronize()
    assert np.array_equal(np.asarray(hr), dr.cpu().numpy())
    assert np.array_equal(np.asarray(hi), di.cpu().numpy())


def _rader_primes_above_one_cta(limit=65537):
    def prime(p):
        if p < 2:
            return False
        d = 2
        while d * d <= p:
            if p % d == 0:
                return False
            d += 1
        return True

    def smooth7(m):
        for f in (2, 3, 5, 7):
            while m % f == 0:
                m //= f
        return m == 1

    return [p for p in range(16387, limit + 1, 2) if prime(p) and smooth7(p - 1)]


def test_every_supported_rader_prime_creates_a_plan(cuda):
    """faf_is_size_supported(FFT, p) and faf_create_fft agree on every Rader
    prime above one CTA, up to 65537."""
    import fastandfourier_b200 as F
    L = F.lib()
    primes = _rader_primes_above_one_cta()
    assert 17011 in primes and 65537 in primes and len(primes) >= 50
    for p in primes:
        assert L.faf_is_size_supported(F.T_FFT, p)
        t = F.Transform.fft(p)
        assert t.kind == "rader", p
        t.close()
