"""Uneven batches: transforms of mixed lengths (5-smooth, codelet, Rader
primes, lengths above one CTA) in one persistent launch, against the oracle
and FP64, and identical to the plain one-launch-per-length method."""
import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu

CONFIG3_LENGTHS = [12, 17, 31, 60, 240, 1000, 3072, 6000, 16384, 65536]


def ragged(lengths, seed):
    rng = seeded(seed)
    total = sum(lengths)
    re = rng.uniform(-1, 1, total).astype(np.float32)
    im = rng.uniform(-1, 1, total).astype(np.float32)
    return re, im


def check_against_fp64(lengths, re, im, gr, gi, inverse=False, norm=1):
    off = 0
    worst = 0.0
    for n in lengths:
        want = orc.fp64_c2c(re[off:off + n][None], im[off:off + n][None], inverse=inverse,
                            norm=norm)[0]
        e = orc.rel_l2_complex(gr[off:off + n], gi[off:off + n], want)
        worst = max(worst, e)
        off += n
    return worst


@pytest.mark.parametrize("measure", [False, True])
def test_uneven_config_lengths(cuda, measure):
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(2)
    lengths = list(rng.choice(CONFIG3_LENGTHS, 96))
    re, im = ragged(lengths, 3)
    u = F.Uneven(lengths, measure=measure)
    assert u.total == sum(lengths)
    dr, di = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    yr, yi = torch.empty_like(dr), torch.empty_like(di)
    u.execute(dr, di, yr, yi)
    gr, gi = yr.cpu().numpy(), yi.cpu().numpy()
    assert check_against_fp64(lengths, re, im, gr, gi) <= REL_L2_TOL
    # replay of the captured graph with the same buffers
    u.execute(dr, di, yr, yi)
    assert np.array_equal(yr.cpu().numpy(), gr)
    # the plain method (one launch per run of equal lengths) agrees
    pr, pi = torch.empty_like(dr), torch.empty_like(di)
    u.execute(dr, di, pr, pi, plain=True)
    assert orc.rel_l2_complex(pr.cpu().numpy(), pi.cpu().numpy(), gr + 1j * gi) <= REL_L2_TOL


def test_uneven_short_power_of_two_classes_land(cuda, monkeypatch):
    """Power-of-two classes of 256 and 512 points, many transforms each at
    ragged offsets, land their inputs by bulk copy in the graph: equal to FP64
    and bit-identical to the direct loads."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(21)
    lengths = list(rng.choice([256, 512, 60, 1024], 3000))
    re, im = ragged(lengths, 22)
    dr, di = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()

    def run():
        u = F.Uneven(lengths)
        yr, yi = torch.empty_like(dr), torch.empty_like(di)
        u.execute(dr, di, yr, yi)
        return yr.cpu().numpy(), yi.cpu().numpy()

    gr, gi = run()
    assert check_against_fp64(lengths, re, im, gr, gi) <= REL_L2_TOL
    monkeypatch.setenv("FAF_CUDA_NO_STAGING", "1")
    dr2, di2 = run()
    assert np.array_equal(gr, dr2) and np.array_equal(gi, di2)


def test_uneven_matches_single_size_oracle(cuda):
    """Each transform against the oracle restatement of the reference."""
    import fastandfourier_b200 as F
    torch = cuda
    lengths = [12, 17, 31, 60, 240, 1000, 3072, 6000, 7, 11, 2, 1, 16384]
    re, im = ragged(lengths, 9)
    u = F.Uneven(lengths, inverse=True, norm=F.N_ORTHO)
    dr, di = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    yr, yi = torch.empty_like(dr), torch.empty_like(di)
    u.execute(dr, di, yr, yi)
    gr, gi = yr.cpu().numpy(), yi.cpu().numpy()
    off = 0
    for n in lengths:
        wr, wi = orc.c2c(re[off:off + n][None], im[off:off + n][None], inverse=True, norm=2)
        assert orc.rel_l2_complex(gr[off:off + n], gi[off:off + n], wr[0] + 1j * wi[0]) <= REL_L2_TOL, n
        off += n


def test_uneven_new_buffers_recapture(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    lengths = [60, 240, 17, 65536, 1000]
    u = F.Uneven(lengths)
    for seed in (20, 21):
        re, im = ragged(lengths, seed)
        dr, di = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
        yr, yi = torch.empty_like(dr), torch.empty_like(di)
        u.execute(dr, di, yr, yi)
        assert check_against_fp64(lengths, re, im, yr.cpu().numpy(), yi.cpu().numpy()) <= REL_L2_TOL


def test_uneven_tensor_core_form(cuda):
    """FAF_FLAG_TENSOR_CORE: the power-of-two classes run as FP16 hi+lo MMAs;
    every transform stays within rel L2 1e-5 of FP64."""
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(21)
    lengths = list(rng.choice(CONFIG3_LENGTHS + [256, 1024, 4096], 120))
    re, im = ragged(lengths, 22)
    for r in (re, im):
        r[rng.random(r.shape) < 0.01] *= 1e3
    u = F.Uneven(lengths, tensor_core=True)
    dr, di = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    yr, yi = torch.empty_like(dr), torch.empty_like(di)
    u.execute(dr, di, yr, yi)
    assert check_against_fp64(lengths, re, im, yr.cpu().numpy(), yi.cpu().numpy()) <= REL_L2_TOL
