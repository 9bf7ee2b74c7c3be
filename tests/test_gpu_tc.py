"""Tensor-core precision form (FAF_FLAG_TENSOR_CORE): power-of-two C2C whose
radix-16 stages run as FP16 tcgen05 MMAs with hi + lo split operands and FP32
accumulation.  Checked against FP64 (rel L2 <= 1e-5) and the oracle on the
heavy-tailed input of the 16384-point workload (1% of entries x 1e3)."""
import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu

TC_SIZES = [256, 512, 1024, 2048, 4096, 8192, 16384]


def heavy_tailed(n, batch, seed):
    rng = seeded(seed)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    for a in (re, im):
        a[rng.random(a.shape) < 0.01] *= 1e3
    return re, im


@pytest.mark.parametrize("n", TC_SIZES)
@pytest.mark.parametrize("inverse", [False, True])
def test_tc_c2c_accuracy(cuda, n, inverse):
    import fastandfourier_b200 as F
    torch = cuda
    batch = max(3, 65536 // n) + 1  # a ragged last group
    re, im = heavy_tailed(n, batch, 400 + n)
    t = F.Transform.fft(n, inverse=inverse, flags=F.FLAG_TENSOR_CORE)
    assert t.kind == "c2c-tc"
    yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    assert t.tc_status() == 0
    gr, gi = yr.cpu().numpy(), yi.cpu().numpy()
    want = orc.fp64_c2c(re, im, inverse=inverse)
    e64 = orc.rel_l2_complex(gr, gi, want)
    assert e64 <= REL_L2_TOL, (n, inverse, e64)
    if n <= 4096:
        o_r, o_i = orc.c2c(re[:2], im[:2], inverse=inverse)
        assert orc.rel_l2_complex(gr[:2], gi[:2], o_r + 1j * o_i) <= REL_L2_TOL


def test_tc_matches_plain_path(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    n, batch = 16384, 40
    re, im = heavy_tailed(n, batch, 3)
    dr, di = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    tr, ti = F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE).c2c(dr, di)
    pr, pi = F.Transform.fft(n).c2c(dr, di)
    assert orc.rel_l2_complex(tr.cpu().numpy(), ti.cpu().numpy(),
                              pr.cpu().numpy() + 1j * pi.cpu().numpy()) <= REL_L2_TOL


def test_tc_flag_ignored_where_unsupported(cuda):
    import fastandfourier_b200 as F
    for n in (60, 128, 32768):
        t = F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE)
        assert t.kind != "c2c-tc" and t.tc_status() == -1


@pytest.mark.parametrize("n,batch", [(8192, 400), (16384, 300)])
def test_tc_landed_inputs_over_several_rounds(cuda, n, batch):
    """More transforms than SMs: every CTA lands a second (and third)
    transform in its workspace while it finishes the previous one."""
    import fastandfourier_b200 as F
    torch = cuda
    re, im = heavy_tailed(n, batch, 900 + n)
    t = F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE)
    yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    got = yr.cpu().numpy() + 1j * yi.cpu().numpy()
    want = orc.fp64_c2c(re, im)
    assert float(np.linalg.norm(got - want) / np.linalg.norm(want)) <= REL_L2_TOL
    assert t.wait_status() == 0 and t.tc_status() == 0
