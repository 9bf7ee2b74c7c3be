"""Tensor-core precision form (FAF_FLAG_TENSOR_CORE): power-of-two C2C whose
DFT stages run as FP16 tcgen05 MMAs with hi + lo split operands and FP32
accumulation -- radix-16 stages for 256..2048 points, 64-point DFTs (two
passes) for 4096..16384, where FAF_CUDA_TC_RADIX=16 selects the radix-16
kernels instead.  Checked against FP64 (rel L2 <= 1e-5) and the oracle on the
heavy-tailed input of the 16384-point workload (1% of entries x 1e3)."""
import os

import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu

TC_SIZES = [256, 512, 1024, 2048, 4096, 8192, 16384]
TC64_SIZES = [4096, 8192, 16384]


def tc_kind(n):
    return "c2c-tc64" if n in TC64_SIZES else "c2c-tc"


@pytest.fixture
def radix16(monkeypatch):
    """Plans created inside the test take the radix-16 kernels."""
    monkeypatch.setenv("FAF_CUDA_TC_RADIX", "16")


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
    assert t.kind == tc_kind(n)
    yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    assert t.tc_status() == 0
    gr, gi = yr.cpu().numpy(), yi.cpu().numpy()
    want = orc.fp64_c2c(re, im, inverse=inverse)
    e64 = orc.rel_l2_complex(gr, gi, want)
    assert e64 <= REL_L2_TOL, (n, inverse, e64)
    if n <= 4096:
        o_r, o_i = orc.c2c(re[:2], im[:2], inverse=inverse)
        assert orc.rel_l2_complex(gr[:2], gi[:2], o_r + 1j * o_i) <= REL_L2_TOL


@pytest.mark.parametrize("n", TC64_SIZES)
@pytest.mark.parametrize("inverse", [False, True])
def test_tc_radix16_kernels_where_radix64_is_default(cuda, radix16, n, inverse):
    import fastandfourier_b200 as F
    torch = cuda
    batch = max(3, 65536 // n) + 1
    re, im = heavy_tailed(n, batch, 700 + n)
    t = F.Transform.fft(n, inverse=inverse, flags=F.FLAG_TENSOR_CORE)
    assert t.kind == "c2c-tc"
    yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    assert t.tc_status() == 0
    want = orc.fp64_c2c(re, im, inverse=inverse)
    assert orc.rel_l2_complex(yr.cpu().numpy(), yi.cpu().numpy(), want) <= REL_L2_TOL


@pytest.mark.parametrize("n", TC64_SIZES)
def test_tc64_interleaved_ortho_and_unaligned(cuda, n):
    """The radix-64 kernels on interleaved buffers (ortho norm), and on split
    planes one float off 16-byte alignment, which take the direct loads."""
    import fastandfourier_b200 as F
    torch = cuda
    batch = 2 * (4096 // (n // 4096)) // 64 + 3
    re, im = heavy_tailed(n, batch, 800 + n)
    z = np.stack([re, im], axis=-1).reshape(batch, 2 * n)
    t = F.Transform.fft(n, layout=F.L_INTERLEAVED, norm=F.N_ORTHO, flags=F.FLAG_TENSOR_CORE)
    assert t.kind == "c2c-tc64"
    y = t.c2c(torch.from_numpy(z).cuda()).cpu().numpy().reshape(batch, n, 2)
    want = orc.fp64_c2c(re, im) / np.sqrt(n)
    assert orc.rel_l2_complex(y[..., 0], y[..., 1], want) <= REL_L2_TOL
    br = torch.zeros(batch * n + 1, device="cuda")
    bi = torch.zeros(batch * n + 1, device="cuda")
    br[1:] = torch.from_numpy(re.ravel()).cuda()
    bi[1:] = torch.from_numpy(im.ravel()).cuda()
    u = F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE)
    yr, yi = u.c2c(br[1:].view(batch, n), bi[1:].view(batch, n))
    assert orc.rel_l2_complex(yr.cpu().numpy(), yi.cpu().numpy(),
                              orc.fp64_c2c(re, im)) <= REL_L2_TOL
    assert t.tc_status() == 0 and u.tc_status() == 0


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
        assert t.kind not in ("c2c-tc", "c2c-tc64") and t.tc_status() == -1


@pytest.mark.parametrize("n,batch", [(8192, 400), (16384, 300), (4096, 1500)])
@pytest.mark.parametrize("radix", [16, 64])
def test_tc_landed_inputs_over_several_rounds(cuda, monkeypatch, n, batch, radix):
    """More transforms than SMs: every CTA lands a second (and third)
    transform in its workspace while it finishes the previous one (the
    radix-64 kernels from 4096 points, the radix-16 ones from 8192; the
    radix-16 4096-point kernel loads directly, over several rounds)."""
    import fastandfourier_b200 as F
    torch = cuda
    if radix == 16:
        monkeypatch.setenv("FAF_CUDA_TC_RADIX", "16")
    re, im = heavy_tailed(n, batch, 900 + n)
    t = F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE)
    assert t.kind == ("c2c-tc" if radix == 16 else "c2c-tc64")
    yr, yi = t.c2c(torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda())
    got = yr.cpu().numpy() + 1j * yi.cpu().numpy()
    want = orc.fp64_c2c(re, im)
    assert float(np.linalg.norm(got - want) / np.linalg.norm(want)) <= REL_L2_TOL
    assert t.wait_status() == 0 and t.tc_status() == 0
