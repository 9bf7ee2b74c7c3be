"""faf_cuda_execute_c2c_noalloc: the four-step C2C with its scratch in a fixed
array instead of an allocation, for callers that must not allocate device
memory while they run (a real-time callback that cannot wait inside the
driver's allocator, or a program whose device memory is fully reserved by
another allocator).

Checked through the C ABI against the regular entry point (faf_execute_batched
on the same plan) on two calls in a row: the array keeps the previous call's
contents and the second call must not depend on them.  The file is named so
that pytest collects it last: a run that stops at the first failure has run
every other test before it."""
import ctypes

import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_call_allocates_nothing(cuda):
    """On a freshly created plan, the driver's free device memory is the same
    before and after a call: creating the plan set up the static array and
    loaded the kernels, so the call itself allocates nothing."""
    import fastandfourier_b200 as F
    torch = cuda
    L = F.lib()
    n, batch = 65536, 3
    rng = seeded(901)
    re = torch.from_numpy(rng.uniform(-1, 1, (batch, n)).astype(np.float32)).cuda()
    im = torch.from_numpy(rng.uniform(-1, 1, (batch, n)).astype(np.float32)).cuda()
    out_r, out_i = torch.empty_like(re), torch.empty_like(im)
    t = F.Transform.fft(n)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = L.faf_cuda_execute_c2c_noalloc(t.ptr, _ptr(out_r), _ptr(out_i), _ptr(re), _ptr(im), batch)
    assert rc == 0, F.C.error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    exact = orc.fp64_c2c(re.cpu().numpy(), im.cpu().numpy())
    assert orc.rel_l2_complex(out_r.cpu().numpy(), out_i.cpu().numpy(), exact) <= REL_L2_TOL


@pytest.mark.parametrize("n,inverse,batches", [
    (32768, False, (5, 6)), (65536, False, (5, 6)), (40000, True, (5, 6)),
    # past one chunk of the array: 64 transforms of 32768, 32 of 65536 fit
    (32768, True, (70, 3)), (65536, False, (40, 33))])
def test_noalloc_matches_regular_entry_point_twice(cuda, n, inverse, batches):
    import fastandfourier_b200 as F
    torch = cuda
    L = F.lib()
    t = F.Transform.fft(n, inverse=inverse)
    assert t.kind == "c2c-4step"
    for call, batch in enumerate(batches):
        rng = seeded(500 + n + call + batch)
        re = torch.from_numpy(rng.uniform(-1, 1, (batch, n)).astype(np.float32)).cuda()
        im = torch.from_numpy(rng.uniform(-1, 1, (batch, n)).astype(np.float32)).cuda()
        want_r, want_i = t.c2c(re, im)
        got_r, got_i = torch.empty_like(re), torch.empty_like(im)
        rc = L.faf_cuda_execute_c2c_noalloc(t.ptr, _ptr(got_r), _ptr(got_i), _ptr(re), _ptr(im),
                                            batch)
        assert rc == 0, F.C.error()
        torch.cuda.synchronize()
        w = want_r.cpu().numpy() + 1j * want_i.cpu().numpy()
        g_r, g_i = got_r.cpu().numpy(), got_i.cpu().numpy()
        assert orc.rel_l2_complex(g_r, g_i, w) <= REL_L2_TOL
        exact = orc.fp64_c2c(re.cpu().numpy(), im.cpu().numpy(), inverse=inverse)
        assert orc.rel_l2_complex(g_r, g_i, exact) <= REL_L2_TOL


def test_noalloc_rejects_what_it_cannot_run(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    L = F.lib()
    small = F.Transform.fft(1024)
    buf = torch.zeros(1024, device="cuda")
    assert L.faf_cuda_execute_c2c_noalloc(small.ptr, _ptr(buf), _ptr(buf), _ptr(buf), _ptr(buf),
                                          1) != 0
    assert "four-step" in F.C.error()
    big = F.Transform.fft(32768)
    h = np.zeros(32768, np.float32)
    hp = ctypes.c_void_p(h.ctypes.data)
    assert L.faf_cuda_execute_c2c_noalloc(big.ptr, hp, hp, hp, hp, 1) != 0
    assert "device memory" in F.C.error()
