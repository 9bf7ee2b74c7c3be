"""Inverse STFT (faf_cuda_create_istft): frames -> irfft -> Hann window ->
overlap-add / summed squared window, against the FP64 oracle and as the
inverse of the framed STFT."""
import numpy as np
import pytest

from conftest import REL_L2_TOL, seeded
from oracle import orc

pytestmark = pytest.mark.gpu


def well_covered(frames, n, win, hop):
    """Samples whose window envelope is at least 1 % of its peak: there the
    division by the envelope is well conditioned (near the ends of a
    symmetric Hann window it divides by ~0)."""
    i = np.arange(win)
    w = 0.5 * (1 - np.cos(2 * np.pi * i / (win - 1)))
    env = np.zeros((frames - 1) * hop + win)
    for f in range(frames):
        env[f * hop:f * hop + win] += w * w
    return env >= 0.01 * env.max()


@pytest.mark.parametrize("n,win,hop", [(1024, 1024, 256), (512, 400, 160), (2048, 2048, 512),
                                       (1000, 800, 200)])
def test_istft_matches_oracle(cuda, n, win, hop):
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(n + win)
    frames = 37
    nb = n // 2 + 1
    Xr = rng.standard_normal((3, frames, nb)).astype(np.float32)
    Xi = rng.standard_normal((3, frames, nb)).astype(np.float32)
    Xi[..., 0] = 0
    Xi[..., -1] = 0
    t = F.Transform.istft(n, win=win, hop=hop)
    assert t.kind == "istft"
    y = t.istft_frames(torch.from_numpy(Xr).cuda(), torch.from_numpy(Xi).cuda()).cpu().numpy()
    want = orc.istft(Xr, Xi, n, win, hop)
    assert y.shape == want.shape == (3, (frames - 1) * hop + win)
    m = well_covered(frames, n, win, hop)
    assert orc.rel_l2(y[:, m], want[:, m]) <= REL_L2_TOL
    assert np.all(y[:, 0] == 0)  # zero window envelope


def test_istft_more_signals_than_grid_rows(cuda):
    """70000 signals: the overlap-add walks signals along the grid's y axis
    (at most 65535 rows), so signals past the first 65535 take a second
    pass.  Every signal matches the FP64 oracle."""
    import fastandfourier_b200 as F
    torch = cuda
    n = win = 64
    hop, frames, n_sig = 16, 9, 70000
    nb = n // 2 + 1
    rng = seeded(70000)
    Xr = rng.standard_normal((n_sig, frames, nb)).astype(np.float32)
    Xi = rng.standard_normal((n_sig, frames, nb)).astype(np.float32)
    Xi[..., 0] = 0
    Xi[..., -1] = 0
    t = F.Transform.istft(n, win=win, hop=hop)
    y = t.istft_frames(torch.from_numpy(Xr).cuda(), torch.from_numpy(Xi).cuda()).cpu().numpy()
    m = well_covered(frames, n, win, hop)
    for sl in (slice(0, 3), slice(65533, 65538), slice(n_sig - 3, n_sig)):
        want = orc.istft(Xr[sl], Xi[sl], n, win, hop)
        assert orc.rel_l2(y[sl][:, m], want[:, m]) <= REL_L2_TOL


def test_istft_inverts_stft(cuda):
    import fastandfourier_b200 as F
    torch = cuda
    rng = seeded(77)
    L = 1 << 16
    x = rng.standard_normal((2, L)).astype(np.float32)
    s = F.Transform.stft(1024, win=1024, hop=256)
    Xr, Xi = s.stft_frames(torch.from_numpy(x).cuda())
    y = F.Transform.istft(1024, win=1024, hop=256).istft_frames(Xr, Xi).cpu().numpy()
    Lr = y.shape[-1]
    sl = slice(256, Lr - 256)  # interior: window envelope well above zero
    assert orc.rel_l2(y[:, sl], x[:, :Lr][:, sl]) <= REL_L2_TOL


def test_istft_host_buffers_and_errors(cuda):
    import fastandfourier_b200 as F
    rng = seeded(78)
    Xr = rng.standard_normal((1, 9, 257)).astype(np.float32)
    Xi = rng.standard_normal((1, 9, 257)).astype(np.float32)
    t = F.Transform.istft(512, win=512, hop=128)
    y = t.istft_frames(Xr, Xi)
    m = well_covered(9, 512, 512, 128)
    assert orc.rel_l2(y[:, m], orc.istft(Xr, Xi, 512, 512, 128)[:, m]) <= REL_L2_TOL
    with pytest.raises(F.FafError):
        F.Transform.istft(512, win=600, hop=128)
    with pytest.raises(F.FafError):
        F.Transform.istft(1023, win=512, hop=128)
