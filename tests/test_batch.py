"""PathBatch's layout and launch order (host side, no GPU)."""
import numpy as np
import torch

from feffgpu_b200 import PathBatch


def _groups(rng):
    out = []
    for nleg, B in ((2, 7), (5, 300), (3, 40)):
        c = np.concatenate([np.zeros((B, 1, 3)), rng.normal(0, 2, (B, nleg - 1, 3))], 1)
        ip = np.ones((B, nleg), int)
        ip[:, 0] = 0
        out.append((c, ip, rng.random(B), rng.integers(0, 3, B)))
    return out


def test_layout_and_orders():
    rng = np.random.default_rng(0)
    gs = _groups(rng)
    b = PathBatch(gs, nrows=4, device="cpu")
    assert b.n == 347 and b.nleg_max == 5 and b.nrows == 4
    nleg = b.nleg.numpy()
    order = b.order.numpy()
    assert sorted(order.tolist()) == list(range(b.n))
    assert np.all(np.diff(nleg[order]) <= 0)             # costliest (most legs) first
    row = b.row.numpy()
    assert np.array_equal(row, np.concatenate([g[3] for g in gs]))
    assert b.max_ipot == 1 and b.counts == {2: 7, 3: 40, 5: 300}
    # padding: legs past nleg are zero
    c = b.coords.numpy()
    assert np.all(c[nleg == 2][:, 2:] == 0)
    assert torch.equal(b.coords[:7, :2].cpu(), torch.as_tensor(gs[0][0]))


def test_errors():
    import pytest
    c = np.zeros((1, 10, 3))
    with pytest.raises(ValueError):
        PathBatch([(c, np.zeros((1, 10), int))], device="cpu")
    with pytest.raises(ValueError):
        PathBatch([(np.zeros((2, 3, 3)), np.zeros((2, 3), int), None, np.array([0, 5]))], nrows=2, device="cpu")
