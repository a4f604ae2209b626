"""PathBatch's launch order and fixed summation order (host-side layout, no GPU)."""
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
    b = PathBatch(gs, nrows=4, device="cpu", chunk=64)
    assert b.n == 347 and b.nleg_max == 5 and b.nrows == 4
    nleg = b.nleg.numpy()
    order = b.order.numpy()
    assert sorted(order.tolist()) == list(range(b.n))
    assert np.all(np.diff(nleg[order]) <= 0)             # costliest (most legs) first
    row = b.row.numpy()
    srt = b.sorted.numpy()
    assert np.all(np.diff(row[srt]) >= 0)               # grouped by row
    bounds, rc = b.chunk_bounds.numpy(), b.row_chunks.numpy()
    assert bounds[0] == 0 and bounds[-1] == b.n and np.all(np.diff(bounds) <= 64) and np.all(np.diff(bounds) > 0)
    assert rc[0] == 0 and rc[-1] == b.nchunks and len(rc) == b.nrows + 1
    for r in range(b.nrows):                            # every chunk of a row holds only that row's paths
        for c in range(rc[r], rc[r + 1]):
            assert np.all(row[srt[bounds[c]:bounds[c + 1]]] == r)
    assert rc[4] - rc[3] == 0                           # an empty row owns no chunk
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
