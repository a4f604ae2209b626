"""Periodic cells in the reference's forms (feffgpu_b200.cell, feffgpu_b200.model.MinImage; no GPU): the forms
as_cell accepts, the cell words the kernels read, and the minimum image against the reference's rule
(src/feffgpu/cell.py:26-35) restated in numpy."""
import numpy as np
import pytest
import torch

from feffgpu_b200.cell import as_cell, cell_words
from feffgpu_b200.model import MinImage


def test_forms():
    assert as_cell(None) is None
    assert as_cell(12.5) == 12.5 and as_cell(torch.tensor(12.5)) == 12.5
    assert np.array_equal(as_cell([10.0, 11.0, 12.0]), np.diag([10.0, 11.0, 12.0]))
    c = np.array([[10.0, 0, 0], [2.0, 11.0, 0], [1.0, -1.5, 12.0]])
    assert np.array_equal(as_cell(torch.tensor(c, dtype=torch.float32)), c.astype(np.float32).astype(float))
    with pytest.raises(ValueError):
        as_cell(np.zeros((2, 3)))
    with pytest.raises(ValueError):
        as_cell(np.zeros((3, 3)))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_cell_words_hold_the_cell_and_its_inverse(dtype):
    c = np.array([[10.0, 0, 0], [2.1, 11.0, 0], [1.3, -1.7, 12.0]])
    w = cell_words(c, dtype)
    assert w.dtype == dtype and w.shape == (18,)
    assert np.allclose(w[:9].reshape(3, 3) @ w[9:].reshape(3, 3), np.eye(3), atol=1e-6 if dtype == np.float32 else 1e-14)


def test_min_image_matches_the_reference_rule():
    rng = np.random.default_rng(0)
    c = 12.0 * np.array([[1.0, 0, 0], [0.21, 1.0, 0], [0.13, -0.17, 1.0]])
    rel = rng.uniform(-30, 30, size=(500, 3))
    f = rel @ np.linalg.inv(c)
    want = (f - np.round(f)) @ c
    got = MinImage(c, "cpu")(torch.tensor(rel)).numpy()
    assert np.abs(got - want).max() < 1e-10
    cub = MinImage(12.0, "cpu")(torch.tensor(rel)).numpy()
    assert np.allclose(cub, rel - 12.0 * np.round(rel / 12.0))
    assert np.array_equal(MinImage(None, "cpu")(torch.tensor(rel)).numpy(), rel)


def test_min_width_and_the_pair_tables_refuse_narrow_cells():
    """The smallest perpendicular width of a cell; PairTables refuses a cell narrower than twice its cutoff, as the
    reference's front end does, before it touches a device."""
    from feffgpu_b200.cell import min_width
    from feffgpu_b200.pairs import PairTables
    assert min_width(None) == float("inf") and min_width(11.0) == 11.0
    c = np.array([[10.0, 0, 0], [5.0, 10.0, 0], [0, 0, 12.0]])
    assert abs(min_width(c) - 10.0 * 10.0 / np.hypot(5.0, 10.0)) < 1e-12
    with pytest.raises(ValueError, match="narrower than twice the cutoff"):
        PairTables(None, np.arange(10) * 0.1, box=11.0, rmax=6.0)
    with pytest.raises(ValueError, match="narrower than twice the cutoff"):
        PairTables(None, np.arange(10) * 0.1, box=c, rmax=5.0)
