"""Periodic cells in the forms the reference's front ends pass them (src/feffgpu/cell.py:11-35): None (a cluster), a
cubic length, (3,) edge lengths of an orthorhombic cell, or a 3 x 3 cell with the lattice vectors as rows.  The
minimum image is the reference's: the cubic rule rel - b round(rel / b) for a length, fractional rounding
(f = rel inv(cell), rel = (f - round(f)) cell) for a cell."""
from __future__ import annotations

import numpy as np
import torch


def as_cell(box):
    """None -> None; a number (or 0-d tensor) -> float; (3,) -> the diagonal cell; (3, 3) -> the cell (float64)."""
    if box is None:
        return None
    if torch.is_tensor(box):
        if box.dim() == 0:
            return float(box)
        c = box.detach().cpu().numpy().astype(np.float64)
    else:
        if np.isscalar(box):
            return float(box)
        c = np.asarray(box, np.float64)
    if c.shape == (3,):
        c = np.diag(c)
    if c.shape != (3, 3):
        raise ValueError("box must be None, a length, (3,) edge lengths or a 3 x 3 cell (lattice vectors as rows)")
    if abs(np.linalg.det(c)) <= 0.0:
        raise ValueError("the periodic cell is singular")
    return c


def cell_words(cell: np.ndarray, dtype) -> np.ndarray:
    """(18,) the cell (row-major) and then its inverse, both in dtype, the inverse computed in dtype as the reference
    computes it (torch.linalg.inv of the cell in the working precision)."""
    tdt = torch.float32 if np.dtype(dtype) == np.float32 else torch.float64
    c = torch.tensor(cell, dtype=tdt)
    inv = torch.linalg.inv(c)
    return np.concatenate([c.numpy().ravel(), inv.numpy().ravel()]).astype(dtype)


def min_width(cell) -> float:
    """The smallest perpendicular width of a cell from as_cell (A): the length of a cubic box, inf for a cluster."""
    if cell is None:
        return float("inf")
    if isinstance(cell, float):
        return cell
    vol = abs(np.linalg.det(cell))
    return float(min(vol / np.linalg.norm(np.cross(cell[(i + 1) % 3], cell[(i + 2) % 3])) for i in range(3)))
