"""CPU restatement of the reference's single-scattering pair tables (src/feffgpu/exafs/forward.py:178-320) -- test
infrastructure only (the checker of feffgpu_b200/pairs.py and csrc/fg_pairs.cu; never used by the product).

* tables (forward.py:226-243): per scatterer potential p, the two-leg chi(q) of a path along z at every distance of
  the grid r_min + dr * i, i < nr = round((rmax - r_min) / dr) + 1, from the oracle's path stage (FP64);
* histogram (forward.py:248-289): for chosen absorbers of one configuration, every neighbour j with
  1e-6 < r^2 <= rmax^2 (minimum image) adds 1 - f to bin i0 and f to bin i0 + 1 of row ipot[j], with
  u = (r - r_min) / dr, i0 = clamp(floor(u), 0, nr - 2), f = clamp(u - i0, 0, 1); pairs closer than r_min are counted;
* single scattering (forward.py:303-319): every atom of every copy an absorber, chi = sum_p h_p @ T_p / (C n), and its
  gradient with respect to the positions (the derivative of the interpolation weight, 1/dr where 0 <= u - i0 <= 1).
Pinned against the reference's outputs in tests/golden/pairs_nio.npz.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def grid(r_min, rmax, dr):
    nr = int(round((rmax - r_min) / dr)) + 1
    return nr, r_min + dr * np.arange(nr)


def tables(P, q, r_min=1.5, rmax=9.4, dr=0.002):
    """(nph, nr, NK) FP64: row i of table p is the two-leg chi(q) at distance r_i for scatterer potential p + 1."""
    orc = O.Oracle(P)
    S = orc.linear_matrix(q)
    nr, r = grid(r_min, rmax, dr)
    out = np.zeros((P.nph, nr, len(q)))
    coords = np.zeros((nr, 2, 3))
    coords[:, 1, 2] = r
    for p in range(1, P.nph + 1):
        ipots = np.tile(np.array([[0, p]]), (nr, 1))
        cc, rf = orc.cchi(coords, ipots)
        out[p - 1] = O.chi_fine(cc, rf, q, S)
    return out


def _pairs(pos, a, box, rmax):
    rel = pos - pos[a]
    if box is not None and np.ndim(box) == 0:
        rel = rel - box * np.round(rel / box)
    elif box is not None:
        # a cell (cell.py:11-35): (3,) edges -> the diagonal cell; f = rel inv(cell), rel = (f - round(f)) cell
        c = np.asarray(box, float)
        c = np.diag(c) if c.shape == (3,) else c
        f = rel @ np.linalg.inv(c)
        rel = (f - np.round(f)) @ c
    r2 = (rel * rel).sum(-1)
    mask = (r2 <= rmax * rmax) & (r2 > 1e-6)
    return np.nonzero(mask)[0], rel[mask], np.sqrt(r2[mask])


def _weights(r, r_min, dr, nr):
    u = (r - r_min) / dr
    i0 = np.clip(np.floor(u), 0, nr - 2).astype(int)
    f = np.clip(u - i0, 0.0, 1.0)
    inside = (u - i0 >= 0.0) & (u - i0 <= 1.0)
    return i0, f, inside


def histogram(pos, absorbers, ipot, box, r_min, dr, nr, rmax, nph):
    """(nph + 1, nr) FP64 histogram of the absorbers' neighbour distances and the number of pairs below r_min."""
    pos = np.asarray(pos, float)
    h = np.zeros((nph + 1, nr))
    short = 0
    for a in absorbers:
        j, _rel, r = _pairs(pos, int(a), box, rmax)
        short += int((r < r_min).sum())
        i0, f, _ = _weights(r, r_min, dr, nr)
        np.add.at(h, (ipot[j], i0), 1.0 - f)
        np.add.at(h, (ipot[j], i0 + 1), f)
    return h, short


def single_scattering(pos, box, ipot, T, r_min, dr, rmax, w=None):
    """chi (NK,) of pos (C, n, 3), every atom an absorber, averaged over C n; with w (NK,) also the gradient of
    sum_k w_k chi_k with respect to pos (C, n, 3)."""
    pos = np.asarray(pos, float)
    C, n, _ = pos.shape
    nph, nr, NK = T.shape
    chi = np.zeros(NK)
    grad = np.zeros_like(pos) if w is not None else None
    D = T @ w if w is not None else None                     # (nph, nr)
    for c in range(C):
        for a in range(n):
            j, rel, r = _pairs(pos[c], a, box, rmax)
            i0, f, inside = _weights(r, r_min, dr, nr)
            p = ipot[j] - 1
            chi += ((1.0 - f)[:, None] * T[p, i0] + f[:, None] * T[p, i0 + 1]).sum(0)
            if w is not None:
                s = np.where(inside, (D[p, i0 + 1] - D[p, i0]) / dr, 0.0) / (C * n)
                g = s[:, None] * rel / r[:, None]                # d/d pos_j of the pair's term
                np.add.at(grad[c], j, g)
                grad[c, a] -= g.sum(0)
    return chi / (C * n), grad
