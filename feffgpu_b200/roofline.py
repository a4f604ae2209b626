"""Algorithmic work of the path stage, the numerator of the roofline.

The unit is one (path, energy) pair.  Its algorithmic FLOP count is the one tabulated for the reference's literal
port of FEFF's GENFMT (``src/feffgpu/genfmt.py:306-447``: scattering matrices, chain product, termination, trace,
cfac; complex multiply 6, complex add 2, complex x real 2, masked terms excluded), K edge, at a uniform number of
partial waves L = lmax + 1:

    legs          2       3       4       5       6       7       8
    L = 25   12,342  17,246  28,718  40,190  51,662  63,134  74,606
    L = 21   10,534  14,614  24,366  34,118  43,870  53,622  63,374

For every leg count the count is affine in L (the partial-wave sums are linear in L), so the two rows fix it:
flops(nleg, L) = A(nleg) + B(nleg) L.  A path's L at one energy is the mean over its scatterers of
lmax(e, ipot) + 1, the partial-wave limit FEFF applies per scatterer and energy.

This counts what the reference computes, not what this package's kernels execute: they fold the Legendre factors
into the per-path rotation tables, accumulate only the flip-canonical scattering-matrix entries and stream the
spherical-wave recursion, so they issue fewer operations for the same result.
"""
from __future__ import annotations

import numpy as np

_L25 = {2: 12342, 3: 17246, 4: 28718, 5: 40190, 6: 51662, 7: 63134, 8: 74606}
_L21 = {2: 10534, 3: 14614, 4: 24366, 5: 34118, 6: 43870, 7: 53622, 8: 63374}
SLOPE = {n: (_L25[n] - _L21[n]) / 4.0 for n in _L25}
OFFSET = {n: _L25[n] - 25 * SLOPE[n] for n in _L25}
# nine legs continue the per-leg increments
SLOPE[9] = 2 * SLOPE[8] - SLOPE[7]
OFFSET[9] = 2 * OFFSET[8] - OFFSET[7]


def flops_per_energy(nleg: int, L: float) -> float:
    """Algorithmic FLOPs of one path at one energy with (mean) partial-wave count L."""
    return OFFSET[nleg] + SLOPE[nleg] * L


def path_flops(nleg, ipots, lmax_e_ip) -> np.ndarray:
    """Algorithmic FLOPs of every path over all energies (n,): the per-path cost the multi-GPU split balances."""
    nleg = np.asarray(nleg, int)
    ipots = np.asarray(ipots, int)
    L = np.asarray(lmax_e_ip, float) + 1.0
    out = np.zeros(len(nleg))
    for n in np.unique(nleg):
        sel = np.nonzero(nleg == n)[0]
        sc = ipots[sel, 1:n]
        counts = np.zeros((len(sc), L.shape[1]))
        np.add.at(counts, (np.repeat(np.arange(len(sc)), n - 1), sc.ravel()), 1.0)
        mean_L = counts @ L.T / (n - 1)
        out[sel] = np.sum(OFFSET[int(n)] + SLOPE[int(n)] * mean_L, axis=1)
    return out


def batch_flops(nleg, ipots, lmax_e_ip) -> float:
    """Total algorithmic FLOPs of a batch over all energies.  nleg (n,), ipots (n, nleg_max) absorber first,
    lmax_e_ip (E, nph+1) the stage's lmax table."""
    nleg = np.asarray(nleg, int)
    ipots = np.asarray(ipots, int)
    L = np.asarray(lmax_e_ip, float) + 1.0                      # (E, nph+1)
    total = 0.0
    for n in np.unique(nleg):
        sel = nleg == n
        sc = ipots[sel, 1:n]                                    # scatterers' potentials
        # sum over paths and energies of the mean scatterer L: per energy, average L[e, ip] over the scatterers
        counts = np.zeros((len(sc), L.shape[1]))
        np.add.at(counts, (np.repeat(np.arange(len(sc)), n - 1), sc.ravel()), 1.0)
        mean_L = counts @ L.T / (n - 1)                         # (paths, E)
        total += float(np.sum(OFFSET[int(n)] + SLOPE[int(n)] * mean_L))
    return total
