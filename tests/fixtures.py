"""Loaders of the golden fixtures in tests/golden (made by tests/golden/make_golden.py from the reference)."""
from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("W", "A000", "A009", "A014", "A018", "L000", "L001")


@lru_cache(maxsize=None)
def npz(name: str):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def phase(name: str):
    from feffgpu_b200.pad import phase_from_npz
    return phase_from_npz(npz(name), prefix="ph_")


def groups(name: str):
    """{nleg: (coords, ipots, deg)} of a fixture's path list."""
    z = npz(name)
    out = {}
    for k in z:
        if k.startswith("coords_"):
            n = int(k.split("_")[1])
            out[n] = (z[k], z[f"ipots_{n}"], z.get(f"deg_{n}", np.ones(len(z[k]))))
    return dict(sorted(out.items()))


def cfg2_phase(nk: int = 401, dk: float = 0.05):
    from feffgpu_b200.pad import phase_from_npz, resample_phase
    return resample_phase(phase_from_npz(npz("cfg2_phase"), prefix="ph_"), np.arange(nk) * dk)


def r_window(name: str, k):
    """kmin, kmax, rmin, rmax of the R-factor for a case (the reference's validation windows)."""
    z = npz(name)
    return dict(kmin=3.0, kmax=float(min(23.0, np.max(k) - 1.0)), rmin=1.0, rmax=float(z["rmax"]))
