"""The path-finder oracle (oracle/pathfinder.py) against the reference finder's own outputs (tests/golden/finder_*.npz):
the same paths in the same order, the same degeneracies, importances to FP32 rounding, the same reference
importance."""
import numpy as np
import pytest

from oracle import pathfinder as OF
from tests.fixtures import npz, phase

CASES = {"cu": "cfg1_cu", "pack": "cfg2_phase", "bcc": "cfg4_fe_phase", "tri": "cfg4_fe_phase"}


def finder_case(name):
    """(fixture, box: None, the cubic length or the 3 x 3 triclinic cell)."""
    z = npz(f"finder_{name}")
    if "cell" in z:
        return z, z["cell"]
    box = float(z["box"]) if float(z["box"]) > 0 else None
    return z, box


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_equals_reference_finder(name):
    z, box = finder_case(name)
    P = phase(CASES[name])
    for ci, crit in enumerate(z["crit"]):
        f = OF.Finder(P, rmax=float(z["rmax"]), nlegmax=int(z["nlegmax"]), critpw=float(crit))
        kept, ref = f.enumerate(z["pos"], box, int(z["absorber"]), z["ipot"])
        assert abs(ref - float(z[f"ref_{ci}"])) <= 1e-6 * abs(float(z[f"ref_{ci}"]))
        legs = sorted(int(k.split("_")[2]) for k in z if k.startswith(f"atoms_{ci}_"))
        for nleg in legs:
            ra = z[f"atoms_{ci}_{nleg}"]
            coords, ip, deg, xp, atoms = kept.get(nleg, (np.zeros((0, nleg, 3)), None, np.zeros(0), np.zeros(0),
                                                         np.zeros((0, nleg - 1), int)))
            assert atoms.shape == ra.shape and np.array_equal(atoms, ra), (name, crit, nleg)
            assert np.array_equal(deg, z[f"deg_{ci}_{nleg}"])
            assert np.allclose(xp, z[f"xport_{ci}_{nleg}"], rtol=2e-5, atol=0)
        assert set(kept) <= set(legs) | {n for n in kept if len(kept[n][4]) == 0}


def test_fbeta_table_matches_legendre_recurrence():
    """|f(beta)| from scipy's Legendre polynomials (the reference's) and from the three-term recurrence the CUDA
    finder's host code uses."""
    from feffgpu_b200.pathfinder import fbeta_table
    P = phase("cfg1_cu")
    a, b = OF.fbeta_table(P), fbeta_table(P)
    assert a.shape == b.shape and np.allclose(a, b, rtol=1e-5, atol=1e-6 * a.max())
