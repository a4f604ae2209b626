"""The path-finder oracle (oracle/pathfinder.py) against the reference finder's own outputs (tests/golden/finder_*.npz):
the same paths in the same order, the same degeneracies, importances to FP32 rounding, the same reference
importance."""
import numpy as np
import pytest

from oracle import pathfinder as OF
from tests.fixtures import npz, phase

CASES = {"cu": "cfg1_cu", "pack": "cfg2_phase", "bcc": "cfg4_fe_phase", "tri": "cfg4_fe_phase",
         # edge cases: no candidate, one, two; a 600-atom packing over several candidate-scan blocks; 2 legs only
         "lone": "cfg4_fe_phase", "one": "cfg4_fe_phase", "two": "cfg4_fe_phase", "blk": "cfg2_phase",
         "ss": "cfg2_phase"}


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


# -- known answers of the reference's own finder tests (tests/test_pathfinder.py:93-162 there), restated ------------
A_SC = 2.823


def simple_cubic(m=3):
    """An ideal simple cubic cluster (lattice constant A_SC, (2m + 1)^3 sites) sorted by distance from the origin."""
    cells = np.stack(np.meshgrid(*[np.arange(-m, m + 1)] * 3, indexing="ij"), -1).reshape(-1, 3) * A_SC
    return cells[np.argsort(np.linalg.norm(cells, axis=1), kind="stable")]


def compact_cluster(seed=3):
    """The absorber and six atoms 1.7 A from it along the axes, slightly displaced: paths of up to eight legs fit
    inside a cutoff of 7.4 A."""
    pos = np.vstack([np.zeros(3), 1.7 * np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])])
    pos[1:] += np.random.default_rng(seed).normal(0, 0.05, (6, 3))
    return np.round(pos, 5)


def plain_enumeration(pos, rmax):
    """Every sequence of scatterers within the cutoff, built without a finder: first and last atom not the absorber,
    no atom following itself, a path and its reverse once, degeneracy 2 (1 for a palindrome); {nleg: {seq: deg}}."""
    D = np.linalg.norm(pos[:, None] - pos[None], axis=2)
    plain = {}

    def grow(seq, length):
        last = seq[-1]
        if last != 0 and length + D[last, 0] <= 2 * rmax:
            plain.setdefault(len(seq) + 1, {})[min(seq, tuple(reversed(seq)))] = 1.0 if seq == tuple(reversed(seq)) else 2.0
        if len(seq) == 8:
            return
        for nxt in range(len(pos)):
            if nxt != last and length + D[last, nxt] + D[nxt, 0] <= 2 * rmax:
                grow(seq + (nxt,), length + D[last, nxt])
    for first in range(1, len(pos)):
        grow((first,), D[0, first])
    return plain


def check_lattice_degeneracies(kept, degenerate_total):
    """Single scattering merged into its three shells (6, 8, 12); the right-angle triangles through two first
    neighbours total 24, the first-second neighbour triangles 48, every member listed (FEFF's paths.dat)."""
    coords, ipots, deg, xp, atoms = (np.asarray(v.cpu() if hasattr(v, "cpu") else v) for v in kept[2])
    assert sorted(deg.tolist()) == [6.0, 8.0, 12.0]
    coords, ipots, deg, xp, atoms = kept[3]
    tot = np.asarray(degenerate_total(coords, deg))
    coords = np.asarray(coords.cpu() if hasattr(coords, "cpu") else coords)
    d1, d2 = np.linalg.norm(coords[:, 1], axis=1), np.linalg.norm(coords[:, 2], axis=1)
    ff = (np.abs(d1 - A_SC) < 1e-3) & (np.abs(d2 - A_SC) < 1e-3)
    fs = ((np.abs(d1 - A_SC) < 1e-3) & (np.abs(d2 - A_SC * 2 ** 0.5) < 1e-3)) | \
         ((np.abs(d2 - A_SC) < 1e-3) & (np.abs(d1 - A_SC * 2 ** 0.5) < 1e-3))
    assert ff.sum() == 12 and np.all(tot[ff] == 24.0)
    assert fs.sum() == 24 and np.all(tot[fs] == 48.0)


def check_plain_enumeration(kept, plain):
    mine = {}
    for n, (coords, ipots, deg, xp, atoms) in kept.items():
        atoms, ipots, deg = (np.asarray(v.cpu() if hasattr(v, "cpu") else v) for v in (atoms, ipots, deg))
        assert np.all((atoms == 0) == (ipots[:, 1:] == 0))         # the absorber inside a path keeps potential 0
        for a, d in zip(atoms.tolist(), deg.tolist()):
            key = min(tuple(a), tuple(reversed(a)))
            assert key not in mine.setdefault(n, {})                 # no path twice
            mine[n][key] = d
    assert set(plain) == set(mine) == {2, 3, 4, 5, 6, 7, 8} and len(plain[8]) > 500 and len(plain[6]) > 2000
    for n in plain:
        assert plain[n] == mine[n], n


def test_oracle_symmetry_degeneracy_totals_on_ideal_lattice():
    f = OF.Finder(phase("case_W"), rmax=5.32, nlegmax=3, critpw=0.0)
    pos = simple_cubic()
    kept, _ = f.enumerate(pos, None, 0, np.ones(len(pos), int))
    check_lattice_degeneracies(kept, OF.Finder.degenerate_total)


def test_oracle_paths_of_up_to_eight_legs_equal_a_plain_enumeration():
    pos = compact_cluster()
    f = OF.Finder(phase("case_W"), rmax=7.4, nlegmax=9, critpw=0.0, merge_degenerate=False)
    kept, _ = f.enumerate(pos, None, 0, np.ones(len(pos), int))
    check_plain_enumeration(kept, plain_enumeration(pos, 7.4))
