"""The CUDA path finder against the reference's finder (golden fixtures) and the oracle (B200).

* finder_{cu,pack,bcc,tri} and the edge cases finder_{lone,one,two,blk,ss} (no candidate, one, two, a 600-atom
  packing over several candidate-scan blocks, single scattering alone): the same kept paths in the same order (atom
  sequences), the same degeneracies, importances within 2e-5 relative (FP32 sums in another order), the same
  reference importance, from the one-absorber call and from the batched call alike;
* batched absorbers equal one call per absorber;
* the benchmark's 3000-atom Fe/O/Pt packing (two absorbers, rmax 8 A, 8 legs, no importance cut, 1.9e5 paths) gives
  the reference finder's paths exactly;
* importance(pts, ipots) and degenerate_total against the oracle.
"""
import numpy as np
import pytest
import torch

from feffgpu_b200 import workloads as W
from oracle import pathfinder as OF
from tests.fixtures import npz, phase
from tests.test_oracle_pathfinder import CASES, finder_case

pytestmark = pytest.mark.gpu


def _finder(name, crit):
    from feffgpu_b200.pathfinder import GPUPathFinder
    z, box = finder_case(name)
    return GPUPathFinder(phase(CASES[name]), device="cuda", rmax=float(z["rmax"]), nlegmax=int(z["nlegmax"]),
                         critpw=float(crit)), z, box


@pytest.mark.parametrize("name", sorted(CASES))
def test_finder_equals_reference(name):
    z, _ = finder_case(name)
    for ci, crit in enumerate(z["crit"]):
        f, z, box = _finder(name, crit)
        kept, ref = f.enumerate(z["pos"], box, int(z["absorber"]), z["ipot"])
        assert abs(ref - float(z[f"ref_{ci}"])) <= 2e-5 * abs(float(z[f"ref_{ci}"]))
        legs = sorted(int(k.split("_")[2]) for k in z if k.startswith(f"atoms_{ci}_"))
        got = {n: v for n, v in kept.items() if v[0].shape[0] > 0}
        assert set(got) == {n for n in legs if len(z[f"atoms_{ci}_{n}"])}, (name, crit, set(got))
        for nleg in legs:
            ra = z[f"atoms_{ci}_{nleg}"]
            if len(ra) == 0:
                continue
            coords, ip, deg, xp, atoms = (t.cpu().numpy() for t in kept[nleg])
            assert np.array_equal(atoms, ra), (name, crit, nleg, atoms.shape, ra.shape)
            assert np.array_equal(deg, z[f"deg_{ci}_{nleg}"])
            assert np.allclose(xp, z[f"xport_{ci}_{nleg}"], rtol=2e-5, atol=0)
            assert coords.shape == (len(ra), nleg, 3) and np.all(coords[:, 0] == 0)
            print(f"finder_{name} critpw {crit} nleg {nleg}: {len(ra)} paths equal")
        # the batched path (one absorber slot) gives the same paths bit for bit and the same reference importance
        many = f.enumerate_many(z["pos"], box, [int(z["absorber"])], z["ipot"])
        assert float(many["ref"][0]) == ref
        got_many = {n: v for n, v in many["paths"].items() if v[0].shape[0] > 0}
        assert set(got_many) == set(got), (name, crit)
        for nleg, v in got.items():
            for x, y in zip(v, got_many[nleg][:5]):
                assert x.dtype == y.dtype and torch.equal(x, y), (name, crit, nleg)


@pytest.mark.parametrize("merge,crit", [(True, 0.5), (True, 0.0), (False, 0.5)])
def test_batched_absorbers_equal_single_calls(merge, crit):
    """enumerate_many over six absorbers (merges and cut on the device) against one enumerate per absorber (the
    single-slot merges and cut on the host): the same paths bit for bit, the same reference importance."""
    from feffgpu_b200.pathfinder import GPUPathFinder
    z, box = finder_case("pack")
    pos, ipot = z["pos"], z["ipot"]
    abs_ = [int(a) for a in np.nonzero(ipot == 1)[0][:6]]
    f = GPUPathFinder(phase("cfg2_phase"), device="cuda", rmax=5.5, nlegmax=5, critpw=crit, merge_degenerate=merge)
    many = f.enumerate_many(pos, box, abs_, ipot)
    for s, a in enumerate(abs_):
        kept, ref = f.enumerate(pos, box, a, ipot)
        assert float(many["ref"][s]) == ref
        assert set(kept) == set(many["paths"])
        for nleg, v in kept.items():
            sel = many["paths"][nleg][5] == s
            for x, y in zip(v, many["paths"][nleg][:5]):
                assert x.dtype == y.dtype and torch.equal(x, y[sel]), (a, nleg)


def test_feopt_paths_equal_reference():
    """The benchmark packing (3000 atoms, two most central Fe absorbers, rmax 8 A, 8 legs, no importance cut) in one
    batched call: per absorber and leg count the reference finder's count, atom sequences (SHA-256, first and last
    16), degeneracy sum (tests/golden/finder_feopt.npz)."""
    import hashlib
    from feffgpu_b200.pad import phase_from_npz
    from feffgpu_b200.pathfinder import GPUPathFinder
    z = npz("finder_feopt")
    pos, lab, box = W.random_packing(3000, 0.08, 1.8, seed=2024)
    ipot = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    f = GPUPathFinder(phase_from_npz(npz("cfg2_phase"), prefix="ph_"), device="cuda", rmax=8.0, nlegmax=8, critpw=0.0)
    res = f.enumerate_many(pos, box, z["absorbers"], ipot)
    for s in range(len(z["absorbers"])):
        assert abs(float(res["ref"][s]) - float(z[f"ref_{s}"])) <= 2e-5 * abs(float(z[f"ref_{s}"]))
        counts = {}
        for nleg, v in res["paths"].items():
            sel = (v[5] == s).cpu().numpy()
            atoms = np.ascontiguousarray(v[4].cpu().numpy()[sel].astype(np.int64))
            counts[nleg] = len(atoms)
            assert len(atoms) == int(z[f"count_{s}_{nleg}"])
            assert hashlib.sha256(atoms.tobytes()).digest() == bytes(z[f"sha_{s}_{nleg}"])
            assert np.array_equal(atoms[:16], z[f"head_{s}_{nleg}"]) and np.array_equal(atoms[-16:], z[f"tail_{s}_{nleg}"])
            assert float(v[2].cpu().numpy()[sel].sum()) == float(z[f"degsum_{s}_{nleg}"])
        print(f"feopt absorber {int(z['absorbers'][s])}: {counts} equal to the reference finder")


def test_importance_and_degeneracy_against_oracle():
    from feffgpu_b200.pathfinder import GPUPathFinder
    P = phase("cfg1_cu")
    f = GPUPathFinder(P, device="cuda", rmax=6.0, nlegmax=4, critpw=0.0)
    o = OF.Finder(P, rmax=6.0, nlegmax=4, critpw=0.0)
    z = npz("cfg1_cu")
    for nleg in (2, 3, 4):
        c, ip = z[f"coords_{nleg}"].astype(np.float32), z[f"ipots_{nleg}"]
        a = f.importance(torch.tensor(c), torch.tensor(ip)).cpu().numpy()
        b = o.importance(c, ip)
        assert np.allclose(a, b, rtol=2e-5, atol=0)
        if nleg > 2:
            deg = np.full(len(c), 2.0, np.float32)
            dt = GPUPathFinder.degenerate_total(torch.tensor(c), torch.tensor(deg)).numpy()
            assert np.array_equal(dt, OF.Finder.degenerate_total(c, deg))


def test_frames_batched_equal_per_frame():
    """Frames of an MD trajectory in one call: (F, n, 3) positions, (F, A) absorbers; slot = frame * A + absorber."""
    from feffgpu_b200.pathfinder import GPUPathFinder
    base, box = W.bcc_supercell(6, 2.87)
    F, A = 3, 4
    pos = np.stack([W.thermal(base, 0.08, seed=40 + f) for f in range(F)])
    rng = np.random.default_rng(1)
    abs_ = np.stack([rng.choice(len(base), A, replace=False) for _ in range(F)])
    f = GPUPathFinder(phase("cfg4_fe_phase"), device="cuda", rmax=5.5, nlegmax=4, critpw=1.0)
    many = f.enumerate_many(pos, box, abs_, np.ones(len(base), int))
    for fr in range(F):
        one = f.enumerate_many(pos[fr], box, abs_[fr], np.ones(len(base), int))
        assert torch.equal(many["ref"][fr * A:(fr + 1) * A], one["ref"])
        for nleg, v in one["paths"].items():
            w = many["paths"][nleg]
            sel = (w[5] >= fr * A) & (w[5] < (fr + 1) * A)
            for x, y in zip(v[:5], w[:5]):
                assert torch.equal(x, y[sel]), (fr, nleg)
            assert torch.equal(v[5] + fr * A, w[5][sel])


def test_symmetry_degeneracy_totals_on_ideal_lattice():
    """FEFF's merge of symmetry-equivalent paths on an ideal simple cubic cluster: single scattering in its three
    shells (6, 8, 12); triangles through two first neighbours total 24, first-second neighbour triangles 48."""
    from feffgpu_b200.pathfinder import GPUPathFinder
    from tests.test_oracle_pathfinder import check_lattice_degeneracies, simple_cubic
    f = GPUPathFinder(phase("case_W"), device="cuda", rmax=5.32, nlegmax=3, critpw=0.0)
    pos = simple_cubic()
    kept, _ = f.enumerate(pos, None, 0, np.ones(len(pos), int))
    check_lattice_degeneracies(kept, lambda c, d: GPUPathFinder.degenerate_total(c, d).cpu().numpy())


def test_paths_of_up_to_eight_legs_equal_a_plain_enumeration():
    """Every path of up to eight legs of a compact 7-atom cluster (rmax 7.4 A, no merge, no cut) against a plain
    recursive enumeration; nine legs is the largest count accepted."""
    from feffgpu_b200.pathfinder import NLEG_MAX, GPUPathFinder
    from tests.test_oracle_pathfinder import check_plain_enumeration, compact_cluster, plain_enumeration
    pos = compact_cluster()
    f = GPUPathFinder(phase("case_W"), device="cuda", rmax=7.4, nlegmax=9, critpw=0.0, merge_degenerate=False)
    kept, _ = f.enumerate(pos, None, 0, np.ones(len(pos), int))
    check_plain_enumeration(kept, plain_enumeration(pos, 7.4))
    assert NLEG_MAX == 9
    with pytest.raises(ValueError, match="between 2 and 9"):
        GPUPathFinder(phase("case_W"), device="cuda", rmax=7.4, nlegmax=10)
