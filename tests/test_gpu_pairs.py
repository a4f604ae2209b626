"""Pair tables on a B200 against the reference's PairTables (tests/golden/pairs_nio.npz, a cubic periodic box, and
pairs_nio_tri.npz, a triclinic cell) and the oracle.

Tables: every 25th row against the reference's (FP64 stage here, FP32 copies there: 1e-6 of the largest entry; the
mixed form to 2e-5).  Histogram of chosen absorbers: the reference's to 1e-9 (weights summed in 2^-32 fixed point),
the same count of short pairs, bit-identical on a repeat.  All-pairs spectrum and its position gradient: the
reference's (FP32 positions and tables there) to 1e-5 and 1e-4 of the largest value, the oracle's (FP64) to 1e-10 and
1e-9; the gradient bit-identical on a repeat and against central differences of the spectrum.
"""
import numpy as np
import pytest
import torch

from oracle import pairs as OP
from tests.fixtures import npz, phase
from tests.test_oracle_pairs import pairs_case

CASES = ["pairs_nio", "pairs_nio_tri"]

pytestmark = pytest.mark.gpu


def _tables(dtype=torch.complex128, name="pairs_nio"):
    from feffgpu_b200.pairs import PairTables
    z, box, r0, dr, rmax = pairs_case(name)
    pt = PairTables(phase("cfg5_nik_phase"), z["k"], np.zeros(len(z["k"])), 0.0, box=box,
                    rmax=rmax, r_min=r0, dr=dr, device="cuda", dtype=dtype)
    pt.ipot = torch.tensor(z["ipot"])
    return pt, z, box


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-6), (torch.complex64, 2e-5)])
def test_tables_equal_reference(dtype, tol):
    pt, z, _ = _tables(dtype)
    assert pt.nr == int(z["nr"])
    for p, t in pt.tables.items():
        ref = z[f"table_{p}"]
        assert np.abs(t.cpu().numpy()[::25] - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.parametrize("name", CASES)
def test_histogram_equals_reference_and_repeats(name):
    pt, z, box = _tables(name=name)
    h1, s1 = pt.histogram(z["pos"][0], z["absorbers"], z["ipot"], box=box)
    h2, s2 = pt.histogram(z["pos"][0], z["absorbers"], z["ipot"], box=box)
    assert torch.equal(h1, h2) and s1 == s2 == int(z["short"])
    assert np.abs(h1.cpu().numpy() - z["hist"]).max() <= 1e-9


@pytest.mark.parametrize("name", CASES)
def test_single_scattering_and_gradient(name):
    pt, z, box = _tables(name=name)
    w = torch.tensor(z["w"], device="cuda")
    out = []
    for _ in range(2):
        x = torch.tensor(z["pos"], device="cuda", requires_grad=True)
        chi = pt.single_scattering(x)
        (chi * w).sum().backward()
        out.append((chi.detach(), x.grad))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    chi, grad = out[0][0].cpu().numpy(), out[0][1].cpu().numpy()
    assert np.abs(chi - z["chi"]).max() <= 1e-5 * np.abs(z["chi"]).max()
    assert np.abs(grad - z["grad"]).max() <= 1e-4 * np.abs(z["grad"]).max()
    T = pt.T.cpu().numpy()
    oc, og = OP.single_scattering(z["pos"], box, z["ipot"], T, pt.r0, pt.dr, pt.rmax, w=z["w"])
    assert np.abs(chi - oc).max() <= 1e-10 * np.abs(oc).max()
    assert np.abs(grad - og).max() <= 1e-9 * np.abs(og).max()
    # central differences on the largest gradient entries
    with torch.no_grad():
        for idx in np.argsort(-np.abs(grad).ravel())[:4]:
            c, i, q = np.unravel_index(idx, grad.shape)
            h = 1e-5
            xp, xm = z["pos"].copy(), z["pos"].copy()
            xp[c, i, q] += h
            xm[c, i, q] -= h
            fd = float(((pt.single_scattering(torch.tensor(xp, device="cuda")) -
                         pt.single_scattering(torch.tensor(xm, device="cuda"))) * w).sum()) / (2 * h)
            assert abs(fd - grad[c, i, q]) <= 1e-6 * np.abs(grad).max(), (idx, fd, grad[c, i, q])


def test_pair_tables_equal_the_two_leg_paths_of_the_path_stage():
    """One element, every atom an absorber (a thermal bcc W block, periodic, e0 = 2 eV): the histogram of pair
    distances times the tables equals the two-leg paths of every absorber through the path finder and the fused stage,
    to the tables' 0.002 A grid (2e-3 of the largest value over k = 3..20; the reference's own check of its
    PairTables, tests/test_shared_layer.py:116-137 there), and is differentiable in the positions."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.pairs import ETOK, PairTables
    from feffgpu_b200.pathfinder import GPUPathFinder
    from feffgpu_b200 import workloads as W
    P = phase("case_W")
    sites, box = W.bcc_supercell(4, 3.1652)
    pos = sites + np.random.default_rng(0).normal(0, 0.05, sites.shape)
    k = np.arange(401) * 0.05
    pt = PairTables(P, k, np.zeros(len(k)), 2.0, box=box, rmax=6.0, device="cuda", dtype=torch.complex64)
    x = torch.tensor(pos, device="cuda", dtype=torch.float32)[None]
    chi = pt.single_scattering(x).cpu().numpy()
    f = GPUPathFinder(P, device="cuda", rmax=6.0, nlegmax=2, critpw=0.0, merge_degenerate=False)
    res = f.enumerate_many(pos, box, np.arange(len(pos)), np.ones(len(pos), int))
    coords, ipots, deg, _xp, _atoms, _slot = res["paths"][2]
    st = GPUPathStage(P, device="cuda", dtype=torch.complex64)
    batch = PathBatch([(coords.double(), ipots, deg.double(), None)], nrows=1, device="cuda")
    en = k ** 2 - 2.0 * ETOK
    q = np.sign(en) * np.sqrt(np.abs(en))
    ref = st.chi_reduce(batch, q)[0].cpu().numpy() / len(pos)
    sel = (k > 3) & (k < 20)
    e = np.abs(chi - ref)[sel].max() / np.abs(ref[sel]).max()
    print(f"pair tables vs two-leg paths of the stage: {e:.2e}")
    assert e < 2e-3
    xg = x.clone().requires_grad_(True)
    (pt.single_scattering(xg) ** 2).sum().backward()
    assert torch.isfinite(xg.grad).all() and float(xg.grad.abs().max()) > 0
