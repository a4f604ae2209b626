"""The benchmark configurations as parity cases (B200).

1. Cu fcc 6 A cluster, K edge: the reference chain's own phases and path finder output (317 paths), chi on
   k = 0..20 step 0.05 against the reference's FP64 chi (R <= 1e-6 mixed, 1e-12 FP64).
3. Adjoint on an 800-atom Fe/O/Pt packing: the path finder's paths, the gradient of the reference's R-space misfit
   with respect to every position against the reference's own autograd, per-path sigma^2 against central
   differences, FP32-vs-FP64 gradient error stated.
4. MD batch: frames of the thermally displaced bcc Fe 16^3 supercell x 32 absorbers, the finder's paths in one
   launch, chi averaged per frame, against the oracle's FP64 sums.
5. Two-edge refinement (Ni K + O K of the 8^3 rock-salt NiO model with vacancies, finder paths): the step captured
   as a CUDA graph equals the eager step and the misfit falls.
"""
import numpy as np
import pytest
import torch

from feffgpu_b200 import workloads as W
from oracle import oracle as O
from tests.fixtures import groups, npz, phase

pytestmark = pytest.mark.gpu

K401 = np.arange(401) * 0.05


def _R(k, ref, x):
    return O.r_factor(np.asarray(k), ref, x, kmin=3.0, kmax=19.0, rmin=1.0, rmax=6.0)


@pytest.mark.parametrize("dtype,tol", [(torch.complex64, 1e-6), (torch.complex128, 1e-12)])
def test_cfg1_cu_cluster(dtype, tol):
    from feffgpu_b200 import GPUPathStage, PathBatch
    z = npz("cfg1_cu")
    st = GPUPathStage(phase("cfg1_cu"), device="cuda", dtype=dtype)
    gs = groups("cfg1_cu")
    assert {n: len(v[0]) for n, v in gs.items()} == {2: 5, 3: 234, 4: 78}
    rows = st.chi_reduce(PathBatch([(c, i, d) for c, i, d in gs.values()], device="cuda"), K401)[0].cpu().numpy()
    R = _R(K401, z["ref_chi"], rows)
    print(f"cfg1 fused {dtype}: R {R:.2e}")
    assert R <= tol
    # the chain's own loop over leg counts (chain.py:45-49) through the drop-in methods
    S = st.linear_matrix(K401)
    chi = torch.zeros(len(K401), dtype=torch.float64, device="cuda")
    with torch.no_grad():
        for c, i, d in gs.values():
            cc, rf = st.cchi(torch.tensor(c), torch.tensor(i))
            chi += (torch.tensor(d, device="cuda")[:, None] * st.chi_fine(cc, rf, K401, S, "feff").double()).sum(0)
    assert _R(K401, z["ref_chi"], chi.cpu().numpy()) <= tol


def test_cfg3_adjoint_800_atoms():
    """Configuration 3 against the reference's own forward model and autograd (tests/golden/cfg3_adjoint.npz: its
    PathSpectra -- path finder, complex128 stage under non-reentrant checkpointing, R-space misfit -- on the seeded
    800-atom Fe/O/Pt packing, 16 Fe absorbers, rmax 5 A, 4 legs, importance cut 0.5 %, target from a 0.05 A Gaussian
    displacement).  This package: the CUDA finder's paths (the same lists), PathModel + chi_reduce, the misfit with
    PathSpectra's FP32 k grid; the loss and the gradient with respect to all 3 x 800 positions against the reference's
    (FP64 form: 1e-7 relative to the largest component, the rounding of PathSpectra's FP32 window cosines, measured
    2e-9; mixed form: 1e-4, the gradient bar of the mixed form), and per-path
    sigma^2 gradients (no reference counterpart) against central differences.  The FP32-vs-FP64 gradient error is
    printed."""
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200.model import PathModel, finder_groups
    from feffgpu_b200.pathfinder import GPUPathFinder
    from feffgpu_b200.rspace import FitWindow, RSpaceMisfit
    from tests.fixtures import cfg2_phase
    z = npz("cfg3_adjoint")
    P = cfg2_phase()
    pos, box, absorbers, ipot = z["pos"], float(z["box"]), z["absorbers"], z["ipot"]
    # PathSpectra's finder keeps single-scattering paths unmerged (its merge_degenerate=False, forward.py:68-75)
    finder = GPUPathFinder(P, device="cuda", rmax=5.0, nlegmax=4, critpw=0.5, merge_degenerate=False)
    gs = finder_groups(finder, pos, box, absorbers, ipot)
    assert {int(np.asarray(g[0]).shape[1]): len(g[0]) for g in gs} == dict(zip(z["legs"].tolist(), z["counts"].tolist()))
    q = torch.tensor(K401, device="cuda")
    win = FitWindow(kmin=3.0, kmax=16.0, dk=1.0, kweight=2, rmin=1.0, rmax=6.0)
    grads = {}
    for dtype, tol in ((torch.complex128, 1e-7), (torch.complex64, 1e-4)):
        st = GPUPathStage(P, device="cuda", dtype=dtype)
        model = PathModel(st, gs, pos, nrows=1, box=box)
        S = st.linear_matrix(K401).double()
        mis = RSpaceMisfit(len(K401), z["target"], win, k_dtype=np.float32)
        x = torch.tensor(pos, device="cuda", requires_grad=True)
        s2 = torch.zeros(model.batch.n, dtype=torch.float64, device="cuda", requires_grad=True)
        loss = mis(model.rows(x, q, S, sigma2=s2))[0]
        loss.backward()
        gx = x.grad.cpu().numpy()
        err_l = abs(float(loss.detach()) - float(z["loss"])) / float(z["loss"])
        err_g = np.abs(gx - z["grad"]).max() / np.abs(z["grad"]).max()
        print(f"cfg3 {dtype}: loss {float(loss.detach()):.6e} (reference {float(z['loss']):.6e}, rel {err_l:.1e}), "
              f"gradient vs reference autograd {err_g:.2e}")
        assert err_l <= tol and err_g <= tol
        grads[dtype] = (gx, s2.grad.cpu().numpy())
        if dtype != torch.complex128:
            continue
        # per-path sigma^2 (new, no reference counterpart): central differences on the largest components
        gsig = grads[dtype][1]
        with torch.no_grad():
            for p in np.argsort(-np.abs(gsig))[:4]:
                sp, sm = s2.detach().clone(), s2.detach().clone()
                sp[p] += 1e-6
                sm[p] -= 1e-6
                fd = (float(mis(model.rows(x.detach(), q, S, sigma2=sp))[0]) -
                      float(mis(model.rows(x.detach(), q, S, sigma2=sm))[0])) / 2e-6
                assert abs(gsig[p] - fd) <= 1e-4 * abs(gsig).max(), (p, gsig[p], fd)
    g64, g32 = grads[torch.complex128], grads[torch.complex64]
    e_x = np.abs(g32[0] - g64[0]).max() / np.abs(g64[0]).max()
    e_s = np.abs(g32[1] - g64[1]).max() / np.abs(g64[1]).max()
    print(f"cfg3: FP32 vs FP64 gradient error: positions {e_x:.2e}, sigma2 {e_s:.2e}")
    assert e_x < 1e-4 and e_s < 1e-4


def test_cfg4_md_frames_times_absorbers():
    """Configuration 4 at its per-frame size: frames of the thermally displaced bcc Fe 16^3 supercell (8192 atoms,
    sigma 0.08 A) x 32 absorbers each, every path of up to 3 legs within 5.5 A from the CUDA path finder (all frames
    and absorbers in one call, as the benchmark's MD leg), all paths in one fused launch with chi averaged per frame;
    each frame's row against the oracle's FP64 sum of the same paths (R <= 1e-6 mixed, 1e-12 FP64).  Four frames
    (about 33,000 paths) keep the oracle's share of the test to seconds."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.pathfinder import GPUPathFinder
    P = phase("cfg4_fe_phase")
    frames, A = 4, 32
    base, box = W.bcc_supercell(16, 2.87)
    rng = np.random.default_rng(12)
    pos = np.stack([W.thermal(base, 0.08, seed=100 + f) for f in range(frames)]).astype(np.float32)
    abs_ = np.stack([rng.choice(len(base), size=A, replace=False) for _ in range(frames)])
    res = GPUPathFinder(P, device="cuda", rmax=5.5, nlegmax=3, critpw=0.0).enumerate_many(
        pos, box, abs_, np.ones(len(base), int))
    groups = []
    for nleg, (coords, ipots, deg, _xp, _atoms, slot) in sorted(res["paths"].items()):
        groups.append((coords.double().cpu().numpy(), ipots.cpu().numpy(), deg.double().cpu().numpy() / A,
                       torch.div(slot, A, rounding_mode="floor").cpu().numpy()))
    assert sum(len(g[0]) for g in groups) > 25000
    orc = O.Oracle(P)
    So = orc.linear_matrix(K401)
    ref = np.zeros((frames, len(K401)))
    for coords, ipots, deg, row in groups:
        cc, rf = orc.cchi(coords, ipots)
        np.add.at(ref, row, deg[:, None] * O.chi_fine(cc, rf, K401, So))
    batch = PathBatch(groups, nrows=frames, device="cuda")
    for dtype, tol in ((torch.complex64, 1e-6), (torch.complex128, 1e-12)):
        rows = GPUPathStage(P, device="cuda", dtype=dtype).chi_reduce(batch, K401).cpu().numpy()
        for f in range(frames):
            R = _R(K401, ref[f], rows[f])
            print(f"cfg4 {dtype} frame {f}: R {R:.2e}")
            assert R <= tol


def test_cfg5_two_edge_refinement_graph():
    """Configuration 5 at its stated size: rock-salt NiO 8^3 cells (4096 sites, 5 % vacancies, 0.1 A disorder), Ni K
    and O K edges, 32 absorbers each with the CUDA finder's paths (rmax 5 A, 4 legs, importance cut 2 %, unmerged
    single scattering: the reference GpuRmc's defaults); the refinement step captured as one CUDA graph equals the
    same steps run eagerly (losses and positions to 1e-9) and the misfit falls over 15 steps."""
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200.model import GraphedRefinement, PathModel, finder_groups
    from feffgpu_b200.pathfinder import GPUPathFinder
    from feffgpu_b200.rspace import FitWindow, RSpaceMisfit
    pos0, lab, box = W.rock_salt_supercell(8, 4.177)
    rng = np.random.default_rng(5)
    keep = rng.random(len(pos0)) >= 0.05
    pos0, lab = pos0[keep], lab[keep]
    pos = W.thermal(pos0, 0.1, seed=6)
    hidden = W.thermal(pos, 0.03, seed=7)
    q = torch.tensor(K401, device="cuda")
    ipot_of = np.array([{"Ni": 1, "O": 2}[x] for x in lab])
    models, npaths = [], 0
    for edge, fname in (("Ni", "cfg5_nik_phase"), ("O", "cfg5_ok_phase")):
        P = phase(fname)
        st = GPUPathStage(P, device="cuda", dtype=torch.complex64)
        finder = GPUPathFinder(P, device="cuda", rmax=5.0, nlegmax=4, critpw=2.0, merge_degenerate=False)
        gs = finder_groups(finder, pos, box, W.central_atom(pos, box, lab, edge, 32), ipot_of)
        model = PathModel(st, gs, pos, nrows=1, box=box)
        npaths += model.batch.n
        S = st.linear_matrix(K401).double().contiguous()
        with torch.no_grad():
            target = model.rows(torch.tensor(hidden, device="cuda"), q, S)[0]
        models.append((model, q, S, RSpaceMisfit(len(K401), target, FitWindow(kmin=3.0, kmax=14.0, rmin=1.0, rmax=5.0))))
    assert len(pos) > 3800 and npaths > 5000
    g = GraphedRefinement(models, pos, lr=0.002)
    eager_pos = torch.tensor(pos, device="cuda", requires_grad=True)        # the same steps without the graph
    opt = torch.optim.Adam([eager_pos], lr=0.002, capturable=True)
    losses = []
    for it in range(15):
        g.step()
        opt.zero_grad()
        loss = sum(mis(m.rows(eager_pos, qq, SS).mean(0, keepdim=True))[0] for m, qq, SS, mis in models)
        loss.backward()
        opt.step()
        torch.cuda.synchronize()
        losses.append(float(g.loss))
        assert abs(float(g.loss) - float(loss)) <= 1e-9 * abs(float(loss)), (it, float(g.loss), float(loss))
    assert torch.allclose(g.pos.detach(), eager_pos.detach(), rtol=0, atol=1e-9)
    print(f"cfg5: {npaths} paths, misfit {losses[0]:.4e} -> {losses[-1]:.4e}")
    assert losses[-1] < 0.8 * losses[0]


@pytest.mark.parametrize("dtype,tol", [(torch.complex64, 1e-6), (torch.complex128, 1e-12)])
def test_cfg1_end_to_end_from_the_path_finder(dtype, tol):
    """The whole configuration on the device: the path finder on the Cu cluster (rmax 6 A, 4 legs, importance cut
    2.5 %) gives the reference chain's path list (coordinates and degeneracies), the fused stage its chi."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.pathfinder import GPUPathFinder
    z = npz("cfg1_cu")
    P = phase("cfg1_cu")
    pts = W.fcc_cluster(3.61, 6.0)
    kept, _ = GPUPathFinder(P, device="cuda", rmax=6.0, nlegmax=4, critpw=2.5).enumerate(
        pts, None, 0, np.ones(len(pts), int))
    gs = []
    for nleg, (c, ip, deg, _xp, _atoms) in sorted(kept.items()):
        c, ip, deg = c.cpu().numpy(), ip.cpu().numpy(), deg.cpu().numpy()
        assert np.array_equal(c.astype(np.float64), z[f"coords_{nleg}"]), nleg
        assert np.array_equal(ip, z[f"ipots_{nleg}"]) and np.array_equal(deg.astype(np.float64), z[f"deg_{nleg}"])
        gs.append((c.astype(np.float64), ip, deg.astype(np.float64)))
    st = GPUPathStage(P, device="cuda", dtype=dtype)
    rows = st.chi_reduce(PathBatch(gs, device="cuda"), K401)[0].cpu().numpy()
    R = _R(K401, z["ref_chi"], rows)
    print(f"cfg1 from the path finder {dtype}: R {R:.2e}")
    assert R <= tol


def test_path_model_and_graph_in_a_triclinic_cell():
    """PathModel and GraphedRefinement with a triclinic cell (the bcc Fe frame of tests/golden/finder_tri.npz): the
    paths of four absorbers from the CUDA finder (the cell's minimum image, FP32), held as atom indices and rebuilt by
    the model's FP64 minimum image of the cell, give the finder's coordinates to 1e-5 A and the same rows to 1e-6;
    two graph-replayed refinement steps equal the same steps run eagerly."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.model import GraphedRefinement, PathModel
    from feffgpu_b200.pathfinder import GPUPathFinder
    from feffgpu_b200.rspace import FitWindow, RSpaceMisfit
    z = npz("finder_tri")
    pos, cell = z["pos"], z["cell"]
    P = phase("cfg4_fe_phase")
    f = GPUPathFinder(P, device="cuda", rmax=5.0, nlegmax=4, critpw=2.0)
    res = f.enumerate_many(pos, cell, np.array([0, 57, 190, 301]), np.ones(len(pos), int))
    absorbers = np.array([0, 57, 190, 301])
    st = GPUPathStage(P, device="cuda", dtype=torch.complex64)
    gs, cg = [], []
    for nleg, (coords, ipots, deg, _xp, atoms, slot) in sorted(res["paths"].items()):
        ab = torch.as_tensor(absorbers, device="cuda")[slot.long()][:, None]
        gs.append((torch.cat([ab, atoms], 1).cpu().numpy(), ipots.cpu().numpy(), deg.cpu().numpy(),
                   np.zeros(len(deg), int)))
        cg.append((coords.double(), ipots, deg.double(), None))
    model = PathModel(st, gs, pos, nrows=1, box=cell)
    x = torch.tensor(pos, device="cuda")
    mc = model.coords(x)
    fc = PathBatch(cg, nrows=1, device="cuda").coords
    assert torch.abs(mc - fc).max() < 1e-5
    q = torch.tensor(K401, device="cuda")
    S = st.linear_matrix(K401).double().contiguous()
    with torch.no_grad():
        rows = model.rows(x, q, S)
        ref = st.chi_reduce(PathBatch(cg, nrows=1, device="cuda"), q, S)
    assert torch.abs(rows - ref).max() <= 1e-6 * torch.abs(ref).max()
    target = (model.rows(torch.tensor(pos + 0.02, device="cuda"), q, S)[0]).detach()
    mis = RSpaceMisfit(len(K401), target, FitWindow(kmin=3.0, kmax=14.0, rmin=1.0, rmax=5.0))
    g = GraphedRefinement([(model, q, S, mis)], pos, lr=0.002)
    eager = torch.tensor(pos, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([eager], lr=0.002, capturable=True)
    for _ in range(2):
        g.step()
        opt.zero_grad()
        loss = mis(model.rows(eager, q, S).mean(0, keepdim=True))[0]
        loss.backward()
        opt.step()
        torch.cuda.synchronize()
        assert abs(float(g.loss) - float(loss)) <= 1e-9 * abs(float(loss))
    assert torch.allclose(g.pos.detach(), eager.detach(), rtol=0, atol=1e-9)


def test_refinement_refreshes_the_path_lists_and_recaptures():
    """GraphedRefinement with refresh_every: every third step the CUDA finder lists the paths again at the current
    positions (the reference's refinement loop does this every refresh_every steps, src/feffgpu/rmc/refine.py:176-179)
    and the step is captured again.  The graph-replayed run equals an eager run with the same refreshes (losses and
    positions to 1e-9), the optimiser state carries over the refreshes, and the model after a refresh holds the
    finder's paths at those positions."""
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200.model import GraphedRefinement, PathModel, finder_groups
    from feffgpu_b200.pathfinder import GPUPathFinder
    from feffgpu_b200.rspace import FitWindow, RSpaceMisfit
    pos0, lab, box = W.rock_salt_supercell(3, 4.177)
    pos = W.thermal(pos0, 0.1, seed=6)
    hidden = W.thermal(pos, 0.05, seed=7)
    P = phase("cfg5_nik_phase")
    st = GPUPathStage(P, device="cuda", dtype=torch.complex64)
    ipot_of = np.array([{"Ni": 1, "O": 2}[x] for x in lab])
    absorbers = W.central_atom(pos, box, lab, "Ni", 4)
    finder = GPUPathFinder(P, device="cuda", rmax=4.5, nlegmax=4, critpw=0.5)
    q = torch.tensor(K401, device="cuda")
    S = st.linear_matrix(K401).double().contiguous()

    def build(x):
        return PathModel(st, finder_groups(finder, np.asarray(x), box, absorbers, ipot_of), np.asarray(x), nrows=1,
                         box=box)

    m0 = build(pos)
    with torch.no_grad():
        target = m0.rows(torch.tensor(hidden, device="cuda"), q, S)[0]
    mis = RSpaceMisfit(len(K401), target, FitWindow(kmin=3.0, kmax=14.0, rmin=1.0, rmax=4.5))

    def rebuild(x, models):
        return [(build(x.cpu().numpy()), q, S, mis)]

    g = GraphedRefinement([(m0, q, S, mis)], pos, lr=0.01, rebuild=rebuild, refresh_every=3)
    eager = torch.tensor(pos, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([eager], lr=0.01, capturable=True)
    model = m0
    for it in range(8):
        if it and it % 3 == 0:
            model = build(eager.detach().cpu().numpy())
        g.step()
        opt.zero_grad()
        loss = mis(model.rows(eager, q, S).mean(0, keepdim=True))[0]
        loss.backward()
        opt.step()
        torch.cuda.synchronize()
        assert abs(float(g.loss) - float(loss)) <= 1e-9 * abs(float(loss)), (it, float(g.loss), float(loss))
    assert torch.allclose(g.pos.detach(), eager.detach(), rtol=0, atol=1e-9)
    assert [s for s, _ in g.refreshes] == [3, 6]
    assert g.models[0][0].batch.n == model.batch.n
    assert torch.equal(g.models[0][0].atoms, model.atoms)
    print(f"refresh: {[round(ms, 1) for _, ms in g.refreshes]} ms to find and re-capture")
