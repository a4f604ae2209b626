"""GPU parity of the hand-written adjoint: d(loss)/d(coords) and d(loss)/d(sigma^2).

Oracles: the reference stage's gradient under torch.utils.checkpoint(use_reentrant=False) (golden fixtures,
tests/golden/grad_*.npz) and central finite differences (h = 1e-4 A) of the oracle / of the stage itself.
Tolerances (relative to the largest gradient component): FP64 form 1e-7 against the reference's autograd (its own
agreement with finite differences is ~1e-6), mixed form 1e-4 (the gradient bar of the mixed form); finite differences 1e-4.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.fixtures import npz, phase

pytestmark = pytest.mark.gpu

TOL = {torch.complex128: 1e-7, torch.complex64: 1e-4}
DTYPES = [torch.complex128, torch.complex64]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


GRAD_CASES = ["grad_L001", "grad_A000", "grad_A014", "grad_A009"]     # K, K, L3, M5 edges


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", GRAD_CASES)
def test_cchi_chi_fine_gradient_equals_reference_autograd(name, dtype):
    """The reference callers' pattern: cchi -> chi_fine -> weighted sum, backward through both custom adjoints."""
    from feffgpu_b200 import GPUPathStage
    z = npz(name)
    st = GPUPathStage(phase(name), device="cuda", dtype=dtype)
    q = z["q"]
    S = st.linear_matrix(q)
    w = torch.tensor(z["w"], device="cuda")
    for nleg in sorted(int(k.split("_")[1]) for k in z if k.startswith("coords_")):
        x = torch.tensor(z[f"coords_{nleg}"], device="cuda", dtype=st.rdtype, requires_grad=True)
        cc, rf = st.cchi(x, torch.tensor(z[f"ipots_{nleg}"]))
        chi = st.chi_fine(cc, rf, q, S)
        loss = (torch.tensor(z[f"deg_{nleg}"], device="cuda")[:, None] * chi.double() * w[None]).sum()
        loss.backward()
        e = _rel(x.grad.double().cpu().numpy(), z[f"grad_{nleg}"])
        print(f"{name} nleg {nleg} {dtype}: gradient vs reference autograd {e:.2e}")
        assert e < TOL[dtype], (nleg, e)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", GRAD_CASES)
def test_fused_gradient_equals_reference_autograd(name, dtype):
    """The same loss through the fused stage (one persistent launch over every leg count, its adjoint): rows =
    sum_p deg_p chi_p, loss = sum_q w_q rows_q."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    z = npz(name)
    st = GPUPathStage(phase(name), device="cuda", dtype=dtype)
    legs = sorted(int(k.split("_")[1]) for k in z if k.startswith("coords_"))
    b = PathBatch([(z[f"coords_{n}"], z[f"ipots_{n}"], z[f"deg_{n}"]) for n in legs], nrows=1, device="cuda")
    x = b.coords.clone().requires_grad_(True)
    rows = st.chi_reduce(b, z["q"], coords=x)
    (rows[0] * torch.tensor(z["w"], device="cuda")).sum().backward()
    g = x.grad.cpu().numpy()
    s = 0
    for n in legs:
        m = len(z[f"coords_{n}"])
        e = _rel(g[s:s + m, :n], z[f"grad_{n}"])
        print(f"{name} fused nleg {n} {dtype}: gradient vs reference autograd {e:.2e}")
        assert e < TOL[dtype], (n, e)
        assert np.all(g[s:s + m, n:] == 0)
        s += m


@pytest.mark.parametrize("dtype", DTYPES)
def test_checkpointed_call_as_the_reference_callers_make_it(dtype):
    """torch.utils.checkpoint(use_reentrant=False) around cchi + chi_fine (exafs/forward.py:158-159) works."""
    from torch.utils.checkpoint import checkpoint
    from feffgpu_b200 import GPUPathStage
    z = npz("grad_L001")
    st = GPUPathStage(phase("grad_L001"), device="cuda", dtype=dtype)
    q = z["q"]
    S = st.linear_matrix(q)
    x = torch.tensor(z["coords_3"], device="cuda", dtype=st.rdtype, requires_grad=True)
    ip = torch.tensor(z["ipots_3"])

    def f(c):
        cc, rf = st.cchi(c, ip)
        return st.chi_fine(cc, rf, q, S)

    chi = checkpoint(f, x, use_reentrant=False)
    (torch.tensor(z["deg_3"], device="cuda")[:, None] * chi.double() * torch.tensor(z["w"], device="cuda")).sum().backward()
    assert _rel(x.grad.double().cpu().numpy(), z["grad_3"]) < TOL[dtype]


def _distinct_atoms(coords):
    """True if no two atoms of the path coincide (a path that revisits an atom scatters straight back, where the
    Euler angles are not differentiable and only the reference's branch choice defines a gradient)."""
    c = np.asarray(coords)
    d = np.linalg.norm(c[:, None] - c[None], axis=-1) + np.eye(len(c))
    return bool(d.min() > 1e-3)


@pytest.mark.parametrize("dtype", DTYPES)
def test_walk_gradients_equal_reference_autograd(dtype):
    """2-8-leg lattice walks (W phases, l up to 47), including paths that revisit an atom, against the reference's
    checkpointed autograd.  A revisit (A -> B -> A) puts B's scattering angle exactly at pi, where the Euler angles
    are not differentiable: the gradient there is the reference's branch choice, reproduced up to the rounding that
    decides the branch tests (1e-4 relative for such paths)."""
    from feffgpu_b200 import GPUPathStage
    z, zg = npz("walks_W"), npz("grad_walks_W")
    st = GPUPathStage(phase("case_W"), device="cuda", dtype=dtype)
    q = zg["q"]
    S = st.linear_matrix(q)
    w = torch.tensor(zg["w"], device="cuda")
    for nleg in range(2, 9):
        x = torch.tensor(z[f"coords_{nleg}"], device="cuda", dtype=st.rdtype, requires_grad=True)
        cc, rf = st.cchi(x, torch.tensor(z[f"ipots_{nleg}"]))
        (st.chi_fine(cc, rf, q, S).double() * w[None]).sum().backward()
        g = x.grad.double().cpu().numpy()
        for b in range(len(g)):
            e = _rel(g[b], zg[f"grad_{nleg}"][b])
            smooth = _distinct_atoms(z[f"coords_{nleg}"][b])
            print(f"walk nleg {nleg} path {b} {dtype} {'distinct' if smooth else 'revisit'}: vs reference autograd {e:.2e}")
            assert e < (TOL[dtype] if smooth else max(TOL[dtype], 1e-4)), (nleg, b, e)


def test_finite_differences_of_the_stage_two_to_eight_legs():
    """Central differences of the FP64 stage's own loss (h = 1e-4 A) on the 2-8-leg walks whose atoms are distinct."""
    from feffgpu_b200 import GPUPathStage
    z = npz("walks_W")
    st = GPUPathStage(phase("case_W"), device="cuda", dtype=torch.complex128)
    q = np.arange(1, 401) * 0.05
    S = st.linear_matrix(q)
    rng = np.random.default_rng(2)
    w = torch.tensor(rng.normal(size=len(q)) * q ** 2, device="cuda")
    checked = 0
    for nleg in range(2, 9):
        for b in range(len(z[f"coords_{nleg}"])):
            if not _distinct_atoms(z[f"coords_{nleg}"][b]):
                continue
            c0 = torch.tensor(z[f"coords_{nleg}"][b:b + 1], device="cuda")
            ip = torch.tensor(z[f"ipots_{nleg}"][b:b + 1])

            def loss(c):
                cc, rf = st.cchi(c, ip)
                return (st.chi_fine(cc, rf, q, S) * w[None]).sum()

            x = c0.clone().requires_grad_(True)
            loss(x).backward()
            g = x.grad.cpu().numpy()[0]
            fd = np.zeros_like(g)
            h = 1e-4
            with torch.no_grad():
                for i in range(nleg):
                    for k in range(3):
                        cp, cm = c0.clone(), c0.clone()
                        cp[0, i, k] += h
                        cm[0, i, k] -= h
                        fd[i, k] = (float(loss(cp)) - float(loss(cm))) / (2 * h)
            e = _rel(g, fd)
            print(f"walk nleg {nleg} path {b}: adjoint vs central differences {e:.2e}")
            assert e < 1e-4, (nleg, b, e)
            checked += 1
    assert checked >= 7


def test_reff_output_gradient():
    """d(sum reff)/d(coords): reff is half the closed path length, so each atom gets half the sum of the unit vectors
    from its two neighbours."""
    from feffgpu_b200 import GPUPathStage
    st = GPUPathStage(phase("case_L001"), device="cuda", dtype=torch.complex128)
    rng = np.random.default_rng(4)
    c0 = torch.tensor(np.concatenate([np.zeros((2, 1, 3)), rng.normal(0, 1.5, (2, 4, 3))], 1), device="cuda")
    ip = torch.ones(2, 5, dtype=torch.long)
    ip[:, 0] = 0
    x = c0.clone().requires_grad_(True)
    _, rf = st.cchi(x, ip)
    rf.sum().backward()
    c = c0.cpu().numpy()
    fd = np.zeros_like(c)
    # analytic: reff = sum of leg lengths / 2; each atom's gradient = (unit vector to previous + to next) / 2
    for b in range(2):
        ring = list(range(5))
        for j in ring:
            prv, nxt = c[b, ring[j - 1]], c[b, ring[(j + 1) % 5]]
            u1 = (c[b, j] - prv) / np.linalg.norm(c[b, j] - prv)
            u2 = (c[b, j] - nxt) / np.linalg.norm(c[b, j] - nxt)
            fd[b, j] = 0.5 * (u1 + u2)
    assert _rel(x.grad.cpu().numpy(), fd) < 1e-12


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_gradient_coords_and_sigma2(dtype):
    """chi_reduce's adjoint: coordinates against the reference's autograd, sigma^2 against the analytic factor."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    z = npz("grad_L001")
    st = GPUPathStage(phase("grad_L001"), device="cuda", dtype=dtype)
    q = z["q"]
    nlegs = sorted(int(k.split("_")[1]) for k in z if k.startswith("coords_"))
    b = PathBatch([(z[f"coords_{n}"], z[f"ipots_{n}"], z[f"deg_{n}"]) for n in nlegs], device="cuda")
    x = b.coords.clone().requires_grad_(True)
    s2 = torch.zeros(b.n, dtype=torch.float64, device="cuda", requires_grad=True)
    rows = st.chi_reduce(b, q, coords=x, sigma2=s2)
    w = torch.tensor(z["w"], device="cuda")
    (rows[0] * w).sum().backward()
    g = x.grad.cpu().numpy()
    off = 0
    for n in nlegs:
        m = len(z[f"coords_{n}"])
        e = _rel(g[off:off + m, :n], z[f"grad_{n}"])
        print(f"fused nleg {n} {dtype}: gradient vs reference autograd {e:.2e}")
        assert e < TOL[dtype], (n, e)
        assert np.all(g[off:off + m, n:] == 0)
        off += m
    # sigma^2: d/dsigma2_p of sum_q w_q deg_p chi_p(q) exp(-2 sigma2 q^2) at sigma2 = 0 is -2 sum_q q^2 w_q deg_p chi_p
    orc = O.Oracle(phase("grad_L001"))
    S = orc.linear_matrix(q)
    ref = []
    for n in nlegs:
        cc, rf = orc.cchi(z[f"coords_{n}"], z[f"ipots_{n}"])
        chi = O.chi_fine(cc, rf, q, S)
        ref.append((-2 * q ** 2 * z["w"] * z[f"deg_{n}"][:, None] * chi).sum(1))
    e = _rel(s2.grad.cpu().numpy(), np.concatenate(ref))
    print(f"fused sigma2 {dtype}: {e:.2e}")
    assert e < TOL[dtype]


def test_fused_gradient_mixed_leg_counts_and_rows_by_finite_differences():
    """Random paths of 2-8 legs (distinct atoms) over several rows with non-zero sigma^2: adjoint of the FP64 fused
    stage against central differences of the oracle's FP64 sums."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    from tests.fixtures import cfg2_phase
    z = npz("cfg2_sample")
    P = cfg2_phase()
    st = GPUPathStage(P, device="cuda", dtype=torch.complex128)
    rng = np.random.default_rng(9)
    groups = []
    for n in range(2, 9):
        ok = [i for i in range(len(z[f"coords_{n}"])) if _distinct_atoms(z[f"coords_{n}"][i])]
        if ok:
            i = ok[0]
            groups.append((z[f"coords_{n}"][i:i + 1], z[f"ipots_{n}"][i:i + 1], np.array([1.0 + n]), np.array([n % 3])))
    assert len(groups) >= 5
    b = PathBatch(groups, nrows=3, device="cuda")
    q = np.arange(1, 401) * 0.05
    s2 = rng.uniform(0.001, 0.01, b.n)
    W = rng.normal(size=(3, len(q)))
    x = b.coords.clone().requires_grad_(True)
    st_s2 = torch.tensor(s2, device="cuda", requires_grad=True)
    rows = st.chi_reduce(b, q, coords=x, sigma2=st_s2)
    (rows * torch.tensor(W, device="cuda")).sum().backward()
    orc = O.Oracle(P)
    S = orc.linear_matrix(q)
    nl = b.nleg.cpu().numpy()
    deg, row = b.deg.cpu().numpy(), b.row.cpu().numpy()

    def loss(coords, sig):
        chi = np.zeros((b.n, len(q)))
        for i in range(b.n):
            n = nl[i]
            cc, rf = orc.cchi(coords[i:i + 1, :n], b.ipots.cpu().numpy()[i:i + 1, :n], nthreads=1)
            chi[i] = O.chi_fine(cc, rf, q, S)[0]
        return float((O.chi_rows(chi, deg, row, 3, q, sig) * W).sum())

    c0 = b.coords.cpu().numpy()
    g = x.grad.cpu().numpy()
    h = 1e-4
    fd = np.zeros_like(c0)
    for i in range(b.n):
        for j in range(nl[i]):
            for k in range(3):
                cp, cm = c0.copy(), c0.copy()
                cp[i, j, k] += h
                cm[i, j, k] -= h
                fd[i, j, k] = (loss(cp, s2) - loss(cm, s2)) / (2 * h)
    e = _rel(g, fd)
    print(f"fused mixed legs: adjoint vs central differences {e:.2e}")
    assert e < 1e-4
    fds = np.zeros(b.n)
    for i in range(b.n):
        sp, sm = s2.copy(), s2.copy()
        sp[i] += 1e-5
        sm[i] -= 1e-5
        fds[i] = (loss(c0, sp) - loss(c0, sm)) / 2e-5
    assert _rel(st_s2.grad.cpu().numpy(), fds) < 1e-5


def test_nine_legs_forward_and_gradient():
    """Paths of nine legs (eight scatterers, FEFF's own limit): the stage against the oracle (FP64 to 1e-10, mixed to
    2e-5 of max|cchi|) and the FP64 adjoint against central differences of the stage (h = 1e-4 A), with distinct
    atoms (W phases, bcc walks of the Fe/O/Pt packing's kind drawn by workloads.random_paths)."""
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200 import workloads as W
    P = phase("case_W")
    base, box = W.bcc_supercell(6, 3.1652)
    pos = W.thermal(base, 0.05, seed=9)
    ab = int(W.central_atom(pos, box, None, None, 1)[0])
    paths = W.random_paths(pos, box, ab, {9: 80}, rmax=13.5, leg_max=4.0, seed=4)
    coords, ip, atoms = paths[9]
    keep = [b for b in range(len(atoms)) if len(set(atoms[b].tolist()) | {ab}) == 9][:4]
    coords, ip = coords[keep], ip[keep]
    assert len(coords) >= 2
    orc = O.Oracle(P)
    oc, _ = orc.cchi(coords, ip)
    for dtype, tol in ((torch.complex128, 1e-10), (torch.complex64, 2e-5)):
        st = GPUPathStage(P, device="cuda", dtype=dtype)
        cc, _ = st.cchi(torch.tensor(coords), torch.tensor(ip))
        e = _rel(cc.cpu().numpy(), oc)
        print(f"nine legs {dtype}: cchi vs oracle {e:.2e}")
        assert e < tol
    st = GPUPathStage(P, device="cuda", dtype=torch.complex128)
    q = np.arange(1, 401) * 0.05
    S = st.linear_matrix(q)
    w = torch.tensor(np.random.default_rng(8).normal(size=len(q)) * q ** 2, device="cuda")

    def loss(c):
        cc, rf = st.cchi(c, torch.tensor(ip))
        return (st.chi_fine(cc, rf, q, S) * w[None]).sum()

    x = torch.tensor(coords, device="cuda", requires_grad=True)
    loss(x).backward()
    g = x.grad.cpu().numpy()
    h = 1e-4
    with torch.no_grad():
        for b, j, k in [(0, 3, 0), (0, 8, 2), (1, 5, 1), (1, 1, 2)]:
            cp, cm = coords.copy(), coords.copy()
            cp[b, j, k] += h
            cm[b, j, k] -= h
            fd = (float(loss(torch.tensor(cp, device="cuda"))) - float(loss(torch.tensor(cm, device="cuda")))) / (2 * h)
            assert abs(fd - g[b, j, k]) <= 1e-4 * np.abs(g).max(), (b, j, k, fd, g[b, j, k])


AXIAL_PATHS = {   # angstrom, absorber first; legs lying on (or within 0.06 degrees of) the z axis, no collinear atoms
    "first leg on z": [[0, 0, 0], [0, 0, 2.3], [1.7, 0.9, 2.6]],
    "last leg on z": [[0, 0, 0], [1.7, 0.9, 2.6], [0, 0, 2.3]],
    "middle leg on z": [[0, 0, 0], [1.1, 0.4, 1.9], [1.1, 0.4, 4.2]],
    "two legs on z": [[0, 0, 0], [0, 0, 2.4], [1.9, 0.3, 2.4], [1.9, 0.3, -0.3]],
    "near-axial first leg": [[0, 0, 0], [0.002, 0.0015, 2.3], [1.7, 0.9, 2.6]],
    "axial lattice walk": [[0, 0, 0], [0, 0, 2.55], [2.55, 0, 2.55], [2.55, 0, 0], [0, 2.55, 0]],
}


@pytest.mark.parametrize("dtype", DTYPES)
def test_axial_legs_gradient_matches_finite_differences(dtype):
    """A leg along z leaves FEFF's Euler angles undefined (the reference's autograd gives NaN there; its constant
    branches give no derivative).  The signal is invariant under a rotation of the whole path, and the adjoint
    differentiates such paths in a rotated frame: the gradient must equal central differences (h = 1e-5 A) of the
    FP64 stage's own loss, through cchi -> chi_fine and through the fused stage."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    z = npz("grad_L001")
    P = phase("grad_L001")
    q = z["q"]
    ref = GPUPathStage(P, device="cuda", dtype=torch.complex128)
    st = GPUPathStage(P, device="cuda", dtype=dtype)
    S64, S = ref.linear_matrix(q), st.linear_matrix(q)
    w = torch.tensor(z["w"], device="cuda")
    h = 1e-5
    tol = 1e-6 if dtype == torch.complex128 else 1e-4
    for name, c in AXIAL_PATHS.items():
        c = np.asarray(c, float)
        ip = torch.tensor(np.r_[0, [1] * (len(c) - 1)][None])

        def loss64(cc):
            with torch.no_grad():
                a, rf = ref.cchi(torch.tensor(cc[None], device="cuda"), ip)
                return float((ref.chi_fine(a, rf, q, S64) * w[None]).sum())

        fd = np.zeros_like(c)
        for i in range(len(c)):
            for k in range(3):
                cp, cm = c.copy(), c.copy()
                cp[i, k] += h
                cm[i, k] -= h
                fd[i, k] = (loss64(cp) - loss64(cm)) / (2 * h)
        x = torch.tensor(c[None], device="cuda", dtype=st.rdtype, requires_grad=True)
        a, rf = st.cchi(x, ip)
        (st.chi_fine(a, rf, q, S) * w[None]).sum().backward()
        e = _rel(x.grad[0].double().cpu().numpy(), fd)
        b = PathBatch([(c[None], ip.numpy(), np.ones(1))], nrows=1, device="cuda")
        xf = b.coords.clone().requires_grad_(True)
        (st.chi_reduce(b, q, coords=xf)[0] * w).sum().backward()
        ef = _rel(xf.grad[0, :len(c)].cpu().numpy(), fd)
        print(f"{name} {dtype}: gradient vs finite differences {e:.2e} (fused {ef:.2e})")
        assert np.isfinite(e) and e < tol, (name, e)
        assert np.isfinite(ef) and ef < tol, (name, ef)


IORDER_CASES = ["grad_L001_io0", "grad_L001_io1", "grad_A014_io0", "grad_A014_io1",    # K and L3 edges
                "grad_L001_io3", "grad_A014_io3", "grad_A009_io3"]                      # order 3: K, L3, M5


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", IORDER_CASES)
def test_lower_lambda_orders_equal_reference(name, dtype):
    """GPUPathStage(..., iorder=0, 1 or 3), the reference's other multiple-scattering lambda sets (setlam,
    genfmt.py:115-153; 1, 3 and 10 entries): per-path cchi against the reference stage at the same order, and the
    gradient of the weighted fine-grid sum, per-path and fused, against its checkpointed autograd."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    z = npz(name)
    io = int(z["iorder"])
    st = GPUPathStage(phase(name), device="cuda", dtype=dtype, iorder=io)
    q = z["q"]
    S = st.linear_matrix(q)
    w = torch.tensor(z["w"], device="cuda")
    legs = sorted(int(k.split("_")[1]) for k in z if k.startswith("coords_"))
    tol_c = {torch.complex128: 1e-10, torch.complex64: 2e-5}[dtype]
    for n in legs:
        x = torch.tensor(z[f"coords_{n}"], device="cuda", dtype=st.rdtype, requires_grad=True)
        cc, rf = st.cchi(x, torch.tensor(z[f"ipots_{n}"]))
        ec = _rel(cc.detach().cpu().numpy(), z[f"cchi_{n}"])
        chi = st.chi_fine(cc, rf, q, S)
        (torch.tensor(z[f"deg_{n}"], device="cuda")[:, None] * chi.double() * w[None]).sum().backward()
        eg = _rel(x.grad.double().cpu().numpy(), z[f"grad_{n}"])
        print(f"{name} nleg {n} {dtype}: cchi {ec:.2e}, gradient {eg:.2e}")
        assert ec < tol_c and eg < TOL[dtype], (n, ec, eg)
    b = PathBatch([(z[f"coords_{n}"], z[f"ipots_{n}"], z[f"deg_{n}"]) for n in legs], nrows=1, device="cuda")
    x = b.coords.clone().requires_grad_(True)
    rows = st.chi_reduce(b, q, coords=x)
    (rows[0] * w).sum().backward()
    g = x.grad.cpu().numpy()
    s = 0
    for n in legs:
        m = len(z[f"coords_{n}"])
        assert _rel(g[s:s + m, :n], z[f"grad_{n}"]) < TOL[dtype], n
        s += m
    # the order is a property of the multiple-scattering paths only: two-leg paths are the same at every order
    if 2 in legs:
        ref2 = GPUPathStage(phase(name), device="cuda", dtype=dtype).cchi(torch.tensor(z["coords_2"], dtype=st.rdtype),
                                                                            torch.tensor(z["ipots_2"]))[0]
        got2 = st.cchi(torch.tensor(z["coords_2"], dtype=st.rdtype), torch.tensor(z["ipots_2"]))[0]
        assert torch.equal(ref2, got2)
