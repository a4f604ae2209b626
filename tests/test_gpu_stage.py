"""GPU parity of the path stage against the oracle and the reference's golden outputs (runs on a B200).

Tolerances (written here, checked here):
  FP64 form (complex128): per-path cchi within 1e-10 of max|cchi| of the reference stage below k = 20 1/A (the
    reference's own bar against its literal port is 1e-8, tests/test_pathfinder.py:226); chi R < 1e-12.
  Mixed form (complex64): per-path cchi within 2e-5 of max|cchi|; chi R <= 1e-6 against the reference's FP64 chi
    (the parity gate of the path stage).
  Both: FEFF's chi.dat to the reference's bars (R < 1e-9 for W, tests/test_xsph.py:122; R < 2e-5 otherwise,
    tests/test_validation_cases.py:50).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.fixtures import CASES, cfg2_phase, groups, npz, phase, r_window

pytestmark = pytest.mark.gpu

TOL_CCHI = {torch.complex128: 1e-10, torch.complex64: 2e-5}
TOL_R = {torch.complex128: 1e-12, torch.complex64: 1e-6}
DTYPES = [torch.complex128, torch.complex64]


def _stage(P, dtype):
    from feffgpu_b200 import GPUPathStage
    return GPUPathStage(P, device="cuda", dtype=dtype)


def _rel(a, b, sel=None):
    a, b = np.asarray(a), np.asarray(b)
    if sel is not None:
        a, b = a[:, sel], b[:, sel]
    return float(np.abs(a - b).max() / np.abs(b).max())


def _R(name, k, a, b):
    k0 = np.concatenate([[0.0], k])
    z0 = lambda c: np.concatenate([[0.0], c])
    return O.r_factor(k0, z0(a), z0(b), **r_window(name, k))


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("case", CASES)
def test_cchi_equals_reference_stage(case, dtype):
    name = f"case_{case}"
    P = phase(name)
    st = _stage(P, dtype)
    z = npz(name)
    orc = O.Oracle(P)
    low = orc.kgrid() < 20.0
    for nleg, (coords, ipots, deg) in groups(name).items():
        cc, rf = st.cchi(torch.tensor(coords), torch.tensor(ipots))
        assert cc.dtype == dtype and rf.dtype == st.rdtype and cc.shape == (len(coords), st.E)
        cc = cc.cpu().numpy()
        k = min(4, len(coords))
        e_ref = _rel(cc[:k], z[f"ref_cchi_{nleg}"], low)
        oc, orf = orc.cchi(coords, ipots)
        e_orc = _rel(cc, oc, low)
        print(f"{case} nleg {nleg} {dtype}: vs reference {e_ref:.2e}, vs oracle {e_orc:.2e}")
        assert e_ref < TOL_CCHI[dtype] and e_orc < TOL_CCHI[dtype], (nleg, e_ref, e_orc)
        assert np.allclose(rf.cpu().numpy(), orf, rtol=1e-6 if dtype == torch.complex64 else 1e-12)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("case", CASES)
def test_chi_equals_reference_and_feff(case, dtype):
    """FEFF's own path list -> chi through cchi + chi_fine + degeneracy sum, as chain.run does (chain.py:45-49)."""
    name = f"case_{case}"
    st = _stage(phase(name), dtype)
    z = npz(name)
    kf = z["feff_k"]
    S = st.linear_matrix(kf)
    chi = torch.zeros(len(kf), dtype=torch.float64, device="cuda")
    with torch.no_grad():
        for nleg, (coords, ipots, deg) in groups(name).items():
            cc, rf = st.cchi(torch.tensor(coords), torch.tensor(ipots))
            chi += (torch.tensor(deg, device="cuda")[:, None] * st.chi_fine(cc, rf, kf, S, "feff").double()).sum(0)
    chi = chi.cpu().numpy()
    r_ref, r_feff = _R(name, kf, z["ref_chi"], chi), _R(name, kf, z["feff_chi"], chi)
    print(f"{case} {dtype}: R(ref) {r_ref:.2e}  R(FEFF) {r_feff:.2e}")
    assert r_ref <= TOL_R[dtype]
    assert r_feff < (1e-9 if case == "W" else 2e-5)


@pytest.mark.parametrize("dtype", DTYPES)
def test_walks_two_to_eight_legs(dtype):
    st = _stage(phase("case_W"), dtype)
    z = npz("walks_W")
    low = (st.xk.double().cpu().numpy() / 0.52917721067) < 20.0
    for nleg in range(2, 9):
        cc, rf = st.cchi(torch.tensor(z[f"coords_{nleg}"]), torch.tensor(z[f"ipots_{nleg}"]))
        e = _rel(cc.cpu().numpy(), z[f"ref_cchi_{nleg}"], low)
        print(f"walk nleg {nleg} {dtype}: {e:.2e}")
        assert e < TOL_CCHI[dtype], (nleg, e)
        assert np.allclose(rf.cpu().numpy(), z[f"ref_reff_{nleg}"], rtol=1e-6 if dtype == torch.complex64 else 1e-10)


@pytest.mark.parametrize("dtype", DTYPES)
def test_resampled_401k_tables(dtype):
    """The Fe/O/Pt tables (lmax 24) resampled to 401 k points, paths of 2-8 legs, against the reference stage."""
    st = _stage(cfg2_phase(), dtype)
    z = npz("cfg2_sample")
    for nleg in range(2, 9):
        cc, rf = st.cchi(torch.tensor(z[f"coords_{nleg}"]), torch.tensor(z[f"ipots_{nleg}"]))
        e = _rel(cc.cpu().numpy(), z[f"ref_cchi_{nleg}"])
        print(f"cfg2 nleg {nleg} {dtype}: {e:.2e}")
        assert e < TOL_CCHI[dtype], (nleg, e)


def _batch_of(name, rows_of=None):
    from feffgpu_b200 import PathBatch
    gs = []
    for nleg, (coords, ipots, deg) in groups(name).items():
        row = None if rows_of is None else rows_of(len(coords))
        gs.append((coords, ipots, deg, row))
    return PathBatch(gs, device="cuda")


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("case", ["W", "A009", "A014", "L001"])
def test_fused_chi_reduce(case, dtype):
    """One persistent launch over all leg counts, fine grid and degeneracy sum: equals the oracle and the reference."""
    name = f"case_{case}"
    st = _stage(phase(name), dtype)
    z = npz(name)
    kf = z["feff_k"]
    b = _batch_of(name)
    rows = st.chi_reduce(b, kf)
    assert rows.shape == (1, len(kf)) and rows.dtype == torch.float64
    chi = rows[0].cpu().numpy()
    r_ref = _R(name, kf, z["ref_chi"], chi)
    print(f"fused {case} {dtype}: R(ref) {r_ref:.2e}")
    assert r_ref <= TOL_R[dtype]
    # deterministic: a second launch gives the same bits
    assert torch.equal(rows, st.chi_reduce(b, kf))


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_rows_and_sigma2(dtype):
    """Paths spread over rows, with per-path sigma^2 damping exp(-2 sigma^2 q^2), against the oracle's FP64 sums."""
    name = "case_A000"
    P = phase(name)
    st = _stage(P, dtype)
    rng = np.random.default_rng(1)
    b = _batch_of(name, rows_of=lambda n: rng.integers(0, 5, n))
    s2 = rng.uniform(0, 0.01, b.n)
    q = np.arange(1, 401) * 0.05
    rows = st.chi_reduce(b, q, sigma2=torch.tensor(s2)).cpu().numpy()
    orc = O.Oracle(P)
    S = orc.linear_matrix(q)
    coords, ipots, nleg = b.coords.cpu().numpy(), b.ipots.cpu().numpy(), b.nleg.cpu().numpy()
    chi_p = np.zeros((b.n, len(q)))
    for n in np.unique(nleg):
        sel = np.nonzero(nleg == n)[0]
        cc, rf = orc.cchi(coords[sel, :n], ipots[sel, :n])
        chi_p[sel] = O.chi_fine(cc, rf, q, S)
    ref = O.chi_rows(chi_p, b.deg.cpu().numpy(), b.row.cpu().numpy(), b.nrows, q, s2)
    for r in range(b.nrows):
        Rr = O.r_factor(np.concatenate([[0.0], q]), np.concatenate([[0.0], ref[r]]), np.concatenate([[0.0], rows[r]]),
                        kmin=3, kmax=19, rmin=1, rmax=6)
        assert Rr <= TOL_R[dtype], (r, Rr)
    if dtype == torch.complex128:
        assert np.abs(rows - ref).max() < 1e-10 * np.abs(ref).max()


def test_edge_cases():
    from feffgpu_b200 import GPUPathStage, PathBatch
    P = phase("case_L001")
    st = GPUPathStage(P, device="cuda", dtype=torch.complex128)
    cc, rf = st.cchi(torch.zeros(0, 3, 3), torch.zeros(0, 3, dtype=torch.long))
    assert cc.shape == (0, st.E) and rf.shape == (0,)
    with pytest.raises(IndexError):
        st.cchi(torch.tensor([[[0, 0, 0], [1.5, 0, 0.2]]]), torch.tensor([[0, 7]]))
    with pytest.raises(ValueError):
        st.cchi(torch.zeros(1, 10, 3), torch.zeros(1, 10, dtype=torch.long))
    # nine legs (the largest the path finder allows) against the oracle
    rng = np.random.default_rng(3)
    coords = np.concatenate([np.zeros((2, 1, 3)), rng.normal(0, 1.5, (2, 8, 3))], 1)
    ipots = np.ones((2, 9), int)
    ipots[:, 0] = 0
    cc, _ = st.cchi(torch.tensor(coords), torch.tensor(ipots))
    oc, _ = O.Oracle(P).cchi(coords, ipots)
    assert _rel(cc.cpu().numpy(), oc) < 1e-10
    # coords on the host and float32 input are accepted, as in the reference
    cc32, _ = st.cchi(torch.tensor(coords, dtype=torch.float32), torch.tensor(ipots))
    assert cc32.device.type == "cuda"
    # an empty batch and an empty row
    b = PathBatch([(coords, ipots, None, np.array([0, 2]))], nrows=3, device="cuda")
    rows = st.chi_reduce(b, np.arange(1, 101) * 0.1)
    assert rows.shape == (3, 100) and torch.all(rows[1] == 0)


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_stage_reports_bad_potential_indices_and_layouts(dtype):
    """An out-of-range potential index in a fused batch raises IndexError in the Python layer before any launch, and
    through the C ABI the kernels clamp it (no out-of-bounds read), turn the rows NaN and the call returns
    FG_ERR_VALUE; the backward likewise.  A malformed launch order (a path index past n) is reported the same way
    and never used to address memory.  The reference raises IndexError from its table lookup (stage.py:244)."""
    import ctypes as C
    from feffgpu_b200 import GPUPathStage, PathBatch, _lib
    P = phase("case_L001")
    st = GPUPathStage(P, device="cuda", dtype=dtype)
    gs = groups("case_L001")
    coords, ipots, deg = gs[3]
    bad = ipots[:4].copy()
    bad[2, 1] = P.nph + 3
    b = PathBatch([(coords[:4], bad, deg[:4])], device="cuda")
    q = np.arange(1, 401) * 0.05
    with pytest.raises(IndexError):
        st.chi_reduce(b, q)
    qt = torch.tensor(q, dtype=torch.float64, device="cuda")
    S = st.linear_matrix(q).double().contiguous()
    span = st._span(S)
    stream = torch.cuda.current_stream().cuda_stream

    def call(batch, order=None):
        ps = st._paths_struct(batch, batch.coords, None)
        if order is not None:
            ps.order = order.data_ptr()
        rows = torch.zeros(batch.nrows, 400, dtype=torch.float64, device="cuda")
        n = int(st._lib.fg_chi_reduce_workspace(st._h, C.byref(ps), 400))
        ws = torch.empty(n, dtype=torch.uint8, device="cuda")
        cc = torch.empty(batch.n, st.E, dtype=st.cdtype, device="cuda")
        rf = torch.empty(batch.n, dtype=torch.float64, device="cuda")
        rc = st._lib.fg_chi_reduce(st._h, st.prec, C.byref(ps), 400, qt.data_ptr(), S.data_ptr(), span.data_ptr(),
                                   rows.data_ptr(), cc.data_ptr(), rf.data_ptr(), ws.data_ptr(), n, stream)
        return rc, rows, ps, cc, rf

    rc, rows, ps, cc, rf = call(b)
    msg = st._lib.fg_last_error().decode()
    assert rc == _lib.FG_ERR_VALUE and "potential index" in msg
    assert torch.isnan(rows).all()
    rc2 = st._lib.fg_chi_reduce_noalloc(st._h, st.prec, C.byref(ps), 400, qt.data_ptr(), S.data_ptr(),
                                        span.data_ptr(), rows.data_ptr(), stream)
    assert rc2 == _lib.FG_ERR_VALUE and "potential index" in st._lib.fg_last_error().decode()
    with pytest.raises(IndexError):
        _lib.check(rc2)
    # the backward of the same batch reports it too
    g = torch.ones(1, 400, dtype=torch.float64, device="cuda")
    gc = torch.empty_like(b.coords)
    nb = int(st._lib.fg_chi_reduce_backward_workspace(st._h, C.byref(ps), 400))
    wsb = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rc3 = st._lib.fg_chi_reduce_backward(st._h, st.prec, C.byref(ps), 400, qt.data_ptr(), S.data_ptr(),
                                         span.data_ptr(), st._span(S, True).data_ptr(), g.data_ptr(), cc.data_ptr(),
                                         rf.data_ptr(), gc.data_ptr(), None, wsb.data_ptr(), nb, stream)
    assert rc3 == _lib.FG_ERR_VALUE and "potential index" in st._lib.fg_last_error().decode()
    # a valid batch with a launch order that names a path past n: reported, rows NaN
    good = PathBatch([(coords[:4], ipots[:4], deg[:4])], device="cuda")
    order = torch.tensor([0, 1, 7, 3], dtype=torch.int32, device="cuda")
    rc4, rows4, *_ = call(good, order)
    assert rc4 == _lib.FG_ERR_VALUE and "malformed" in st._lib.fg_last_error().decode()
    assert torch.isnan(rows4).all()
    # and the same batch with its own order is fine afterwards (the status word is cleared per call)
    rc5, rows5, *_ = call(good)
    assert rc5 == _lib.FG_OK and torch.isfinite(rows5).all()


@pytest.mark.parametrize("dtype", DTYPES)
def test_larch_spline_convention_equals_reference(dtype):
    """spline_matrix (scipy UnivariateSpline s=0, the reference's stage.py:341-351) and chi_fine(..., "larch") on the
    W case's stored paths against the reference's (tests/golden/larch_W.npz): the matrix to 1e-12, chi to 1e-10 of its
    largest value in FP64 (the mixed form: 5e-5; its spline weights are FP32, as the reference's complex64 form casts
    them, and the spline's weights alternate in sign, so their rounding is not damped as linear weights' is)."""
    from feffgpu_b200 import GPUPathStage
    z = npz("larch_W")
    case = npz("case_W")
    st = GPUPathStage(phase("case_W"), device="cuda", dtype=dtype)
    S = st.spline_matrix(z["q"])
    assert np.abs(S.double().cpu().numpy() - z["S"]).max() <= (1e-12 if dtype == torch.complex128 else 1e-6)
    for nleg in (2, 3, 4):
        cc = torch.tensor(case[f"ref_cchi_{nleg}"], device="cuda").to(dtype)
        rf = torch.tensor(case[f"ref_reff_{nleg}"], device="cuda")
        chi = st.chi_fine(cc, rf, z["q"], convention="larch").double().cpu().numpy()
        e = _rel(chi, z[f"chi_{nleg}"])
        print(f"larch nleg {nleg} {dtype}: chi vs reference {e:.2e}")
        assert e <= (1e-10 if dtype == torch.complex128 else 5e-5), (nleg, e)


def test_gaussian_frames_damp_the_first_shell_like_the_sigma2_factor():
    """Frames of independent Gaussian displacements (s = 0.04 A per component, 40 frames of a bcc W block, every atom
    an absorber, the first shell's two-leg paths through the batched finder and the fused stage): the frame average
    decays against the ideal lattice like exp(-2 k^2 sigma^2) with sigma^2 = 2 s^2 (the reference's check of its MD
    averaging, tests/md/test_spectrum.py:166-201 there), and its envelope equals that of the ideal lattice's spectrum
    with the per-path factor exp(-2 sigma^2 q^2) of sigma^2 = 2 s^2 to 3 % over k = 3..14 (the spectra themselves
    differ by the phase of the mean-distance shift of a 3D Gaussian, sigma_perp^2 / R, which the factor leaves out).
    Envelopes: the magnitude of the analytic signal (scipy's hilbert) on q = 0.05..19.95."""
    from scipy.signal import hilbert
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.pathfinder import GPUPathFinder
    s, F = 0.04, 40
    sites, box = W.bcc_supercell(4, 3.1652)
    n = len(sites)
    frames = sites[None] + np.random.default_rng(1).normal(0.0, s, (F, n, 3))
    P = phase("case_W")
    f = GPUPathFinder(P, device="cuda", rmax=2.95, nlegmax=2, critpw=0.0, merge_degenerate=False)
    st = GPUPathStage(P, device="cuda", dtype=torch.complex128)
    q = np.arange(1, 400) * 0.05          # to 19.95: the envelope's edge effects stay away from the fit window

    def rows(pos, sigma2=None):
        fr = pos if pos.ndim == 3 else pos[None]
        res = f.enumerate_many(fr, box, np.arange(n), np.ones(n, int))
        coords, ipots, deg, _xp, _atoms, slot = res["paths"][2]
        b = PathBatch([(coords.double(), ipots, deg.double(), torch.div(slot, n, rounding_mode="floor"))],
                      nrows=fr.shape[0], device="cuda")
        s2 = None if sigma2 is None else torch.full((b.n,), sigma2, device="cuda", dtype=torch.float64)
        return st.chi_reduce(b, q, sigma2=s2).cpu().numpy() / n

    avg = rows(frames).mean(0)
    ideal = rows(sites)[0]
    damped = rows(sites, 2 * s * s)[0]
    m = (q >= 5.0) & (q <= 14.0)
    env = lambda y: np.abs(hilbert(y))
    y = np.log(env(avg)[m] / env(ideal)[m])
    A = np.vstack([np.ones(m.sum()), q[m] ** 2]).T
    (c, slope), *_ = np.linalg.lstsq(A, y, rcond=None)
    sigma2 = -slope / 2
    print(f"sigma^2 from the frames' spectrum {sigma2:.5f} (2 s^2 = {2 * s * s:.5f}), offset {c:.3f}")
    assert np.abs(y - A @ np.array([c, slope])).max() < 0.05 and abs(c) < 0.03
    assert abs(sigma2 - 2 * s * s) < 0.1 * 2 * s * s
    w = (q >= 3.0) & (q <= 14.0)
    e = np.abs(env(avg)[w] / env(damped)[w] - 1.0).max()
    print(f"envelope of the frame average vs the sigma^2 factor on the ideal lattice: {e:.3f}")
    assert e < 0.03


@pytest.mark.parametrize("dtype", DTYPES)
def test_geometry_equals_reference(dtype):
    """GPUPathStage.geometry (stage.py:170-206): ri, beta, eta of 2-8-leg paths -- random ones and the degenerate
    cases the reference's branch choices define (a leg along z, collinear atoms, a revisit) -- and the gradient of a
    weighted sum of them, against the reference's values and autograd (tests/golden/geometry_ref.npz).  For the leg
    along z the reference's autograd gives NaN in the components that pass through its small-vector branch (its
    Euler angles are constants there); those are left out, and this gradient is finite everywhere."""
    from feffgpu_b200 import GPUPathStage
    z = npz("geometry_ref")
    st = GPUPathStage(phase("case_L001"), device="cuda", dtype=dtype)
    for nleg in range(2, 9):
        x = torch.tensor(z[f"coords_{nleg}"], device="cuda", requires_grad=True)
        ri, beta, eta = st.geometry(x)
        assert ri.dtype == torch.float64 and ri.shape == (len(x), nleg)
        for got, key in ((ri, "ri"), (beta, "beta"), (eta, "eta")):
            ref = z[f"{key}_{nleg}"]
            assert np.abs(got.detach().cpu().numpy() - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (nleg, key)
        w = [torch.tensor(z[f"{k}_{nleg}"], device="cuda") for k in ("wr", "wb", "we")]
        (w[0] * ri + w[1] * beta + w[2] * eta).sum().backward()
        g, ref = x.grad.cpu().numpy(), z[f"grad_{nleg}"]
        ok = np.isfinite(ref)
        assert np.all(np.isfinite(g)) and ok.mean() > 0.9, nleg
        assert np.abs(g - np.where(ok, ref, g)).max() <= 1e-10 * np.abs(ref[ok]).max(), nleg
    # float32 coordinates come back as float32, still differentiable
    x32 = torch.tensor(z["coords_3"], dtype=torch.float32, requires_grad=True)
    ri32 = st.geometry(x32)[0]
    assert ri32.dtype == torch.float32
    ri32.sum().backward()
    assert x32.grad is not None and x32.grad.dtype == torch.float32


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_stage_reports_terms_out_of_range(dtype):
    """A weighted path term that is not finite (a NaN coordinate) or reaches 2^31 in magnitude (a huge degeneracy)
    cannot enter the exact fixed-point sums: nothing of it is added, the call raises ValueError naming the cause and
    its rows are NaN; the stage works normally afterwards."""
    from feffgpu_b200 import GPUPathStage, PathBatch
    P = phase("case_L001")
    st = GPUPathStage(P, device="cuda", dtype=dtype)
    coords, ipots, deg = groups("case_L001")[3]
    q = np.arange(1, 401) * 0.05
    good = PathBatch([(coords[:5], ipots[:5], deg[:5])], device="cuda")
    ref = st.chi_reduce(good, q)
    huge = deg[:5].copy()
    huge[2] = 1e14
    with pytest.raises(ValueError, match="2\\^31"):
        st.chi_reduce(PathBatch([(coords[:5], ipots[:5], huge)], device="cuda"), q)
    bad = coords[:5].copy()
    bad[1, 1, 0] = np.nan
    with pytest.raises(ValueError, match="not finite"):
        st.chi_reduce(PathBatch([(bad, ipots[:5], deg[:5])], device="cuda"), q)
    assert torch.equal(st.chi_reduce(good, q), ref)
