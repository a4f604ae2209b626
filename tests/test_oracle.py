"""The CPU oracle (oracle/feff_oracle.c + oracle/oracle.py) pinned against the reference's own outputs: per-path
cchi of the reference stage (FP64) and FEFF's chi.dat for the seven stored cases, and 2-8-leg lattice walks."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.fixtures import CASES, groups, npz, phase, r_window


@pytest.mark.parametrize("case", CASES)
def test_oracle_per_path_signal_equals_reference_stage(case):
    P = phase(f"case_{case}")
    orc = O.Oracle(P)
    z = npz(f"case_{case}")
    for nleg, (coords, ipots, deg) in groups(f"case_{case}").items():
        k = min(4, len(coords))
        cc, rf = orc.cchi(coords[:k], ipots[:k])
        ref = z[f"ref_cchi_{nleg}"]
        assert np.abs(cc - ref).max() <= 1e-10 * np.abs(ref).max(), (case, nleg)
        assert np.allclose(rf, z[f"ref_reff_{nleg}"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("case", CASES)
def test_oracle_chi_equals_reference_chi_and_feff(case):
    """FEFF's path list through the oracle: chi equals the reference stage's to R < 1e-14 and FEFF's chi.dat to the
    reference's own bar (R < 2e-5, tests/test_validation_cases.py:50; W: R < 1e-9, tests/test_xsph.py:122)."""
    P = phase(f"case_{case}")
    orc = O.Oracle(P)
    z = npz(f"case_{case}")
    kf = z["feff_k"]
    S = orc.linear_matrix(kf)
    chi = np.zeros(len(kf))
    for nleg, (coords, ipots, deg) in groups(f"case_{case}").items():
        cc, rf = orc.cchi(coords, ipots)
        chi += (deg[:, None] * O.chi_fine(cc, rf, kf, S)).sum(0)
    k0 = np.concatenate([[0.0], kf])
    z0 = lambda c: np.concatenate([[0.0], c])
    w = r_window(f"case_{case}", kf)
    assert O.r_factor(k0, z0(z["ref_chi"]), z0(chi), **w) < 1e-14
    assert O.r_factor(k0, z0(z["feff_chi"]), z0(chi), **w) < (1e-9 if case == "W" else 2e-5)


def test_oracle_walks_two_to_eight_legs():
    """tests/test_pathfinder.py:214-230's bar: |dcchi| < 1e-8 max|cchi| below k = 20 1/A, reff to 1e-10."""
    P = phase("case_W")
    orc = O.Oracle(P)
    z = npz("walks_W")
    low = orc.kgrid() < 20.0
    for nleg in range(2, 9):
        cc, rf = orc.cchi(z[f"coords_{nleg}"], z[f"ipots_{nleg}"])
        ref = z[f"ref_cchi_{nleg}"]
        assert np.abs(cc - ref)[:, low].max() < 1e-8 * np.abs(ref[:, low]).max(), nleg
        assert np.allclose(rf, z[f"ref_reff_{nleg}"], rtol=1e-10)


def test_oracle_gradient_by_finite_differences_matches_reference_autograd():
    """Central differences (h = 1e-4 A) of the oracle's loss against the reference's checkpointed autograd."""
    z = npz("grad_L001")
    P = phase("grad_L001")
    orc = O.Oracle(P)
    q, w = z["q"], z["w"]
    S = orc.linear_matrix(q)
    for nleg in (2, 3):
        coords, ipots, deg, ref = z[f"coords_{nleg}"], z[f"ipots_{nleg}"], z[f"deg_{nleg}"], z[f"grad_{nleg}"]

        def loss(c):
            cc, rf = orc.cchi(c, ipots[:len(c)], nthreads=1)
            return float((deg[:len(c), None] * O.chi_fine(cc, rf, q, S) * w[None]).sum())

        g = O.fd_gradient(loss, coords[:1], h=1e-4)
        rel = np.abs(g - ref[:1]).max() / np.abs(ref[:1]).max()
        assert rel < 1e-4, (nleg, rel)


def test_lambda_sets():
    """setlam (genfmt.py:115-153) for K, L3 and M5 edges."""
    assert O.lambda_set(1, 2)[:4] == ([0, -1, 1, 0, -2, 2], [0, 0, 0, 1, 0, 0], 6, 4)
    assert O.lambda_set(1, 1)[:4] == ([0, -1, 1, 0, -1, 1], [0, 0, 0, 1, 1, 1], 6, 6)
    m, n, lamx, laml0x, mmaxp1, nmax = O.lambda_set(9, 1)
    assert (lamx, laml0x, mmaxp1, nmax) == (15, 15, 4, 2)


def test_wigner_d_unitarity_and_symmetry():
    d = O.wigner_d(1.234, 30)
    for l in (3, 10, 30):
        m = min(l, 3)
        blk = d[l, 3 - m:4 + m, 3 - m:4 + m]
        if l <= 3:
            assert np.allclose(blk @ blk.T, np.eye(2 * m + 1), atol=1e-12)
        for a in range(-m, m + 1):
            for b in range(-m, m + 1):
                assert abs(d[l, a + 3, b + 3] - (-1) ** (a - b) * d[l, -a + 3, -b + 3]) < 1e-12


def test_oracle_on_the_benchmark_batch_sample():
    """The oracle on the reference finder's paths of the benchmark packing (tests/golden/bench_sample.npz: 592 paths,
    every absorber and leg count of the benchmark batch, phase tables resampled to 401 k) equals the reference
    stage's FP64 rows to R < 1e-20 and its per-path cchi to 1e-10."""
    from feffgpu_b200.pad import phase_from_npz, resample_phase
    z = npz("bench_sample")
    q = z["q"]
    P = resample_phase(phase_from_npz(npz("cfg2_phase"), prefix="ph_"), q)
    orc = O.Oracle(P)
    S = orc.linear_matrix(q)
    per = int(z["per_cchi"])
    for r, (s, nleg) in enumerate(z["row_keys"]):
        c = z[f"coords_{s}_{nleg}"].astype(np.float64)
        cc, rf = orc.cchi(c, z[f"ipots_{s}_{nleg}"])
        row = (z[f"deg_{s}_{nleg}"][:, None] * O.chi_fine(cc, rf, q, S)).sum(0)
        assert O.r_factor(q, z["rows"][r], row, kmin=3, kmax=19, rmin=1, rmax=8) < 1e-20
        refc = z[f"cchi_{s}_{nleg}"]
        assert np.abs(cc[:per] - refc).max() <= 1e-10 * np.abs(refc).max()
