"""The parity gate on the benchmark's own batch (runs on a B200).

The benchmark evaluates every path of 2-8 legs within 8 A of the two most central Fe absorbers of the seeded
3000-atom Fe/O/Pt packing (no importance cut; 1.89e5 paths) on the reference's Fe K phase shifts resampled to 401 k.
tests/golden/bench_sample.npz holds a seeded stratified sample of that batch as the reference's own path finder gives
it (48 paths of every absorber and leg count, every 8-leg path) and the reference stage's FP64 (complex128) signals.
Here this package's CUDA path finder regenerates the batch, must give the same atoms at the sampled positions, and
the fused stage's rows of the sample -- one row per absorber and leg count -- are compared with the reference's rows
and with the oracle's:

  mixed form (complex64): R <= 1e-6 per row (the parity gate), per-path cchi within 2e-5 of max|cchi|;
  FP64 form (complex128): R <= 1e-12 per row, per-path cchi within 1e-10 of max|cchi|.

R is the reference's R-factor (compare.py:17-27) with k 3-19 1/A, R 1-8 A, k weight 2.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.fixtures import npz

pytestmark = pytest.mark.gpu

WIN = dict(kmin=3.0, kmax=19.0, rmin=1.0, rmax=8.0)
TOL = {torch.complex64: (1e-6, 2e-5), torch.complex128: (1e-12, 1e-10)}


def _sample_batch():
    from feffgpu_b200 import PathBatch
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.pad import phase_from_npz
    from feffgpu_b200.pathfinder import GPUPathFinder
    z = npz("bench_sample")
    P0 = phase_from_npz(npz("cfg2_phase"), prefix="ph_")
    pos, lab, box = W.random_packing(3000, 0.08, 1.8, seed=2024)
    ipot_of = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    absorbers = W.central_atom(pos, box, lab, "Fe", 2)
    assert np.array_equal(absorbers, z["absorbers"])
    finder = GPUPathFinder(P0, device="cuda", rmax=8.0, nlegmax=8, critpw=0.0)
    groups, sample = [], []
    for row, (s, nleg) in enumerate(z["row_keys"]):
        if nleg == 2 or row == 0:
            kept, _ = finder.enumerate(pos, box, int(absorbers[s]), ipot_of)
        coords, ipots, deg, _xp, atoms = kept[int(nleg)]
        assert int(coords.shape[0]) == int(z[f"count_{s}_{nleg}"])
        idx = torch.as_tensor(z[f"idx_{s}_{nleg}"], device=coords.device)
        assert np.array_equal(atoms[idx].cpu().numpy(), z[f"atoms_{s}_{nleg}"])
        c = coords[idx].cpu().numpy()
        assert np.array_equal(c, z[f"coords_{s}_{nleg}"])
        groups.append((c.astype(np.float64), ipots[idx].cpu().numpy(), deg[idx].double().cpu().numpy(),
                       np.full(len(idx), row)))
        sample.append((s, nleg, c.astype(np.float64), z[f"ipots_{s}_{nleg}"], z[f"deg_{s}_{nleg}"]))
    return PathBatch(groups, nrows=len(z["row_keys"]), device="cuda"), sample


def test_benchmark_batch_sample_against_reference_and_oracle():
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200.pad import phase_from_npz, resample_phase
    z = npz("bench_sample")
    q = z["q"]
    P = resample_phase(phase_from_npz(npz("cfg2_phase"), prefix="ph_"), q)
    batch, sample = _sample_batch()
    assert batch.n >= 500 and set(batch.counts) == set(range(2, 9))
    orc = O.Oracle(P)
    S = orc.linear_matrix(q)
    ref_oracle = np.stack([(deg[:, None] * O.chi_fine(*orc.cchi(c, ip), q, S)).sum(0) for _, _, c, ip, deg in sample])
    per = int(z["per_cchi"])
    for dtype, (tol_r, tol_c) in TOL.items():
        st = GPUPathStage(P, device="cuda", dtype=dtype)
        rows = st.chi_reduce(batch, q).cpu().numpy()
        worst_ref = worst_orc = worst_c = 0.0
        for r, (s, nleg, c, ip, _deg) in enumerate(sample):
            R_ref = O.r_factor(q, z["rows"][r], rows[r], **WIN)
            R_orc = O.r_factor(q, ref_oracle[r], rows[r], **WIN)
            worst_ref, worst_orc = max(worst_ref, R_ref), max(worst_orc, R_orc)
            cc, _ = st.cchi(torch.tensor(c[:per]), torch.tensor(ip[:per]))
            refc = z[f"cchi_{s}_{nleg}"]
            worst_c = max(worst_c, float(np.abs(cc.cpu().numpy() - refc).max() / np.abs(refc).max()))
        print(f"{dtype}: R vs reference {worst_ref:.2e}, vs oracle {worst_orc:.2e}, cchi {worst_c:.2e}")
        assert worst_ref <= tol_r and worst_orc <= tol_r and worst_c <= tol_c
