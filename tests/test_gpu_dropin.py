"""The unmodified reference's own front end with this package installed in place of its path finder and path stage
(feffgpu_b200.install()), against the same front end on the reference's own classes, on the same GPU.

The reference is the copy installed under baseline/_ref (pip, unmodified); without it these tests are skipped.  The
front end is its PathSpectra (src/feffgpu/exafs/forward.py:67-168): path lists from the finder, coordinates rebuilt
from the positions under the minimum image of its cell, the path stage per chunk under checkpointing, the
degeneracy-weighted sum per copy.  The structure is a thermal bcc Fe frame in a triclinic cell (tests/golden/
finder_tri.npz), four absorbers.  Compared: the path counts per leg count (equal), chi per copy and its gradient with
respect to every position, both through the reference's checkpointed autograd -- complex128 to 1e-9 and 1e-7 of the
largest value, complex64 to 2e-4 and 2e-3 (two FP32 chains in different orders).  The same for its
MultipleScattering (rows per absorber, the exact gradient of a loss of the mean spectrum), its chain.run from a
feff.inp (the Cu fcc cluster, complex128), its MD-EXAFS EdgeSpectra (pair tables + multiple scattering) and its RMC
GpuRmc (spectrum, misfit and five refinement steps)."""
import dataclasses
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from tests.fixtures import npz, phase

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref"


@pytest.fixture
def reference(monkeypatch):
    if not (REF / "feffgpu" / "exafs" / "forward.py").exists():
        pytest.skip("the reference is not installed under baseline/_ref")
    monkeypatch.syspath_prepend(str(REF))
    import feffgpu
    import feffgpu.chain
    import feffgpu.exafs.forward as F
    import feffgpu.pathfinder
    import feffgpu.stage
    # the reference's own classes come back after the test
    for mod in (feffgpu, feffgpu.chain, F, feffgpu.stage, feffgpu.pathfinder):
        for name in ("GPUPathStage", "GPUPathFinder"):
            if hasattr(mod, name):
                monkeypatch.setattr(mod, name, getattr(mod, name))
    return feffgpu, F


def _spectra(F, P, pos, cell, absorbers, dtype, w):
    k = np.arange(401) * 0.05
    ps = F.PathSpectra(P, k, np.zeros(len(k)), 0.0, box=torch.tensor(cell), rmax=5.0, nlegmax=3, critpw=0.5,
                       device="cuda", dtype=dtype)
    counts = ps.refresh(pos[None], absorbers[None])
    x = torch.tensor(pos, device="cuda", dtype=torch.float32 if dtype == torch.complex64 else torch.float64,
                     requires_grad=True)
    chi = ps.spectra(x)
    (chi.double() * w[None]).sum().backward()
    return counts, chi.detach().double().cpu().numpy(), x.grad.double().cpu().numpy()


@pytest.mark.parametrize("dtype,tchi,tgrad", [(torch.complex128, 1e-9, 1e-7), (torch.complex64, 2e-4, 2e-3)])
def test_reference_front_end_with_this_package_installed(reference, dtype, tchi, tgrad):
    feffgpu, F = reference
    import feffgpu_b200
    from feffgpu.pad import PhaseData as RefPhase
    ours = phase("cfg4_fe_phase")
    P = RefPhase(**{f.name: getattr(ours, f.name) for f in dataclasses.fields(RefPhase)})
    z = npz("finder_tri")
    pos, cell = z["pos"], z["cell"]
    absorbers = np.array([0, 57, 190, 301])
    w = torch.tensor(np.random.default_rng(6).normal(size=401) * (np.arange(401) * 0.05) ** 2, device="cuda")
    c_ref, chi_ref, g_ref = _spectra(F, P, pos, cell, absorbers, dtype, w)
    done = feffgpu_b200.install()
    assert "feffgpu.exafs.forward.GPUPathStage" in done and "feffgpu.exafs.forward.GPUPathFinder" in done
    assert F.GPUPathStage is feffgpu_b200.GPUPathStage
    c_b200, chi_b200, g_b200 = _spectra(F, P, pos, cell, absorbers, dtype, w)
    assert c_b200 == c_ref, (c_b200, c_ref)
    e_chi = np.abs(chi_b200 - chi_ref).max() / np.abs(chi_ref).max()
    e_grad = np.abs(g_b200 - g_ref).max() / np.abs(g_ref).max()
    print(f"{dtype}: paths {c_ref}; chi {e_chi:.2e}, gradient {e_grad:.2e} against the reference's own classes")
    assert e_chi <= tchi and e_grad <= tgrad


def _multiple(F, P, pos, cell, absorbers):
    k = np.arange(401) * 0.05
    ms = F.MultipleScattering(P, k, 0.0, torch.tensor(cell), rmax=5.0, critpw=2.0, nlegmax=4, device="cuda")
    counts = ms.enumerate(pos[None], absorbers=absorbers)
    x = torch.tensor(pos, device="cuda", dtype=torch.float32)
    rows = ms.full_pass(x).double().cpu().numpy()
    w = torch.tensor(np.random.default_rng(7).normal(size=len(k)) * k ** 2, device="cuda")
    g = ms.full_gradient(x, lambda chi: (chi.double() * w).sum()).double().cpu().numpy()
    return counts, rows, g


def test_reference_multiple_scattering_with_this_package_installed(reference):
    """The reference's MultipleScattering (exafs/forward.py:330-760, complex64, its memory-probed batches under
    checkpointing): the same paths of 3 and 4 legs, rows per absorber and the exact gradient of a loss of the mean
    spectrum, to 2e-4 and 2e-3 of the largest value."""
    feffgpu, F = reference
    import feffgpu_b200
    from feffgpu.pad import PhaseData as RefPhase
    ours = phase("cfg4_fe_phase")
    P = RefPhase(**{f.name: getattr(ours, f.name) for f in dataclasses.fields(RefPhase)})
    z = npz("finder_tri")
    pos, cell = z["pos"], z["cell"]
    absorbers = np.array([0, 57, 190])
    c_ref, rows_ref, g_ref = _multiple(F, P, pos, cell, absorbers)
    feffgpu_b200.install()
    c_b200, rows_b200, g_b200 = _multiple(F, P, pos, cell, absorbers)
    assert c_b200 == c_ref, (c_b200, c_ref)
    e_rows = np.abs(rows_b200 - rows_ref).max() / np.abs(rows_ref).max()
    e_grad = np.abs(g_b200 - g_ref).max() / np.abs(g_ref).max()
    print(f"MultipleScattering: paths {c_ref}; rows {e_rows:.2e}, gradient {e_grad:.2e} against the reference's classes")
    assert e_rows <= 2e-4 and e_grad <= 2e-3


def test_reference_chain_with_this_package_installed(reference, tmp_path):
    """feff.inp to chi(k) through the reference's chain.run (src/feffgpu/chain.py:16-51: potentials, phase shifts,
    path finder, path stage in complex128) on the Cu fcc cluster (a = 3.61 A, 6 A, K edge, NLEG 4): once on its own
    classes, once after install() with the same potentials and phases.  The same paths, chi to 1e-9 of its largest
    value."""
    feffgpu, F = reference
    import feffgpu.chain as chain
    import feffgpu_b200
    from feffgpu_b200 import workloads as W
    pts = W.fcc_cluster(3.61, 6.0)
    lines = ["TITLE Cu fcc a=3.61 cluster 6 A", "CONTROL 1 1 1 1 1 1", "PRINT 0 0 0 0 0 0", "EDGE K", "S02 1.0",
             "NLEG 4", "RPATH 6.0", "", "POTENTIALS", "     0   29  Cu", "     1   29  Cu", "", "ATOMS"]
    lines += [f"  {x:12.6f} {y:12.6f} {z:12.6f}  {0 if i == 0 else 1:d}" for i, (x, y, z) in enumerate(pts)]
    inp = tmp_path / "feff.inp"
    inp.write_text("\n".join(lines + ["END", ""]))
    kf = np.arange(401) * 0.05
    ref = chain.run(str(inp), device="cuda", kgrid=kf)
    feffgpu_b200.install()
    assert chain.GPUPathStage is feffgpu_b200.GPUPathStage
    ours = chain.run(str(inp), device="cuda", kgrid=kf, pot=ref["pot"], phase=ref["phase"])
    assert ours["counts"] == ref["counts"], (ours["counts"], ref["counts"])
    e = np.abs(np.asarray(ours["chi"]) - np.asarray(ref["chi"])).max() / np.abs(np.asarray(ref["chi"])).max()
    print(f"chain.run Cu fcc: paths {ref['counts']}; chi {e:.2e} against the reference's own classes; "
          f"path stage {ref['timing']['chi']:.3f} s -> {ours['timing']['chi']:.3f} s")
    assert e <= 1e-9


def test_reference_md_edge_spectra_with_this_package_installed(reference):
    """The reference's MD-EXAFS front end, EdgeSpectra.spectrum (src/feffgpu/md/spectrum.py:101-340: its own
    PairTables, whose two-leg tables come from the path stage, and MultipleScattering, complex64), on the triclinic
    bcc Fe frame, eight absorbers, 3 legs within 5 A: the same path counts, chi and its single- and
    multiple-scattering parts to 2e-4 of the largest value."""
    feffgpu, F = reference
    import feffgpu_b200
    from feffgpu.md.spectrum import EdgeSpectra, phase_k_range
    from feffgpu.pad import PhaseData as RefPhase
    ours = phase("cfg4_fe_phase")
    P = RefPhase(**{f.name: getattr(ours, f.name) for f in dataclasses.fields(RefPhase)})
    z = npz("finder_tri")
    pos, cell = z["pos"], z["cell"]
    k = np.arange(int(min(20.0, phase_k_range(P)) / 0.05) + 1) * 0.05
    absorbers = np.array([0, 31, 57, 102, 190, 250, 301, 400])
    symbols = np.array(["Fe"] * len(pos))

    def run():
        es = EdgeSpectra(P, "Fe", {"Fe": 1}, ["Fe"], k, rpath=5.0, nleg=3, criteria=2.0, device="cuda")
        return es.spectrum(pos, cell, absorbers, symbols)

    ref = run()
    feffgpu_b200.install()
    got = run()
    assert got.n_paths == ref.n_paths and got.n_short_pairs == ref.n_short_pairs
    errs = {f: np.abs(getattr(got, f) - getattr(ref, f)).max() / np.abs(getattr(ref, f)).max()
            for f in ("chi", "chi_ss", "chi_ms", "ss_histogram")}
    print(f"EdgeSpectra: paths {ref.n_paths}; " + ", ".join(f"{f} {e:.2e}" for f, e in errs.items()))
    assert errs["ss_histogram"] == 0.0
    assert max(errs.values()) <= 2e-4


def test_reference_rmc_with_this_package_installed(reference):
    """The reference's RMC front end, GpuRmc (src/feffgpu/rmc/refine.py:36-260: its PairTables for single scattering,
    MultipleScattering for 3-leg paths, complex64): the exact spectrum and misfit of the triclinic bcc Fe frame
    against a target from a displaced copy, then five seeded gradient steps (sampled absorbers, SGD).  The same
    spectrum to 2e-4 and misfit to 5e-4 relative (a ratio of differences of FP32 spectra); the refined positions to
    1e-4 A."""
    feffgpu, F = reference
    import feffgpu_b200
    from feffgpu.pad import PhaseData as RefPhase
    from feffgpu.rmc.refine import GpuRmc
    ours = phase("cfg4_fe_phase")
    P = RefPhase(**{f.name: getattr(ours, f.name) for f in dataclasses.fields(RefPhase)})
    z = npz("finder_tri")
    pos, cell = z["pos"][None].astype(np.float32), z["cell"]
    k = np.arange(301) * 0.05
    moved = pos + np.random.default_rng(9).normal(0.0, 0.03, pos.shape).astype(np.float32)

    def run():
        target = GpuRmc(P, k, np.zeros(len(k)), 0.0, torch.tensor(cell), window=(3.0, 14.0), rmax=5.0, nleg=3,
                        device="cuda").spectrum_only(moved)[0].double().cpu().numpy()
        rmc = GpuRmc(P, k, target, 0.0, torch.tensor(cell), window=(3.0, 14.0), rmax=5.0, nleg=3, device="cuda")
        chi, mis = rmc.spectrum_only(pos)
        out, _ = rmc.refine(pos, 5, lr=0.003, ms_absorbers=64, value_every=5, refresh_every=250, seed=2,
                            verbose=False, log=lambda *a, **k: None)
        return chi.double().cpu().numpy(), mis, out

    chi_r, mis_r, pos_r = run()
    feffgpu_b200.install()
    chi_b, mis_b, pos_b = run()
    e_chi = np.abs(chi_b - chi_r).max() / np.abs(chi_r).max()
    e_mis = abs(mis_b - mis_r) / abs(mis_r)
    e_pos = np.abs(pos_b - pos_r).max()
    print(f"GpuRmc: chi {e_chi:.2e}, misfit {mis_r:.4e} ({e_mis:.2e}), positions after 5 steps {e_pos:.2e} A "
          f"(moved {np.abs(pos_r - pos).max():.2e} A)")
    assert e_chi <= 2e-4 and e_mis <= 5e-4 and e_pos <= 1e-4
