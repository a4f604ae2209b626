"""Generates the golden fixtures of tests/golden/ from the reference implementation (nmarcella/feffGPU).

Run where a copy of the reference's source tree is at hand, giving its root (the directory holding src/feffgpu):

    python tests/golden/make_golden.py REFERENCE_ROOT [--only NAME ...]

The reference is imported read-only from its source tree and run on the CPU in FP64 (complex128).  Outputs are small
.npz files; nothing at test time reads the reference itself.

* case_<name>.npz -- for FEFF's seven stored cases (tests/data/W and data/validation/*): the phase tables the path
  stage reads (first ne1 energies, l up to the largest lmax), FEFF's own path list (paths.dat) and chi (chi.dat),
  the reference stage's chi on chi.dat's k grid from that path list, and its per-path cchi/reff for a few paths
  of every leg count (the procedure of the reference's tests/test_xsph.py:85-123).
* walks_W.npz -- 2- to 8-leg bcc lattice walks with the W phases and the reference stage's cchi (the procedure of
  tests/test_pathfinder.py:193-230, seed 5).
* grad_walks_W.npz -- the same for the W walks (loss sum_q w_q chi(q) with seeded w).
* grad_L001.npz, grad_A000.npz, grad_A014.npz (L3), grad_A009.npz (M5) -- d(loss)/d(coords) of the reference stage under torch.utils.checkpoint
  (use_reentrant=False, as src/feffgpu/exafs/forward.py:683 calls it), loss = sum_p deg_p sum_q w_q chi_p(q).
* L001_phase.pad -- FEFF's phase.pad of the L001 case, copied as written by FEFF, for the reader's test.
* cfg1_cu.npz -- the Cu fcc cluster (a = 3.61 A, 6 A radius, K edge) through the reference chain
  (src/feffgpu/chain.py:16-51): phase tables, the path finder's paths (NLEG 4, RPATH 6, default importance cut) and chi on
  k = 0..20 A^-1 step 0.05.
* cfg4_fe_phase.npz, cfg5_nik_phase.npz, cfg5_ok_phase.npz -- bcc Fe (K edge) and rock-salt NiO (Ni K and O K
  edges) phase tables of 6 A clusters through the reference chain, for the MD-batch and two-edge refinement cases.
* geometry_ref.npz -- the reference stage's geometry (ri, beta, eta) of 2-8-leg paths, degenerate ones included, and
  the gradient of a weighted sum of it by its autograd;
* grad_L001_io0/io1/io3.npz, grad_A014_io0/io1/io3.npz, grad_A009_io3.npz -- as grad_*.npz with the reference
  stage at lambda-set orders 0, 1 and 3 (GPUPathStage(..., iorder=k)), with its cchi of every path;
* finder_lone/one/two/blk/ss.npz -- the same for the enumeration's edge cases: an absorber with no candidate, with one
  (single scattering only) and with two, a 600-atom packing in a box (3 legs), and single scattering alone (2 legs);
* finder_cu.npz, finder_pack.npz, finder_bcc.npz -- the reference's path finder on the Cu cluster (rmax 6, 4 legs),
  a 400-atom periodic Fe/O/Pt packing (rmax 6.5, 7 legs) and a thermal bcc Fe frame (rmax 5.5, 3 legs), each without
  and with an importance cut; finder_feopt.npz -- the reference finder's paths on the benchmark packing (counts,
  hashes and ends of the atom sequences per leg count, two absorbers, rmax 8 A, 8 legs); finder_tri.npz -- a thermal
  bcc Fe frame in a triclinic cell (the supercell sheared by SHEAR, rmax 5, 4 legs), the reference finder given the
  3 x 3 cell.
* feffdat_W.npz -- FEFF's own feff0001..0008.dat of the W case: path geometry and the seven columns.
* larch_W.npz -- the reference stage's cubic-spline interpolation matrix and its "larch"-convention fine-grid chi of
  the W case's stored paths.
* pairs_nio.npz -- the reference's single-scattering pair tables, histogram, all-pairs spectrum and its position
  gradient on a thermal rock-salt NiO supercell (Ni K edge); pairs_nio_tri.npz -- the same in a triclinic cell.
* bench_sample.npz -- a stratified sample of the benchmark batch with the reference's FP64 signals (make_bench_sample);
  rspace_ref.npz -- the reference's R-space losses and gradients (make_rspace); cfg3_adjoint.npz -- configuration 3's
  loss and position gradient through the reference's PathSpectra and autograd (make_cfg3).
* cfg2_phase.npz -- Fe K-edge phase tables (potentials Fe*, Fe, O, Pt, lmax 24) of a cluster cut from the seeded
  3000-atom Fe/O/Pt packing, on FEFF's own energy grid; cfg2_sample.npz -- the reference stage's cchi on those
  tables resampled to 401 k points, for a sample of synthetic paths.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF: Path = Path()      # the reference's source root, set by main() from its required argument
CASES: dict = {}
sys.path.insert(0, str(REPO))

import torch  # noqa: E402

from feffgpu_b200.pad import phase_to_arrays, phase_from_npz, resample_phase  # noqa: E402
from feffgpu_b200 import workloads as W  # noqa: E402

def set_reference(root: str) -> None:
    """Import the reference read-only from root/src and locate FEFF's stored cases under root."""
    global REF, CASES
    REF = Path(root).resolve()
    if not (REF / "src" / "feffgpu" / "stage.py").exists():
        raise SystemExit(f"{REF} does not hold the reference's src/feffgpu")
    sys.path.insert(0, str(REF / "src"))
    CASES = {"W": REF / "tests/data/W", **{c: REF / "data/validation" / c for c in
                                           ("A000", "A009", "A014", "A018", "L000", "L001")}}


def parse_paths(fname):
    """FEFF's paths.dat: (nleg, deg, coords absorber-first (nleg, 3), ipots (nleg,)) per path."""
    lines = Path(fname).read_text().splitlines()
    out, i = [], 2
    while i < len(lines):
        if "index, nleg" not in lines[i]:
            i += 1
            continue
        w = lines[i].split()
        nleg, deg = int(w[1]), float(w[2])
        rows = [lines[i + 2 + j].split() for j in range(nleg)]
        pts = np.array([[float(v) for v in r[:3]] for r in rows])
        ip = [int(r[3]) for r in rows]
        out.append((nleg, deg, np.concatenate([np.zeros((1, 3)), pts[:-1]]), np.array([0] + ip[:-1])))
        i += 2 + nleg
    return out


def parse_chi(fname):
    rows = [l.split() for l in Path(fname).read_text().splitlines() if l.strip() and not l.startswith("#")]
    tab = np.array([[float(r[0]), float(r[1])] for r in rows if len(r) >= 2 and r[0].replace(".", "", 1).isdigit()])
    return tab[:, 0], tab[:, 1]


def ref_stage(P, iorder=2):
    from feffgpu.stage import GPUPathStage
    return GPUPathStage(P, device="cpu", dtype=torch.complex128, iorder=iorder)


def make_case(name):
    from feffgpu.pad import read_phase_pad
    from feffgpu.compare import r_factor
    d = CASES[name]
    P = read_phase_pad(str(d / "phase.pad"))
    paths = parse_paths(d / "paths.dat")
    kf, chi_feff = parse_chi(d / "chi.dat")
    if name == "W":
        kf, chi_feff = kf[:601], chi_feff[:601]
    pos = kf > 1e-9                      # the R-factor grid starts with an added k = 0 (tests/test_validation_cases.py:51)
    kf, chi_feff = kf[pos], chi_feff[pos]
    g = ref_stage(P)
    S = g.linear_matrix(kf)
    out = phase_to_arrays(P, prefix="ph_")
    chi = np.zeros(len(kf))
    with torch.no_grad():
        for nleg in sorted({p[0] for p in paths}):
            grp = [p for p in paths if p[0] == nleg]
            coords = np.stack([p[2] for p in grp])
            ipots = np.stack([p[3] for p in grp])
            deg = np.array([p[1] for p in grp])
            cc, rf = g.cchi(torch.tensor(coords, dtype=torch.float64), torch.tensor(ipots))
            chi += (torch.tensor(deg)[:, None] * g.chi_fine(cc, rf, kf, S, "feff")).sum(0).numpy()
            out[f"coords_{nleg}"] = coords
            out[f"ipots_{nleg}"] = ipots
            out[f"deg_{nleg}"] = deg
            keep = min(4, len(grp))
            out[f"ref_cchi_{nleg}"] = cc[:keep].numpy()
            out[f"ref_reff_{nleg}"] = rf[:keep].numpy()
    out["feff_k"], out["feff_chi"], out["ref_chi"] = kf, chi_feff, chi
    k0 = np.concatenate([[0.0], kf])
    z0 = lambda c: np.concatenate([[0.0], c])
    inp = (d / "feff.inp").read_text().split()
    rmax = 9.3 if name == "W" else float(inp[[w.upper() for w in inp].index("RPATH") + 1]) if "RPATH" in [w.upper() for w in inp] else 6.0
    out["rmax"] = np.asarray(rmax)
    out["R_ref_vs_feff"] = np.asarray(r_factor(k0, z0(chi_feff), z0(chi), kmin=3.0, kmax=float(min(23.0, kf.max() - 1.0)),
                                               rmin=1.0, rmax=rmax))
    np.savez_compressed(HERE / f"case_{name}.npz", **out)
    print(name, "paths", len(paths), "R(ref, FEFF) = %.2e" % out["R_ref_vs_feff"])


def lattice_walk(rng, nleg, a=3.1652, sd=0.06):
    """A path of nleg legs over first and second neighbours of a bcc lattice, atoms displaced at random (an atom met
    twice keeps its displacement; the absorber may be met again and stays at the origin)."""
    steps = np.vstack([np.array([[i, j, l] for i in (-.5, .5) for j in (-.5, .5) for l in (-.5, .5)]),
                       np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])]) * a
    while True:
        site, sites = np.zeros(3), []
        for _ in range(nleg - 1):
            site = site + steps[rng.integers(len(steps))]
            sites.append(site.copy())
        if np.linalg.norm(sites[-1]) > 1e-6:
            break
    moved, shift = [np.zeros(3)], {}
    for s in sites:
        key = tuple(np.round(s, 3))
        if np.linalg.norm(s) > 1e-6 and key not in shift:
            shift[key] = rng.normal(0, sd, 3)
        moved.append(s + shift.get(key, 0.0))
    return np.array(moved), np.array([0] + [0 if np.linalg.norm(s) < 1e-6 else 1 for s in sites])


def make_walks():
    from feffgpu.pad import read_phase_pad
    P = read_phase_pad(str(CASES["W"] / "phase.pad"))
    g = ref_stage(P)
    rng = np.random.default_rng(5)
    out = {}
    with torch.no_grad():
        for nleg in range(2, 9):
            cs, ips = zip(*[lattice_walk(rng, nleg) for _ in range(2)])
            coords, ipots = np.stack(cs), np.stack(ips)
            cc, rf = g.cchi(torch.tensor(coords), torch.tensor(ipots))
            out[f"coords_{nleg}"], out[f"ipots_{nleg}"] = coords, ipots
            out[f"ref_cchi_{nleg}"], out[f"ref_reff_{nleg}"] = cc.numpy(), rf.numpy()
    np.savez_compressed(HERE / "walks_W.npz", **out)
    print("walks_W written")


def make_grad(name, nlegs=(2, 3, 4, 5, 6), per=3, seed=11, iorder=2):
    """Reference gradients: the stage under checkpoint(use_reentrant=False) as the reference's callers use it.  With
    iorder != 2 the fixture is grad_<name>_io<iorder>.npz and also holds the reference's cchi of every path."""
    from feffgpu.pad import read_phase_pad
    from torch.utils.checkpoint import checkpoint
    P = read_phase_pad(str(CASES[name] / "phase.pad"))
    g = ref_stage(P, iorder)
    rng = np.random.default_rng(seed)
    q = np.arange(1, 401) * 0.05
    S = g.linear_matrix(q)
    w = torch.tensor(rng.normal(0, 1, len(q)) * q ** 2 / 100.0)
    out = {"q": q, "w": w.numpy()}
    src = parse_paths(CASES[name] / "paths.dat")
    for nleg in nlegs:
        grp = [p for p in src if p[0] == nleg][:per]
        if not grp:
            continue
        coords = np.stack([p[2] for p in grp]) + rng.normal(0, 0.02, (len(grp), nleg, 3)) * (np.arange(nleg) > 0)[None, :, None]
        ipots = np.stack([p[3] for p in grp])
        deg = np.array([p[1] for p in grp])
        x = torch.tensor(coords, requires_grad=True)

        def f(c):
            cc, rf = g.cchi(c, torch.tensor(ipots))
            return g.chi_fine(cc, rf, q, S, "feff")

        chi = checkpoint(f, x, use_reentrant=False)
        loss = (torch.tensor(deg)[:, None] * chi * w[None]).sum()
        (gx,) = torch.autograd.grad(loss, x)
        out[f"coords_{nleg}"], out[f"ipots_{nleg}"], out[f"deg_{nleg}"] = coords, ipots, deg
        out[f"grad_{nleg}"], out[f"loss_{nleg}"] = gx.numpy(), np.asarray(float(loss.detach()))
        if iorder != 2:
            with torch.no_grad():
                out[f"cchi_{nleg}"] = g.cchi(torch.tensor(coords), torch.tensor(ipots))[0].numpy()
    out.update(phase_to_arrays(P, prefix="ph_"))
    out["iorder"] = np.asarray(iorder)
    tag = name if iorder == 2 else f"{name}_io{iorder}"
    np.savez_compressed(HERE / f"grad_{tag}.npz", **out)
    print(f"grad_{tag} written")


def make_grad_walks():
    """Reference gradients of the 2-8-leg walks (W phases), loss sum_q w_q chi(q), seeded w: includes paths that
    revisit an atom (A -> B -> A), where the Euler angles are not differentiable and the reference's branch
    choices define the gradient."""
    from feffgpu.pad import read_phase_pad
    from torch.utils.checkpoint import checkpoint
    P = read_phase_pad(str(CASES["W"] / "phase.pad"))
    g = ref_stage(P)
    z = np.load(HERE / "walks_W.npz")
    q = np.arange(1, 401) * 0.05
    S = g.linear_matrix(q)
    w = torch.tensor(np.random.default_rng(2).normal(size=len(q)) * q ** 2)
    out = {"q": q, "w": w.numpy()}
    for nleg in range(2, 9):
        x = torch.tensor(z[f"coords_{nleg}"], requires_grad=True)
        ip = torch.tensor(z[f"ipots_{nleg}"])

        def f(c):
            cc, rf = g.cchi(c, ip)
            return g.chi_fine(cc, rf, q, S)

        loss = (checkpoint(f, x, use_reentrant=False) * w[None]).sum()
        (gx,) = torch.autograd.grad(loss, x)
        out[f"grad_{nleg}"] = gx.numpy()
    np.savez_compressed(HERE / "grad_walks_W.npz", **out)
    print("grad_walks_W written")


def _write_inp(path, title, edge, potentials, atoms, extra=""):
    lines = [f"TITLE {title}", "CONTROL 1 1 1 1 1 1", "PRINT 0 0 0 0 0 0", f"EDGE {edge}", "S02 1.0", extra, "",
             "POTENTIALS"]
    lines += [f"  {ip:4d} {z:4d}  {lab}" for ip, z, lab in potentials]
    lines += ["", "ATOMS"]
    lines += [f"  {x:12.6f} {y:12.6f} {z:12.6f}  {ip:d}" for (x, y, z), ip in atoms]
    lines += ["END", ""]
    Path(path).write_text("\n".join(lines))


def make_cfg1(tmp):
    """Cu fcc, a = 3.61 A, 6 A cluster, K edge, reference chain with its defaults (NLEG 4)."""
    from feffgpu.chain import run
    pts = W.fcc_cluster(3.61, 6.0)
    inp = Path(tmp) / "cu_feff.inp"
    _write_inp(inp, "Cu fcc a=3.61 cluster 6 A", "K", [(0, 29, "Cu"), (1, 29, "Cu")],
               [(p, 0 if i == 0 else 1) for i, p in enumerate(pts)], "NLEG 4\nRPATH 6.0")
    kf = np.arange(401) * 0.05
    t = time.time()
    res = run(str(inp), device="cpu", kgrid=kf)
    out = phase_to_arrays(res["phase"], prefix="ph_")
    for nleg, (coords, ipots, deg, xp, atoms) in res["kept"].items():
        if coords.shape[0] == 0:
            continue
        out[f"coords_{nleg}"] = coords.cpu().numpy().astype(np.float64)
        out[f"ipots_{nleg}"] = ipots.cpu().numpy()
        out[f"deg_{nleg}"] = deg.cpu().numpy().astype(np.float64)
    out["k"], out["ref_chi"] = kf, np.asarray(res["chi"])
    out["natoms"] = np.asarray(len(pts))
    np.savez_compressed(HERE / "cfg1_cu.npz", **out)
    print("cfg1_cu: %d atoms, paths %s, %.1f s" % (len(pts), {k: int(v[0].shape[0]) for k, v in res["kept"].items()},
                                                   time.time() - t))


def make_cfg2(tmp):
    """Fe/O/Pt phases (lmax 24) of a 6 A cluster cut around the central Fe of the seeded packing."""
    from feffgpu.chain import run
    pos, lab, box = W.random_packing(3000, 0.08, 1.8, seed=2024)
    ab = int(W.central_atom(pos, box, lab, "Fe", 1)[0])
    rel = pos - pos[ab]
    rel -= box * np.round(rel / box)
    r = np.linalg.norm(rel, axis=1)
    sel = np.argsort(r, kind="stable")
    sel = sel[r[sel] <= 6.0]
    ipmap = {"Fe": 1, "O": 2, "Pt": 3}
    atoms = [(rel[i], 0 if i == ab else ipmap[lab[i]]) for i in sel]
    inp = Path(tmp) / "feopt_feff.inp"
    _write_inp(inp, "Fe/O/Pt random packing, Fe K edge", "K", [(0, 26, "Fe"), (1, 26, "Fe"), (2, 8, "O"), (3, 78, "Pt")],
               atoms, "NLEG 2\nRPATH 2.0\nEXAFS 20.5")
    t = time.time()
    res = run(str(inp), device="cpu", lmax_override=24)
    P = res["phase"]
    np.savez_compressed(HERE / "cfg2_phase.npz", **phase_to_arrays(P, prefix="ph_"))
    print("cfg2_phase: %d atoms in the cluster, ne1 %d, lmax %d, %.1f s" % (len(sel), P.ne1, P.lmax[:P.ne1].max(),
                                                                           time.time() - t))
    # the reference stage on the resampled tables, for a sample of synthetic paths of every leg count
    Q = resample_phase(phase_from_npz(np.load(HERE / "cfg2_phase.npz"), prefix="ph_"), np.arange(401) * 0.05)
    g = ref_stage(Q)
    ipot_of = np.array([ipmap[x] for x in lab])
    paths = W.random_paths(pos, box, ab, {n: 3 for n in range(2, 9)}, rmax=8.0, seed=7, ipot_of=ipot_of)
    out = {}
    with torch.no_grad():
        for nleg, (coords, ipots, _) in paths.items():
            cc, rf = g.cchi(torch.tensor(coords), torch.tensor(ipots))
            out[f"coords_{nleg}"], out[f"ipots_{nleg}"] = coords, ipots
            out[f"ref_cchi_{nleg}"], out[f"ref_reff_{nleg}"] = cc.numpy(), rf.numpy()
    np.savez_compressed(HERE / "cfg2_sample.npz", **out)
    print("cfg2_sample written")


def _cluster_phase(name, pts, labels, center, edge_sym, pots, lmax=None):
    """Phase tables of a cluster cut (6 A) around `center` through the reference chain (NLEG 2, short RPATH)."""
    from feffgpu.chain import run
    import tempfile
    rel = pts - pts[center]
    r = np.linalg.norm(rel, axis=1)
    sel = np.argsort(r, kind="stable")
    sel = sel[r[sel] <= 6.0]
    ipmap = {lab: i + 1 for i, (_, _, lab) in enumerate(pots[1:])}
    atoms = [(rel[i], 0 if i == center else ipmap[labels[i]]) for i in sel]
    with tempfile.TemporaryDirectory() as tmp:
        inp = Path(tmp) / "feff.inp"
        _write_inp(inp, name, edge_sym, pots, atoms, "NLEG 2\nRPATH 2.0\nEXAFS 20.5")
        t = time.time()
        res = run(str(inp), device="cpu", lmax_override=lmax)
    P = res["phase"]
    np.savez_compressed(HERE / f"{name}.npz", **phase_to_arrays(P, prefix="ph_"))
    print(f"{name}: {len(sel)} atoms, ne1 {P.ne1}, lmax {P.lmax[:P.ne1].max()}, {time.time() - t:.1f} s")


def make_cfg45():
    """bcc Fe (the MD batch) and rock-salt NiO with Ni K and O K edges (the two-edge refinement)."""
    pts, box = W.bcc_supercell(6, 2.87)
    c = int(W.central_atom(pts, box, None, None, 1)[0])
    _cluster_phase("cfg4_fe_phase", pts, np.array(["Fe"] * len(pts)), c, "K", [(0, 26, "Fe"), (1, 26, "Fe")])
    pts, lab, box = W.rock_salt_supercell(4, 4.177)
    ni = int(W.central_atom(pts, box, lab, "Ni", 1)[0])
    o = int(W.central_atom(pts, box, lab, "O", 1)[0])
    _cluster_phase("cfg5_nik_phase", pts, lab, ni, "K", [(0, 28, "Ni"), (1, 28, "Ni"), (2, 8, "O")])
    _cluster_phase("cfg5_ok_phase", pts, lab, o, "K", [(0, 8, "O"), (1, 28, "Ni"), (2, 8, "O")])


FINDER_CASES = {
    # name: (structure, phase fixture, absorber species, rmax, nlegmax, critpw list)
    "cu": ("fcc", "cfg1_cu", None, 6.0, 4, (0.0, 2.5)),
    "pack": ("pack", "cfg2_phase", "Fe", 6.5, 7, (0.0, 1.0)),
    "bcc": ("bcc", "cfg4_fe_phase", None, 5.5, 3, (0.0, 2.0)),
    "tri": ("tri", "cfg4_fe_phase", None, 5.0, 4, (0.0, 2.0)),
    # edge cases of the enumeration: no candidate, one candidate (single scattering only), two candidates, a packing
    # whose 600 atoms span several blocks of the one-absorber candidate scan, and single scattering alone
    "lone": ("lone", "cfg4_fe_phase", None, 5.0, 4, (0.0,)),
    "one": ("one", "cfg4_fe_phase", None, 5.0, 4, (0.0, 2.0)),
    "two": ("two", "cfg4_fe_phase", None, 5.0, 5, (0.0, 2.0)),
    "blk": ("blk", "cfg2_phase", "Fe", 5.0, 3, (0.0, 2.0)),
    "ss": ("blk", "cfg2_phase", "Fe", 5.0, 2, (0.0, 2.0)),
}

# triclinic cells of the fixtures: a cubic supercell of edge L sheared to these lattice vectors (rows, units of L)
SHEAR = np.array([[1.0, 0.0, 0.0], [0.21, 1.0, 0.0], [0.13, -0.17, 1.0]])


def sheared(pos, L):
    """Positions and the 3 x 3 cell (rows) of a cubic supercell of edge L sheared by SHEAR."""
    cell = L * SHEAR
    return (np.asarray(pos, float) / L) @ cell, cell


def finder_structure(kind):
    """Positions (n, 3) A, cubic box or None, absorber index, potential index per atom of a finder fixture."""
    if kind == "fcc":
        pts = W.fcc_cluster(3.61, 6.0)
        return pts, None, 0, np.ones(len(pts), int)
    if kind == "pack":
        pos, lab, box = W.random_packing(400, 0.08, 1.8, seed=77)
        ab = int(W.central_atom(pos, box, lab, "Fe", 1)[0])
        return pos, box, ab, np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    if kind == "lone":
        return np.zeros((1, 3)), None, 0, np.ones(1, int)
    if kind == "one":
        pts = np.array([[0.0, 0.0, 0.0], [2.5, 0.1, -0.2], [20.0, 0.0, 0.0]])
        return pts, None, 0, np.ones(3, int)
    if kind == "two":
        pts = np.array([[0.0, 0.0, 0.0], [2.5, 0.1, -0.2], [0.3, 2.6, 0.1], [20.0, 0.0, 0.0]])
        return pts, None, 0, np.ones(4, int)
    if kind == "blk":
        pos, lab, box = W.random_packing(600, 0.08, 1.8, seed=91)
        ab = int(W.central_atom(pos, box, lab, "Fe", 1)[0])
        return pos, box, ab, np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    if kind == "tri":
        base, L = W.bcc_supercell(6, 2.87)
        pos, cell = sheared(base, L)
        pos = W.thermal(pos, 0.08, seed=4)
        return pos, cell, 0, np.ones(len(pos), int)
    base, box = W.bcc_supercell(6, 2.87)
    pos = W.thermal(base, 0.08, seed=3)
    return pos, box, int(W.central_atom(pos, box, None, None, 1)[0]), np.ones(len(pos), int)


def make_finder(names=None):
    """finder_<name>.npz -- the reference's GPUPathFinder (src/feffgpu/pathfinder.py) run on the CPU: the structure,
    parameters, and per importance cut the kept paths' atoms, degeneracies and importances, and the reference
    importance.  The phase tables are those of the named fixture."""
    from feffgpu.pathfinder import GPUPathFinder
    for name, (kind, phase_name, _sp, rmax, nlegmax, crits) in FINDER_CASES.items():
        if names is not None and name not in names:
            continue
        P = phase_from_npz(np.load(HERE / f"{phase_name}.npz"), prefix="ph_")
        pos, box, ab, ipot = finder_structure(kind)
        cellbox = box is not None and np.ndim(box) == 2
        out = {"pos": pos, "box": np.asarray(-1.0 if box is None or cellbox else box), "absorber": np.asarray(ab),
               "ipot": ipot, "rmax": np.asarray(rmax), "nlegmax": np.asarray(nlegmax), "crit": np.asarray(crits)}
        if cellbox:
            out["cell"] = np.asarray(box)
        t = time.time()
        for ci, crit in enumerate(crits):
            f = GPUPathFinder(P, device="cpu", rmax=rmax, nlegmax=nlegmax, critpw=crit)
            kept, ref = f.enumerate(pos, box, ab, ipot)
            out[f"ref_{ci}"] = np.asarray(ref)
            for nleg, (coords, ipots, deg, xp, atoms) in kept.items():
                out[f"atoms_{ci}_{nleg}"] = atoms.cpu().numpy()
                out[f"deg_{ci}_{nleg}"] = deg.cpu().numpy()
                out[f"xport_{ci}_{nleg}"] = xp.cpu().numpy()
            print(f"finder_{name} critpw {crit}: " + str({k: int(v[0].shape[0]) for k, v in kept.items()}))
        np.savez_compressed(HERE / f"finder_{name}.npz", **out)
        print(f"finder_{name}: {time.time() - t:.1f} s")


def make_geometry(seed=5):
    """geometry_ref.npz -- the reference stage's geometry (stage.py:170-206) of 2-8-leg paths in bohr: random paths,
    and the degenerate cases its branch choices define (a leg along z, collinear atoms, a revisit), per leg count the
    coordinates, ri, beta, eta and the gradient of sum(w_r ri + w_b beta + w_e eta) by its autograd."""
    from feffgpu.pad import BOHR
    g = ref_stage(phase_from_npz(np.load(HERE / "cfg1_cu.npz"), prefix="ph_"))
    rng = np.random.default_rng(seed)
    out = {}
    for nleg in range(2, 9):
        c = np.concatenate([np.zeros((6, 1, 3)), rng.normal(0, 2.0, (6, nleg - 1, 3))], 1) / BOHR
        if nleg == 3:
            c[0, 1] = [0.0, 0.0, 4.0]                     # first leg along z
            c[1, 1], c[1, 2] = [2.0, 0.0, 0.0], [4.5, 0.0, 0.0]   # collinear atoms
        if nleg == 4:
            c[0, 3] = c[0, 1]                             # a revisit: A -> B -> C -> B
        x = torch.tensor(c, requires_grad=True)
        ri, beta, eta = g.geometry(x)
        w = [torch.tensor(rng.normal(size=(6, nleg))) for _ in range(3)]
        loss = (w[0] * ri + w[1] * beta + w[2] * eta).sum()
        (gx,) = torch.autograd.grad(loss, x)
        out[f"coords_{nleg}"] = c
        out[f"ri_{nleg}"], out[f"beta_{nleg}"], out[f"eta_{nleg}"] = (t.detach().numpy() for t in (ri, beta, eta))
        out[f"wr_{nleg}"], out[f"wb_{nleg}"], out[f"we_{nleg}"] = (t.numpy() for t in w)
        out[f"grad_{nleg}"] = gx.numpy()
    np.savez_compressed(HERE / "geometry_ref.npz", **out)
    print("geometry_ref written")


def make_finder_feopt():
    """finder_feopt.npz -- the reference's path finder on the benchmark structure (the seeded 3000-atom Fe/O/Pt
    packing of feffgpu_b200.workloads, its two most central Fe absorbers, rmax 8 A, 8 legs, no importance cut): per
    absorber and leg count the number of paths, the SHA-256 of the atom sequences (int64, in the finder's order),
    the degeneracy sum and the first and last 16 sequences."""
    import hashlib
    from feffgpu.pathfinder import GPUPathFinder
    P = phase_from_npz(np.load(HERE / "cfg2_phase.npz"), prefix="ph_")
    pos, lab, box = W.random_packing(3000, 0.08, 1.8, seed=2024)
    ipot = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    abs2 = W.central_atom(pos, box, lab, "Fe", 2)
    out = {"absorbers": np.asarray(abs2)}
    t = time.time()
    f = GPUPathFinder(P, device="cpu", rmax=8.0, nlegmax=8, critpw=0.0)
    for s, ab in enumerate(abs2):
        kept, ref = f.enumerate(pos, box, int(ab), ipot)
        out[f"ref_{s}"] = np.asarray(ref)
        for nleg, (coords, ipots, deg, xp, atoms) in kept.items():
            a = np.ascontiguousarray(atoms.cpu().numpy().astype(np.int64))
            out[f"count_{s}_{nleg}"] = np.asarray(len(a))
            out[f"sha_{s}_{nleg}"] = np.frombuffer(hashlib.sha256(a.tobytes()).digest(), np.uint8)
            out[f"degsum_{s}_{nleg}"] = np.asarray(float(deg.sum()))
            out[f"head_{s}_{nleg}"], out[f"tail_{s}_{nleg}"] = a[:16], a[-16:]
        print(f"finder_feopt absorber {int(ab)}: " + str({n: int(v[0].shape[0]) for n, v in kept.items()}))
    np.savez_compressed(HERE / "finder_feopt.npz", **out)
    print(f"finder_feopt: {time.time() - t:.1f} s")


def make_bench_sample(per=48, per_cchi=4, seed=31):
    """bench_sample.npz -- the parity gate on the benchmark's own paths: the reference finder's paths of the benchmark
    packing (two central Fe absorbers, rmax 8 A, 8 legs, no importance cut, as finder_feopt.npz), a seeded stratified
    sample of up to `per` paths of every (absorber, leg count) -- their index in the finder's output, atom sequences,
    coordinates (FP32, as the finder forms them), potentials and degeneracies -- and the reference stage's FP64 (complex128) signals on the resampled 401-k tables:
    rows (14, 401) = per (absorber, leg count) the degeneracy-weighted sum of chi_fine on q = 0.05 * arange(401)
    (the benchmark's output grid), and cchi/reff of the first `per_cchi` sampled paths of every (absorber, leg
    count)."""
    from feffgpu.pad import PhaseData as RefPhase
    from feffgpu.pathfinder import GPUPathFinder
    import dataclasses
    P0 = phase_from_npz(np.load(HERE / "cfg2_phase.npz"), prefix="ph_")
    q = np.arange(401) * 0.05
    P = resample_phase(P0, q)
    refP = RefPhase(**{f.name: getattr(P, f.name) for f in dataclasses.fields(RefPhase)})
    st = ref_stage(refP)
    S = st.linear_matrix(q)
    pos, lab, box = W.random_packing(3000, 0.08, 1.8, seed=2024)
    ipot = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    abs2 = W.central_atom(pos, box, lab, "Fe", 2)
    rng = np.random.default_rng(seed)
    f = GPUPathFinder(P0, device="cpu", rmax=8.0, nlegmax=8, critpw=0.0)
    out = {"absorbers": np.asarray(abs2), "q": q, "per": np.asarray(per), "per_cchi": np.asarray(per_cchi)}
    rows, keys = [], []
    t = time.time()
    for s_, ab in enumerate(abs2):
        kept, _ = f.enumerate(pos, box, int(ab), ipot)
        for nleg in range(2, 9):
            coords, ipots, deg, _xp, atoms = kept[nleg]
            n = int(coords.shape[0])
            idx = np.sort(rng.choice(n, size=min(per, n), replace=False))
            c = coords[idx].double()
            ip = ipots[idx].long()
            with torch.no_grad():
                cc, rf = st.cchi(c, ip)
                chi = st.chi_fine(cc, rf, q, S, "feff")
            d = deg[idx].double()
            rows.append((d[:, None] * chi).sum(0).numpy())
            keys.append((s_, nleg))
            out[f"idx_{s_}_{nleg}"] = idx.astype(np.int64)
            out[f"atoms_{s_}_{nleg}"] = atoms[idx].numpy().astype(np.int64)
            out[f"coords_{s_}_{nleg}"] = coords[idx].numpy()          # FP32, as the finder forms them
            out[f"ipots_{s_}_{nleg}"] = ipots[idx].numpy().astype(np.int64)
            out[f"deg_{s_}_{nleg}"] = d.numpy()
            out[f"count_{s_}_{nleg}"] = np.asarray(n)
            out[f"cchi_{s_}_{nleg}"] = cc[:per_cchi].numpy()
            out[f"reff_{s_}_{nleg}"] = rf[:per_cchi].numpy()
        print(f"bench_sample absorber {int(ab)}: {time.time() - t:.1f} s")
    out["rows"] = np.stack(rows)
    out["row_keys"] = np.asarray(keys, np.int64)
    np.savez_compressed(HERE / "bench_sample.npz", **out)
    print(f"bench_sample: {sum(len(out[f'idx_{a}_{n}']) for a, n in keys)} paths, {time.time() - t:.1f} s")


def make_rspace(seed=41):
    """rspace_ref.npz -- the reference's R-space loss on seeded spectra: for each window, the R-factor of model rows
    (B, 401) against data (401,) on k = 0.05 * arange(401) and its gradient with respect to the rows, (a) by
    r_factor_torch (src/feffgpu/exafs/transform.py:130-145; FP64 k and window) and (b) as PathSpectra.misfit forms it
    (exafs/forward.py:87-90, 105-110, 165-168: k and the Hanning window in FP32, widened to FP64); both take the R
    window on the FP32 R grid of transform.py:125-127.  One window's limits fall on R grid points, where the FP32 grid
    decides which points are kept."""
    from feffgpu.exafs import transform as T
    rng = np.random.default_rng(seed)
    k = T.KSTEP * np.arange(401)
    kk = k[None, :]
    data = (np.sin(2 * 2.3 * k) * np.exp(-0.01 * k ** 2) + 0.2 * np.sin(2 * 3.9 * k + 0.4) * np.exp(-0.02 * k ** 2)) \
        / np.maximum(k, 0.5)
    models = data[None] * (1 + 0.05 * rng.normal(size=(3, 1))) + 0.01 * rng.normal(size=(3, 401)) * np.exp(-kk / 8)
    windows = [T.FitWindow(3.0, 14.0, 1.0, 2, 1.0, 6.0), T.FitWindow(2.0, 18.0, 0.5, 3, 1.2, 5.0),
               T.FitWindow(3.0, 14.0, 1.0, 1, 25 * T.RSTEP, 150 * T.RSTEP)]
    out = {"k": k, "data": data, "models": models}
    for i, w in enumerate(windows):
        out[f"win_{i}"] = np.array([w.kmin, w.kmax, w.dk, w.kweight, w.rmin, w.rmax])
        m = torch.tensor(models, dtype=torch.float64, requires_grad=True)
        R = T.r_factor_torch(m, torch.tensor(data), torch.tensor(k), w)
        R.sum().backward()
        out[f"R_{i}"], out[f"grad_{i}"] = R.detach().numpy(), m.grad.numpy()
        r = T.r_grid()
        out[f"keep_{i}"] = np.nonzero(((r >= w.rmin) & (r <= w.rmax)).numpy())[0]
        # PathSpectra.misfit's forms: FP32 k and window, FP64 transform
        kt = torch.tensor(k, dtype=torch.float32)
        win = T.hanning_window(kt, torch.tensor([w.kmin]), torch.tensor([w.kmax]), dk=w.dk)
        keep = (r >= w.rmin) & (r <= w.rmax)
        tr = T.ft(torch.tensor(data)[None], kt.double(), win.double(), kweight=w.kweight)[0][keep]
        Rs, gs = [], []
        for b in range(models.shape[0]):
            x = torch.tensor(models[b], dtype=torch.float64, requires_grad=True)
            cr = T.ft(x[None], kt.double(), win.double(), kweight=w.kweight)[0][keep]
            v = ((cr - tr).abs() ** 2).sum() / float((tr.abs() ** 2).sum())
            v.backward()
            Rs.append(float(v.detach()))
            gs.append(x.grad.numpy())
        out[f"R32_{i}"], out[f"grad32_{i}"] = np.asarray(Rs), np.stack(gs)
    np.savez_compressed(HERE / "rspace_ref.npz", **out)
    print(f"rspace_ref: {len(windows)} windows")


def make_cfg3(n_absorbers=16, seed=31):
    """cfg3_adjoint.npz -- configuration 3 through the reference's own forward model: a seeded 800-atom Fe/O/Pt
    packing (feffgpu_b200.workloads, seed 31), its 16 most central Fe absorbers, the reference's PathSpectra
    (src/feffgpu/exafs/forward.py:33-176: its path finder, rmax 5 A, 4 legs, its default importance cut 0.5 %; its
    stage in complex128 on the CPU; chunks through non-reentrant checkpointing) on the Fe K tables resampled to 401 k;
    the target is its spectrum of the same path lists at positions displaced by seeded Gaussian noise (sigma 0.05 A);
    the loss its R-space misfit (k 3-16, R 1-6, kw 2) and the gradient of the loss with respect to every position
    by its autograd.  Stored: positions, box, absorbers, potentials, path counts per leg count, target, loss and the
    (800, 3) gradient."""
    import dataclasses
    from feffgpu.exafs.forward import PathSpectra
    from feffgpu.pad import PhaseData as RefPhase
    q = np.arange(401) * 0.05
    P = resample_phase(phase_from_npz(np.load(HERE / "cfg2_phase.npz"), prefix="ph_"), q)
    refP = RefPhase(**{f.name: getattr(P, f.name) for f in dataclasses.fields(RefPhase)})
    pos, lab, box = W.random_packing(800, 0.08, 1.8, seed=seed)
    ipot = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    absorbers = np.asarray(W.central_atom(pos, box, lab, "Fe", n_absorbers))
    t = time.time()
    ps = PathSpectra(refP, q, np.zeros(401), 0.0, window=(3.0, 16.0), r_range=(1.0, 6.0), box=box, rmax=5.0,
                     nlegmax=4, critpw=0.5, device="cpu", dtype=torch.complex128)
    counts = ps.refresh(pos[None], absorbers[None], ipot=torch.tensor(ipot))
    target_pos = W.thermal(pos, 0.05, seed=77)
    with torch.no_grad():
        target = ps.spectra(torch.tensor(target_pos, dtype=torch.float64).reshape(-1, 3), use_checkpoint=False)[0]
    ps.set_target(target.numpy())
    x = torch.tensor(pos, dtype=torch.float64).reshape(-1, 3).requires_grad_(True)
    loss = ps.misfit(ps.spectra(x).mean(0))
    loss.backward()
    np.savez_compressed(HERE / "cfg3_adjoint.npz", pos=pos, box=np.asarray(box), absorbers=absorbers, ipot=ipot,
                        legs=np.asarray(sorted(counts)), counts=np.asarray([counts[n] for n in sorted(counts)]),
                        target=target.numpy(), target_pos=target_pos, loss=np.asarray(float(loss.detach())),
                        grad=x.grad.numpy().reshape(-1, 3), q=q)
    print(f"cfg3_adjoint: {counts}, loss {float(loss.detach()):.4e}, {time.time() - t:.1f} s")


def make_pairs():
    """pairs_nio.npz -- the reference's single-scattering pair tables (src/feffgpu/exafs/forward.py:178-320) on the
    CPU in FP64: a thermally displaced rock-salt NiO supercell (3^3 cells, 216 sites, sigma 0.1 A, periodic), Ni K
    edge tables on r = 1.5..5 A step 0.02 for k = 0..20 step 0.05, every 25th table row, the histogram of four
    absorbers, the all-pairs single-scattering spectrum of two copies and the gradient of sum_k w_k chi_k with
    respect to the positions (seeded w)."""
    from feffgpu.exafs.forward import PairTables
    P = phase_from_npz(np.load(HERE / "cfg5_nik_phase.npz"), prefix="ph_")
    pos0, lab, box = W.rock_salt_supercell(3, 4.177)
    pos = np.stack([W.thermal(pos0, 0.1, seed=21), W.thermal(pos0, 0.1, seed=22)])
    ipot = np.array([{"Ni": 1, "O": 2}[x] for x in lab])
    k = np.arange(401) * 0.05
    t = time.time()
    pt = PairTables(P, k, np.zeros(len(k)), 0.0, box=box, rmax=5.0, r_min=1.5, dr=0.02, ms=False, device="cpu",
                    dtype=torch.complex128)
    pt.ipot = torch.tensor(ipot)
    out = {"pos": pos, "box": np.asarray(box), "ipot": ipot, "k": k, "rmax": np.asarray(5.0), "r_min": np.asarray(1.5),
           "dr": np.asarray(0.02), "nr": np.asarray(pt.nr)}
    for ip, tab in pt.tables.items():
        out[f"table_{ip}"] = tab.double().numpy()[::25]
    absorbers = np.array([0, 7, 100, 150])
    hist, short = pt.histogram(torch.tensor(pos[0]), torch.tensor(absorbers), torch.tensor(ipot), box=float(box))
    out["absorbers"], out["hist"], out["short"] = absorbers, hist.numpy(), np.asarray(short)
    x = torch.tensor(pos, dtype=torch.float32, requires_grad=True)        # the tables are FP32 (forward.py:237)
    chi = pt.single_scattering(x)
    w = torch.tensor(np.random.default_rng(3).normal(size=len(k)))
    (chi.double() * w).sum().backward()
    out["chi"], out["w"], out["grad"] = chi.detach().double().numpy(), w.numpy(), x.grad.numpy()
    np.savez_compressed(HERE / "pairs_nio.npz", **out)
    print(f"pairs_nio: nr {pt.nr}, {time.time() - t:.1f} s")


def make_pairs_cell():
    """pairs_nio_tri.npz -- as pairs_nio.npz on a triclinic cell: the NiO supercell (3^3 cells) sheared by SHEAR,
    thermally displaced (sigma 0.1 A), the reference's PairTables given the 3 x 3 cell."""
    from feffgpu.exafs.forward import PairTables
    P = phase_from_npz(np.load(HERE / "cfg5_nik_phase.npz"), prefix="ph_")
    pos0, lab, L = W.rock_salt_supercell(3, 4.177)
    pos0, cell = sheared(pos0, L)
    pos = np.stack([W.thermal(pos0, 0.1, seed=31), W.thermal(pos0, 0.1, seed=32)])
    ipot = np.array([{"Ni": 1, "O": 2}[x] for x in lab])
    k = np.arange(401) * 0.05
    t = time.time()
    pt = PairTables(P, k, np.zeros(len(k)), 0.0, box=cell, rmax=5.0, r_min=1.5, dr=0.02, ms=False, device="cpu",
                    dtype=torch.complex128)
    pt.ipot = torch.tensor(ipot)
    out = {"pos": pos, "cell": cell, "ipot": ipot, "k": k, "rmax": np.asarray(5.0), "r_min": np.asarray(1.5),
           "dr": np.asarray(0.02), "nr": np.asarray(pt.nr)}
    absorbers = np.array([0, 7, 100, 150])
    hist, short = pt.histogram(torch.tensor(pos[0]), torch.tensor(absorbers), torch.tensor(ipot), box=torch.tensor(cell))
    out["absorbers"], out["hist"], out["short"] = absorbers, hist.numpy(), np.asarray(short)
    x = torch.tensor(pos, dtype=torch.float32, requires_grad=True)
    chi = pt.single_scattering(x)
    w = torch.tensor(np.random.default_rng(3).normal(size=len(k)))
    (chi.double() * w).sum().backward()
    out["chi"], out["w"], out["grad"] = chi.detach().double().numpy(), w.numpy(), x.grad.numpy()
    np.savez_compressed(HERE / "pairs_nio_tri.npz", **out)
    print(f"pairs_nio_tri: nr {pt.nr}, {time.time() - t:.1f} s")


def make_larch():
    """larch_W.npz -- the reference stage's cubic-spline ("larch") fine grid on the W case: its spline_matrix
    (src/feffgpu/stage.py:341-351) for q = 0..20 1/A step 0.05 and chi_fine(..., "larch") of the stored paths' cchi."""
    from feffgpu.pad import read_phase_pad
    P = read_phase_pad(str(CASES["W"] / "phase.pad"))
    g = ref_stage(P)
    z = np.load(HERE / "case_W.npz")
    q = np.arange(401) * 0.05
    S = g.spline_matrix(q)
    out = {"q": q, "S": S.numpy()}
    for nleg in (2, 3, 4):
        cc = torch.tensor(z[f"ref_cchi_{nleg}"])
        rf = torch.tensor(z[f"ref_reff_{nleg}"])
        out[f"chi_{nleg}"] = g.chi_fine(cc, rf, q, S, "larch").numpy()
    np.savez_compressed(HERE / "larch_W.npz", **out)
    print("larch_W written")


def make_feffdat():
    """feffdat_W.npz -- FEFF's own per-path column files feff0001..0008.dat of the W case (tests/data/W): each path's
    geometry (absorber first), potentials, degeneracy and reff from the file header, and its seven columns (k,
    real[2*phc], mag[feff], phase[feff], red factor, lambda, real[p]) as FEFF printed them."""
    out = {}
    for i in range(1, 9):
        lines = (CASES["W"] / f"feff{i:04d}.dat").read_text().splitlines()
        h = next(j for j, l in enumerate(lines) if "nleg, deg, reff" in l)
        nleg, deg, reff = (float(v) for v in lines[h].split()[:3])
        nleg = int(nleg)
        atoms = [lines[h + 2 + a].split() for a in range(nleg)]
        coords = np.array([[float(v) for v in a[:3]] for a in atoms])
        ipots = np.array([int(a[3]) for a in atoms])
        t = next(j for j, l in enumerate(lines) if l.strip().startswith("k ") and "real[2*phc]" in l)
        cols = np.array([[float(v) for v in l.split()] for l in lines[t + 1:] if l.strip()])
        out[f"coords_{i}"], out[f"ipots_{i}"] = coords, ipots
        out[f"deg_{i}"], out[f"reff_{i}"], out[f"cols_{i}"] = np.asarray(deg), np.asarray(reff), cols
    np.savez_compressed(HERE / "feffdat_W.npz", **out)
    print("feffdat_W: 8 paths")


def main():
    import tempfile
    ap = argparse.ArgumentParser()
    ap.add_argument("reference", help="root of the reference's source tree (the directory holding src/feffgpu)")
    ap.add_argument("--only", nargs="*")
    args = ap.parse_args()
    set_reference(args.reference)
    want = set(args.only or ["cases", "walks", "grad", "cfg1", "cfg2", "cfg45", "finder", "finder_tri",
                             "finder_edges", "pairs", "pairs_tri", "feffdat", "larch", "bench_sample", "rspace", "cfg3",
                             "iorder", "geometry"])
    with tempfile.TemporaryDirectory() as tmp:
        if "cases" in want:
            import shutil
            shutil.copyfile(CASES["L001"] / "phase.pad", HERE / "L001_phase.pad")
            for name in CASES:
                make_case(name)
        if "walks" in want:
            make_walks()
        if "grad" in want:
            make_grad_walks()
            make_grad("L001")
            make_grad("A000", nlegs=(2, 3, 4), per=2)
            make_grad("A014", nlegs=(2, 3, 4, 5), per=2)     # L3 edge: the adjoint's second initial-state class
            make_grad("A009", nlegs=(2, 3, 4, 5), per=2)     # M5 edge: the third
        if "cfg1" in want:
            make_cfg1(tmp)
        if "cfg2" in want:
            make_cfg2(tmp)
        if "cfg45" in want:
            make_cfg45()
        if "finder" in want:
            make_finder()
            make_finder_feopt()
        if "finder_tri" in want:
            make_finder(["tri"])
        if "geometry" in want:
            make_geometry()
        if "iorder" in want:
            for io in (0, 1, 3):
                make_grad("L001", nlegs=(2, 3, 4, 5), per=2, iorder=io)       # K edge
                make_grad("A014", nlegs=(2, 3, 4), per=2, iorder=io)          # L3 edge
            make_grad("A009", nlegs=(2, 3, 4), per=2, iorder=3)               # M5 edge
        if "finder_edges" in want:
            make_finder(["lone", "one", "two", "blk", "ss"])
        if "pairs" in want:
            make_pairs()
        if "pairs_tri" in want:
            make_pairs_cell()
        if "larch" in want:
            make_larch()
        if "feffdat" in want:
            make_feffdat()
        if "bench_sample" in want:
            make_bench_sample()
        if "rspace" in want:
            make_rspace()
        if "cfg3" in want:
            make_cfg3()


if __name__ == "__main__":
    main()
