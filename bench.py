"""bench.py -- throughput of the batched path stage on B200 in path·k-points/s.

Workload (one GPU): the Fe K-edge stage of a seeded random packing of 3000 atoms (Fe/O/Pt, minimum separation
1.8 A, 0.08 atoms/A^3), the two most central Fe absorbers, every path of 2-8 legs within 8 A that the path finder
returns (no importance cut; 1.89e5 paths, found by this package's CUDA path finder, identical to the reference
finder's on this structure), degeneracies included, phase tables lmax 24 of the
reference's own phase-shift stage resampled to 401 k points (0-20 1/A), output chi(k) on the same 401 points.
One step = the whole stage over that batch: geometry, rotation matrices, scattering-matrix chain, termination,
cfac, fine-grid signal and the deterministic degeneracy-weighted sum into the two absorbers' rows, in the
mixed precision form (FP32 complex chain, FP64 phase argument and sums).  Under torchrun every rank evaluates its
own two absorbers (weak scaling, no collective on the data path).

Beside the headline line's value: the end-to-end form (host buffers, copies timed), forward+backward, the plain FP64
form, the MD-EXAFS batch (bcc Fe, 500 frames x 32 absorbers in one launch) and the RMC refinement (NiO, two edges,
each step one CUDA graph replay), the path finder itself, the single-scattering pair tables and the reference's own
GPUPathStage on this GPU and on the host cores (when it is installed under baseline/_ref), each in its own key of the
JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --frontends      # the reference's MD and RMC front ends, its classes vs install()

--impl reference times the reference's path stage on the CPU (the FP64 oracle port of its algorithm with all host
threads) on a bounded stratified sample of the same workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NK = 401
Q = np.arange(NK) * 0.05
METRIC = "path·k-points/s fwd and fwd+bwd vs plain FP64 on same B200 at R<=1e-6"
UNIT = "path·k/s"


# ------------------------------------------------------------------------------------------------ workload
def packing():
    from feffgpu_b200 import workloads as W
    pos, lab, box = W.random_packing(3000, 0.08, 1.8, seed=2024)
    ipot_of = np.array([{"Fe": 1, "O": 2, "Pt": 3}[x] for x in lab])
    return pos, lab, box, ipot_of


def workload(world: int, scale: float = 1.0, finder: str = "gpu"):
    """Phase tables (resampled to 401 k) and the path groups of the job's 2 x world absorbers (the most central Fe
    atoms): every path of 2-8 legs within 8 A that the path finder returns (no importance cut), degeneracies
    included, row = absorber.  finder "gpu": this package's CUDA path finder (the paths are the reference finder's,
    bit for bit); "oracle": the CPU restatement (the reference arm, which runs nothing of this package).  scale < 1
    keeps every k-th path per leg count (profiling runs)."""
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.pad import phase_from_npz, resample_phase
    z = np.load(ROOT / "tests" / "golden" / "cfg2_phase.npz")
    P0 = phase_from_npz(z, prefix="ph_")
    P = resample_phase(P0, Q)
    pos, lab, box = packing()[:3]
    ipot_of = packing()[3]
    absorbers = W.central_atom(pos, box, lab, "Fe", 2 * world)
    groups = []
    if finder == "gpu":
        from feffgpu_b200.pathfinder import GPUPathFinder
        res = GPUPathFinder(P0, device="cuda", rmax=8.0, nlegmax=8, critpw=0.0).enumerate_many(pos, box, absorbers,
                                                                                               ipot_of)
        for nleg, (coords, ip, deg, _xp, _atoms, slot) in sorted(res["paths"].items()):
            sl = slot.cpu().numpy()
            c, i, d = coords.cpu().numpy(), ip.cpu().numpy(), deg.cpu().numpy()
            for a in range(len(absorbers)):
                sel = np.nonzero(sl == a)[0]
                groups.append((a, nleg, c[sel], i[sel], d[sel]))
    else:
        from oracle.pathfinder import Finder
        for a, ab in enumerate(absorbers):
            kept, _ = Finder(P0, rmax=8.0, nlegmax=8, critpw=0.0).enumerate(pos, box, int(ab), ipot_of)
            for nleg, (coords, ip, deg, _xp, _atoms) in sorted(kept.items()):
                groups.append((a, nleg, coords, ip, deg))
    out = []
    for a, nleg, coords, ip, deg in sorted(groups, key=lambda g: (g[0], g[1])):
        if len(coords) == 0:
            continue
        step = max(1, int(round(1.0 / scale)))
        sel = np.arange(0, len(coords), step)
        out.append((coords[sel].astype(np.float64), ip[sel], deg[sel].astype(np.float64), np.full(len(sel), a)))
    return P, out


def workload_config(groups, world: int) -> dict:
    """The job's description, built from the path groups of all its absorbers, the same on both arms."""
    legs: dict = {}
    for c, *_ in groups:
        legs[int(c.shape[1])] = legs.get(int(c.shape[1]), 0) + len(c)
    n_paths = sum(legs.values())
    return {"workload": f"Fe/O/Pt packing 3000 atoms, {2 * world} Fe K absorbers (2 per GPU), every path finder path "
                        f"of 2-8 legs to 8 A, {n_paths} paths, lmax 24 x {NK} k, chi on {NK} k",
            "paths_total": n_paths, "paths_per_gpu": n_paths // world, "nk": NK, "energies": NK,
            "legs": dict(sorted(legs.items())),
            "parallelism": f"dp{world}: the paths of all absorbers split over the GPUs by FLOP cost, rows all-reduced",
            "l2": "GPU arm: flushed between timed steps (256 MB write)"}


def finder_leg(args, dev, world, rank):
    """The path finder itself: every path of 2-8 legs within 8 A of this rank's two absorbers (no importance cut),
    both absorbers in one batched call, timed with CUDA events after one warm-up call."""
    import torch
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.pad import phase_from_npz
    from feffgpu_b200.pathfinder import GPUPathFinder
    P0 = phase_from_npz(np.load(ROOT / "tests" / "golden" / "cfg2_phase.npz"), prefix="ph_")
    pos, lab, box, ipot_of = packing()
    absorbers = W.central_atom(pos, box, lab, "Fe", 2 * world)[2 * rank:2 * rank + 2]     # this GPU's two
    f = GPUPathFinder(P0, device=dev, rmax=8.0, nlegmax=8, critpw=0.0)
    res = f.enumerate_many(pos, box, absorbers, ipot_of)
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = f.enumerate_many(pos, box, absorbers, ipot_of)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    n = sum(int(v[0].shape[0]) for v in res["paths"].values())
    t = float(np.median(ms))
    out = {"ms": t, "paths": n, "paths_per_s": n / (t * 1e-3), "absorbers": len(absorbers),
           "legs": {int(k): int(v[0].shape[0]) for k, v in sorted(res["paths"].items())},
           "note": "enumeration, geometry, importance, merges; identical paths to the reference finder"}
    if rank == 0 and not args.no_cpu:
        # the CPU restatement of the reference finder (numpy, one host thread) on the same absorbers
        import time as _time
        from oracle.pathfinder import Finder
        t0 = _time.perf_counter()
        fo = Finder(P0, rmax=8.0, nlegmax=8, critpw=0.0)
        for a in absorbers:
            fo.enumerate(pos, box, int(a), ipot_of)
        out["cpu_oracle_ms"] = (_time.perf_counter() - t0) * 1e3
    return out


# ------------------------------------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi samples of the GPU's clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid, self.proc, self.lines = uuid, None, []

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.uuid:
            cmd.insert(1, f"--id={self.uuid}")
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for l in self.lines:
            p = [v.strip() for v in l.split(",")]
            if len(p) < 8:
                continue
            try:
                rows.append((float(p[0]), float(p[1]), float(p[2]), p[3], p[4], p[5], p[6], p[7]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r[2] > 200.0] or rows
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in load for n, v in zip(names, r[4:]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in load])), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(load), "reasons": reasons}


# ------------------------------------------------------------------------------------------------ CPU legs
def cpu_sample(P, groups, budget_s: float, nthreads: int):
    """The oracle (FP64, C, pthreads) on a stratified sample of every leg count, extrapolated to the workload:
    cchi of the sampled paths, their fine-grid signal and sum.  Returns (path·k/s, description, samples) with
    samples {nleg: (coords, ipots, chi summed over the sampled paths)} for the parity check."""
    from oracle import oracle as O
    orc = O.Oracle(P)
    S = orc.linear_matrix(Q)
    by_leg: dict = {}
    for c, ip, _deg, _row in groups:
        by_leg.setdefault(c.shape[1], []).append((c, ip))
    counts = {n: sum(len(c) for c, _ in v) for n, v in by_leg.items()}
    rng = np.random.default_rng(0)

    def run(n, m):
        c = np.concatenate([x[0] for x in by_leg[n]])
        ip = np.concatenate([x[1] for x in by_leg[n]])
        sel = rng.choice(len(c), size=min(m, len(c)), replace=False)
        t = time.perf_counter()
        cc, rf = orc.cchi(c[sel], ip[sel], nthreads=nthreads)
        chi = O.chi_fine(cc, rf, Q, S).sum(0)
        return (time.perf_counter() - t) / len(sel), len(sel), chi, c[sel], ip[sel]

    # calibrate with two paths per leg count, then spend the budget in proportion to each bucket's total time
    per = {n: run(n, 2)[0] for n in counts}
    full = sum(counts[n] * per[n] for n in counts)
    scale = budget_s / max(full, 1e-9)
    t_total, sampled, samples = 0.0, 0, {}
    for n in sorted(counts):
        m = max(4, int(counts[n] * scale))
        tp, got, chi, c, ip = run(n, m)
        t_total += counts[n] * tp
        sampled += got
        samples[n] = (c, ip, chi)
    n_paths = sum(counts.values())
    return n_paths * NK / t_total, f"stratified sample of {sampled} of {n_paths} paths (every leg count), " \
                                    f"timed per leg count and extrapolated to the full batch", samples


def parity_vs_oracle(P, samples, dev):
    """This package's rows of the CPU baseline's stratified sample (one row per leg count, every sampled path weight
    one) against the oracle's FP64 sums of the same paths: R-factor per leg count, mixed and FP64 forms."""
    import torch
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.rspace import FitWindow, r_factor
    win = FitWindow(kmin=3.0, kmax=19.0, rmin=1.0, rmax=8.0)
    legs = sorted(samples)
    b = PathBatch([(samples[n][0], samples[n][1], None, np.full(len(samples[n][0]), i)) for i, n in enumerate(legs)],
                  nrows=len(legs), device=dev)
    res = {"paths": b.n, "legs": {int(n): int(len(samples[n][0])) for n in legs}}
    for d, key in ((torch.complex64, "R_mixed_vs_oracle"), (torch.complex128, "R_fp64_vs_oracle")):
        with torch.no_grad():
            rows = GPUPathStage(P, device=dev, dtype=d).chi_reduce(b, Q).cpu().numpy()
        res[key] = max(r_factor(samples[n][2], rows[i], win) for i, n in enumerate(legs))
    return res


def extras(args, stage, batch, P, S, dev, timed, n_total, ms):
    """End-to-end, forward+backward and plain-FP64 measurements beside the headline, each step the same job as the
    headline's (this GPU's share of the paths, rows all-reduced over the GPUs)."""
    import torch
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200.sharded import chi_reduce_all_ranks
    # the path coordinates come from the FP32 path finder: sent as FP32 when that is exact (the stage widens them to
    # FP64 on the device, the same values), else as FP64
    c64 = batch.coords.cpu()
    c32 = c64.to(torch.float32)
    coords_h = (c32 if torch.equal(c32.to(torch.float64), c64) else c64).pin_memory()
    coords_d = torch.empty(coords_h.shape, dtype=coords_h.dtype, device=dev)
    rows_h = torch.empty(batch.nrows, NK, dtype=torch.float64).pin_memory()

    def e2e_step():
        coords_d.copy_(coords_h, non_blocking=True)
        rows = chi_reduce_all_ranks(stage, batch, Q, S, coords=coords_d)
        rows_h.copy_(rows, non_blocking=True)

    with torch.no_grad():
        ms_e2e, _ = timed(e2e_step, args.steps, 1)
    e2e = {"value": n_total * NK / (ms_e2e * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": int(coords_h.numel() * coords_h.element_size()),
           "d2h_bytes_per_step": int(rows_h.numel() * rows_h.element_size())}

    # forward + backward (gradients with respect to every path coordinate and per-path sigma^2)
    fwd_bwd = None
    try:
        s2 = torch.zeros(batch.n, dtype=torch.float64, device=dev, requires_grad=True)
        cg = batch.coords.clone().requires_grad_(True)
        w = torch.randn(batch.nrows, NK, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))

        def fb():
            rows = chi_reduce_all_ranks(stage, batch, Q, S, coords=cg, sigma2=s2)
            (rows * w).sum().backward()

        ms_fb, _ = timed(fb, max(2, args.steps // 2), 1)
        fwd_bwd = {"value": n_total * NK / (ms_fb * 1e-3), "unit": UNIT, "ms_per_step": ms_fb}
    except NotImplementedError as err:
        fwd_bwd = {"value": None, "unit": UNIT, "note": f"not available: {err}"}

    # the plain FP64 drop-in (complex128) on the same batch
    stage64 = GPUPathStage(P, device=dev, dtype=torch.complex128, autotune=not args.no_autotune)
    with torch.no_grad():
        ms64, _ = timed(lambda: chi_reduce_all_ranks(stage64, batch, Q, S), 2, 1)
    plain = {"value": n_total * NK / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64,
             "speedup_mixed_over_fp64": ms64 / ms, "launch_warps": list(stage64._launch)}

    return e2e, fwd_bwd, plain


def md_extra(args, dev, timed, world, rank):
    """MD-EXAFS batch: bcc Fe 16^3 cells (8192 atoms, a = 2.87 A), 500 seeded thermal frames (sigma 0.08 A), 32
    random absorbers per frame; the path finder (every path of up to 3 legs within 5.5 A, no importance cut) runs on
    all 16,000 frame x absorber pairs in one batched call (timed as the median of three calls after a warm-up), then
    all their paths go through one fused launch with chi averaged per frame.  Error: R-factor of each frame's mixed-precision chi against the FP64 form of the same
    batch (the FP64 form matches the oracle to R < 1e-12 in the parity tests)."""
    import torch
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.rspace import FitWindow, r_factor
    from feffgpu_b200.pad import phase_from_npz
    from feffgpu_b200.pathfinder import GPUPathFinder
    P = phase_from_npz(np.load(ROOT / "tests" / "golden" / "cfg4_fe_phase.npz"), prefix="ph_")
    frames, absorbers = args.md_frames, 32
    base, box = W.bcc_supercell(16, 2.87)
    rng = np.random.default_rng(rank)
    pos = np.stack([W.thermal(base, 0.08, seed=rank * 100003 + f + 1) for f in range(frames)]).astype(np.float32)
    abs_ = np.stack([rng.choice(len(base), size=absorbers, replace=False) for _ in range(frames)])
    finder = GPUPathFinder(P, device=dev, rmax=5.5, nlegmax=3, critpw=0.0)
    ipot = np.ones(len(base), np.int64)
    res = finder.enumerate_many(pos, box, abs_, ipot)
    torch.cuda.synchronize(dev)
    finds = []
    for _ in range(3):               # the median of three calls: the first after a warm-up can still grow the allocator
        del res
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = finder.enumerate_many(pos, box, abs_, ipot)
        e1.record()
        e1.synchronize()
        finds.append(e0.elapsed_time(e1))
    ms_find = float(np.median(finds))
    groups = []
    for nleg, (coords, ipots, deg, _xp, _atoms, slot) in sorted(res["paths"].items()):
        groups.append((coords.double(), ipots, deg.double() / absorbers, torch.div(slot, absorbers, rounding_mode="floor")))
    batch = PathBatch(groups, nrows=frames, device=dev)
    del res
    st = GPUPathStage(P, device=dev, dtype=torch.complex64, autotune=not args.no_autotune)
    S = st.linear_matrix(Q)
    with torch.no_grad():
        ms, _ = timed(lambda: st.chi_reduce(batch, Q, S), max(2, args.steps // 2), 1)
        rows = st.chi_reduce(batch, Q, S).cpu().numpy()
        st64 = GPUPathStage(P, device=dev, dtype=torch.complex128, autotune=not args.no_autotune)
        ms64, _ = timed(lambda: st64.chi_reduce(batch, Q, S), 2, 1)
        ref = st64.chi_reduce(batch, Q, S).cpu().numpy()
    win = FitWindow(kmin=3.0, kmax=19.0, rmin=1.0, rmax=5.5)
    R = [r_factor(ref[f], rows[f], win) for f in range(frames)]
    out = {"value": world * batch.n * NK / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "paths_per_gpu": batch.n,
           "frames": frames, "absorbers_per_frame": absorbers, "legs": batch.counts,
           "path_finder_ms": ms_find, "fp64_ms_per_step": ms64, "r_factor_vs_fp64_max": max(R),
           "r_factor_vs_fp64_median": float(np.median(R)), "launch_warps": list(st._launch)}
    del batch
    torch.cuda.empty_cache()
    return out


def _ref_stage_class():
    """The reference's GPUPathStage and PhaseData from baseline/_ref, or (None, reason)."""
    ref = ROOT / "baseline" / "_ref"
    if not (ref / "feffgpu" / "stage.py").exists():
        return None, "reference not installed under baseline/_ref"
    sys.path.insert(0, str(ref))
    try:
        from feffgpu.pad import PhaseData as RefPhase
        from feffgpu.stage import GPUPathStage as RefStage
    except Exception as err:                                   # noqa: BLE001 - report, do not fail the bench
        return None, f"reference import failed: {err!r}"[:200]
    finally:
        sys.path.remove(str(ref))
    return (RefStage, RefPhase), ""


def reference_gpu_leg(args, P, groups, dev, ours: dict, uuid):
    """The reference's own GPUPathStage (installed unmodified under baseline/_ref) on this GPU, on a sample of the
    same batch, the way its callers run it: per leg count chunks of up to 4096 paths (src/feffgpu/chain.py:47),
    cchi -> chi_fine -> degeneracy-weighted sum into the absorber rows.  Per leg count three chunks (the first three
    of that leg count, or the same chunk again when it has fewer paths) are timed with CUDA events after a warm-up
    chunk; the median time per path is extrapolated by the paths of that leg count.  complex64 (its production
    default) and complex128 forward; complex64 forward+backward through non-reentrant checkpointing
    (src/feffgpu/exafs/forward.py:158-159) in chunks of up to 2048 paths, its PathSpectra's default chunk
    (forward.py:69).  The clocks are sampled over the leg.  ``ours`` holds this package's ms per step of the same
    batch.  Parity: the first chunk of every leg count is also evaluated by this package (mixed and FP64 forms) and
    compared with the reference's complex128 rows and per-path cchi."""
    import torch
    cls, why = _ref_stage_class()
    if cls is None:
        return {"unavailable": why}, None
    RefStage, RefPhase = cls
    import dataclasses
    from torch.utils.checkpoint import checkpoint
    refP = RefPhase(**{f.name: getattr(P, f.name) for f in dataclasses.fields(RefPhase)})
    by_leg: dict = {}
    for c, ip, deg, row in groups:
        by_leg.setdefault(c.shape[1], []).append((c, ip, deg, row))
    by_leg = {n: tuple(np.concatenate([x[i] for x in v]) for i in range(4)) for n, v in sorted(by_leg.items())}
    n_paths = sum(len(v[0]) for v in by_leg.values())
    nrows = 1 + max(int(v[3].max()) for v in by_leg.values())

    def ev_time(fn):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1), res

    keep = {}

    def arm(dtype, chunk, grad, save=False):
        stage = RefStage(refP, device=dev, dtype=dtype)
        S = stage.linear_matrix(Q)
        total, sampled, chunks = 0.0, 0, 0
        for n, (c, ip, deg, row) in by_leg.items():
            m = min(len(c), chunk)
            per_path = []
            for j in range(4):                                   # chunk 0 twice: warm-up, then timed
                lo = (max(j - 1, 0) * m) if (max(j - 1, 0) + 1) * m <= len(c) else 0
                coords = torch.as_tensor(c[lo:lo + m], device=dev).to(stage.rdtype)
                ipots = torch.as_tensor(ip[lo:lo + m], device=dev, dtype=torch.long)
                w = torch.as_tensor(deg[lo:lo + m], device=dev, dtype=torch.float64)[:, None]
                rows = torch.as_tensor(row[lo:lo + m], device=dev, dtype=torch.long)

                def fwd(x):
                    return stage.chi_fine(*stage.cchi(x, ipots), Q, S, "feff")

                def step():
                    out = torch.zeros(nrows, NK, device=dev, dtype=torch.float64)
                    if grad:
                        x = coords.clone().requires_grad_(True)
                        chi = checkpoint(fwd, x, use_reentrant=False)
                        out = out.index_add(0, rows, w * chi.to(torch.float64))
                        out.sum().backward()
                    else:
                        with torch.no_grad():
                            out = out.index_add(0, rows, w * fwd(coords).to(torch.float64))
                    return out.cpu()

                t, out = ev_time(step)
                if j == 0:
                    if save:
                        with torch.no_grad():
                            cc, _ = stage.cchi(coords, ipots)
                        keep[n] = (out.numpy(), cc.cpu().numpy(), lo, m)
                    continue
                per_path.append(t / m)
                sampled += m
                chunks += 1
            total += float(np.median(per_path)) * len(c)
            torch.cuda.empty_cache()
        return total, sampled, chunks

    out = {"source": "the reference's GPUPathStage, pip-installed unmodified into baseline/_ref, on this GPU"}
    with Clocks(uuid) as clk:
        for key, dtype, chunk, grad, mine in (("fwd_c64", torch.complex64, 4096, False, ours.get("fwd")),
                                              ("fwd_c128", torch.complex128, 4096, False, ours.get("fwd64")),
                                              ("fwd_bwd_c64", torch.complex64, 2048, True, ours.get("fwd_bwd"))):
            try:
                ms, sampled, chunks = arm(dtype, chunk, grad, save=(key == "fwd_c128"))
            except torch.cuda.OutOfMemoryError as err:
                out[key] = {"unavailable": f"out of memory: {err}"[:200]}
                torch.cuda.empty_cache()
                continue
            out[key] = {"value": n_paths * NK / (ms * 1e-3), "unit": UNIT, "ms_full_batch": ms,
                        "sample": f"{chunks} timed chunks ({sampled} paths of {n_paths}), three per leg count, "
                                  f"median time per path extrapolated per leg count",
                        "ours_over_reference": (ms / mine) if mine else None}
    out["clocks"] = clk.summary()
    return out, (keep, by_leg)


def parity_vs_reference(P, saved, dev):
    """This package's rows and cchi of the reference leg's first chunk of every leg count against the reference's
    complex128 ones: R-factor per (leg count, absorber row) of the mixed and FP64 rows, and the largest per-path
    |cchi - cchi_ref| / max|cchi_ref| of the mixed form."""
    import torch
    from feffgpu_b200 import GPUPathStage, PathBatch
    from feffgpu_b200.rspace import FitWindow, r_factor
    keep, by_leg = saved
    win = FitWindow(kmin=3.0, kmax=19.0, rmin=1.0, rmax=8.0)
    res = {"R_mixed_vs_ref_fp64": 0.0, "R_fp64_vs_ref_fp64": 0.0, "max_rel_cchi_mixed": 0.0, "paths": 0}
    st = {d: GPUPathStage(P, device=dev, dtype=d) for d in (torch.complex64, torch.complex128)}
    for n, (ref_rows, ref_cc, lo, m) in keep.items():
        c, ip, deg, row = (v[lo:lo + m] for v in by_leg[n])
        b = PathBatch([(c, ip, deg, row)], nrows=ref_rows.shape[0], device=dev)
        for d, key in ((torch.complex64, "R_mixed_vs_ref_fp64"), (torch.complex128, "R_fp64_vs_ref_fp64")):
            with torch.no_grad():
                rows = st[d].chi_reduce(b, Q).cpu().numpy()
            for r in range(ref_rows.shape[0]):
                if np.abs(ref_rows[r]).max() > 0:
                    res[key] = max(res[key], r_factor(ref_rows[r], rows[r], win))
        with torch.no_grad():
            cc, _ = st[torch.complex64].cchi(torch.as_tensor(c), torch.as_tensor(ip))
        res["max_rel_cchi_mixed"] = max(res["max_rel_cchi_mixed"],
                                        float(np.abs(cc.cpu().numpy() - ref_cc).max() / np.abs(ref_cc).max()))
        res["paths"] += m
    res["window"] = "k 3-19, R 1-8, kw 2; rows per (leg count, absorber) of the first reference chunk of each leg count"
    return res


def reference_cpu_leg(P, groups, per_leg: int = 48):
    """The reference's own GPUPathStage on the host cores (device="cpu", torch's default thread count, as the
    reference requires): per leg count its first `per_leg` paths through cchi -> chi_fine -> weighted sum, timed
    after a warm-up call and extrapolated by the paths of that leg count; complex64 and complex128."""
    import dataclasses
    import torch
    ref = ROOT / "baseline" / "_ref"
    if not (ref / "feffgpu" / "stage.py").exists():
        return {"unavailable": "reference not installed under baseline/_ref"}
    sys.path.insert(0, str(ref))
    try:
        from feffgpu.pad import PhaseData as RefPhase
        from feffgpu.stage import GPUPathStage as RefStage
    except Exception as err:                                   # noqa: BLE001 - report, do not fail the bench
        return {"unavailable": f"reference import failed: {err!r}"[:200]}
    finally:
        sys.path.remove(str(ref))
    refP = RefPhase(**{f.name: getattr(P, f.name) for f in dataclasses.fields(RefPhase)})
    by_leg: dict = {}
    for c, ip, deg, _row in groups:
        by_leg.setdefault(c.shape[1], []).append((c, ip, deg))
    by_leg = {n: tuple(np.concatenate([x[i] for x in v]) for i in range(3)) for n, v in sorted(by_leg.items())}
    n_paths = sum(len(v[0]) for v in by_leg.values())
    out = {"source": "the reference's GPUPathStage(device='cpu'), pip-installed unmodified into baseline/_ref",
           "cores": torch.get_num_threads()}
    for key, dtype in (("fwd_c64", torch.complex64), ("fwd_c128", torch.complex128)):
        stage = RefStage(refP, device="cpu", dtype=dtype)
        S = stage.linear_matrix(Q)
        total, sampled = 0.0, 0
        with torch.no_grad():
            for n, (c, ip, deg) in by_leg.items():
                m = min(len(c), per_leg)
                x = torch.as_tensor(c[:m]).to(stage.rdtype)
                ipt = torch.as_tensor(ip[:m], dtype=torch.long)
                w = torch.as_tensor(deg[:m], dtype=torch.float64)[:, None]

                def step():
                    return (w * stage.chi_fine(*stage.cchi(x, ipt), Q, S, "feff").to(torch.float64)).sum(0)

                step()
                t0 = time.perf_counter()
                step()
                total += (time.perf_counter() - t0) * len(c) / m
                sampled += m
        out[key] = {"value": n_paths * NK / total, "unit": UNIT, "s_full_batch": total,
                    "sample": f"{sampled} of {n_paths} paths (the first {per_leg} of every leg count), extrapolated"}
    return out


def frontends_leg(dev):
    """The reference's own front ends (installed unmodified under baseline/_ref) timed on its own classes and then
    after feffgpu_b200.install(), each after one warm-up call, wall clock with the device synchronised:
    * MD: EdgeSpectra.spectrum of one thermal bcc Fe frame (16^3 cells, 8192 atoms, sigma 0.08 A) for 32 absorbers,
      paths of up to 3 legs within 5.5 A (src/feffgpu/md/spectrum.py:303-340);
    * RMC: MultipleScattering.full_pass and full_gradient of the same frame for 32 absorbers, 3 legs, critpw 2
      (src/feffgpu/exafs/forward.py:691-723).
    The front ends' own orchestration (per-absorber finder calls, chunk loops, host syncs) is timed too: this is what
    the one-line drop-in buys, not the fused API's figure.  Each figure is the median of three timed calls."""
    import dataclasses
    import torch
    ref = ROOT / "baseline" / "_ref"
    if not (ref / "feffgpu" / "md" / "spectrum.py").exists():
        return {"unavailable": "reference not installed under baseline/_ref"}
    sys.path.insert(0, str(ref))
    try:
        import feffgpu.exafs.forward as F
        from feffgpu.md.spectrum import EdgeSpectra
        from feffgpu.pad import PhaseData as RefPhase
    except Exception as err:                                   # noqa: BLE001 - report, do not fail the bench
        return {"unavailable": f"reference import failed: {err!r}"[:200]}
    import feffgpu_b200
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.pad import phase_from_npz
    ours = phase_from_npz(np.load(ROOT / "tests" / "golden" / "cfg4_fe_phase.npz"), prefix="ph_")
    P = RefPhase(**{f.name: getattr(ours, f.name) for f in dataclasses.fields(RefPhase)})
    base, L = W.bcc_supercell(16, 2.87)
    pos = W.thermal(base, 0.08, seed=11)
    cell = np.eye(3) * L
    absorbers = np.random.default_rng(12).choice(len(pos), 32, replace=False)
    symbols = np.array(["Fe"] * len(pos))
    k = np.arange(401) * 0.05

    def wall(fn, reps=3):
        fn()
        ms = []
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize(dev)
            ms.append((time.perf_counter() - t0) * 1e3)
        return float(np.median(ms))

    def md():
        es = EdgeSpectra(P, "Fe", {"Fe": 1}, ["Fe"], k, rpath=5.5, nleg=3, criteria=2.0, device=str(dev))
        return lambda: es.spectrum(pos, cell, absorbers, symbols)

    def rmc():
        ms = F.MultipleScattering(P, k, 0.0, torch.tensor(cell), rmax=5.5, critpw=2.0, nlegmax=3, device=str(dev))
        x = torch.tensor(pos, device=dev, dtype=torch.float32)
        ms.enumerate(x[None], absorbers=absorbers)
        w = torch.tensor(np.random.default_rng(7).normal(size=len(k)), device=dev)

        def step():
            ms.full_pass(x)
            ms.full_gradient(x, lambda chi: (chi.double() * w).sum())
        return step

    out = {"workload": "bcc Fe 16^3 cells (8192 atoms), 32 absorbers, 3 legs within 5.5 A, 401 k"}
    res = {"reference": {"md_frame_ms": wall(md()), "rmc_pass_and_gradient_ms": wall(rmc())}}
    feffgpu_b200.install()
    res["installed"] = {"md_frame_ms": wall(md()), "rmc_pass_and_gradient_ms": wall(rmc())}
    out.update(res)
    out["speedup"] = {key: res["reference"][key] / res["installed"][key] for key in res["reference"]}
    sys.path.remove(str(ref))
    return out


def pairs_leg(args, dev, world, rank):
    """Single scattering from pair tables: rock-salt NiO 8^3 cells (5 % vacancies, 0.1 A disorder, 3,891 atoms), Ni K
    tables on r = 1.5..6 A step 0.002 (2,251 points x 401 k, one fused-stage call), then the all-pairs
    single-scattering spectrum (every atom an absorber) and its gradient with respect to every position, timed with
    CUDA events (median of 5 after a warm-up)."""
    import time as _time
    import torch
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.pad import phase_from_npz
    from feffgpu_b200.pairs import PairTables
    pos0, lab, box = W.rock_salt_supercell(8, 4.177)
    rng = np.random.default_rng(5 + rank)
    keep = rng.random(len(pos0)) >= 0.05
    pos = W.thermal(pos0[keep], 0.1, seed=6 + rank)
    ipot = np.array([{"Ni": 1, "O": 2}[x] for x in lab[keep]])
    P = phase_from_npz(np.load(ROOT / "tests" / "golden" / "cfg5_nik_phase.npz"), prefix="ph_")
    torch.cuda.synchronize(dev)
    t0 = _time.perf_counter()
    pt = PairTables(P, Q, box=box, rmax=6.0, r_min=1.5, dr=0.002, device=dev, dtype=torch.complex64)
    torch.cuda.synchronize(dev)
    t_tables = (_time.perf_counter() - t0) * 1e3
    pt.ipot = torch.tensor(ipot)
    w = torch.randn(NK, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))

    def step():
        x = torch.tensor(pos, device=dev, requires_grad=True)
        (pt.single_scattering(x) * w).sum().backward()

    step()
    ms = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return {"atoms": len(pos), "grid_points": pt.nr, "tables_ms": t_tables, "spectrum_and_gradient_ms": float(np.median(ms)),
            "pairs_per_s": len(pos) * (len(pos) - 1) / (float(np.median(ms)) * 1e-3)}


def rmc_extra(args, dev, world, rank):
    """RMC refinement: rock-salt NiO 8^3 cells (4096 sites, a = 4.177 A) with 5 % vacancies and 0.1 A disorder; Ni K
    and O K edges, 32 absorbers each, their paths from the CUDA path finder (rmax 5 A, 4 legs, importance cut 2 %,
    single scattering unmerged: the reference GpuRmc's defaults, src/feffgpu/rmc/refine.py:84-89 and
    exafs/forward.py:68-75); targets from a hidden 0.03 A perturbation;
    each step (both edges' rows, R-space misfits, backward, Adam on all positions) one CUDA graph replay with the
    autotuned launch shapes; every `rmc_refresh` steps (the reference's default cadence, refine.py:176-179) the
    paths are found again at the current positions and the step is captured again.  `rmc_steps` steps timed with
    CUDA events and the host clock, refreshes included; the refreshes' own cost is reported beside."""
    import time as _time
    import torch
    from feffgpu_b200 import GPUPathStage
    from feffgpu_b200 import workloads as W
    from feffgpu_b200.model import GraphedRefinement, PathModel, finder_groups
    from feffgpu_b200.pad import phase_from_npz
    from feffgpu_b200.pathfinder import GPUPathFinder
    from feffgpu_b200.rspace import FitWindow, RSpaceMisfit
    pos0, lab, box = W.rock_salt_supercell(8, 4.177)
    rng = np.random.default_rng(5 + rank)
    keep = rng.random(len(pos0)) >= 0.05
    pos0, lab = pos0[keep], lab[keep]
    pos = W.thermal(pos0, 0.1, seed=6 + rank)
    hidden = W.thermal(pos, 0.03, seed=7 + rank)
    q = torch.tensor(Q, device=dev)
    ipot_of = np.array([{"Ni": 1, "O": 2}[x] for x in lab])
    edges = []
    for edge, fname in (("Ni", "cfg5_nik_phase"), ("O", "cfg5_ok_phase")):
        P = phase_from_npz(np.load(ROOT / "tests" / "golden" / f"{fname}.npz"), prefix="ph_")
        st = GPUPathStage(P, device=dev, dtype=torch.complex64, autotune=not args.no_autotune)
        finder = GPUPathFinder(P, device=dev, rmax=5.0, nlegmax=4, critpw=2.0, merge_degenerate=False)
        edges.append((st, finder, W.central_atom(pos, box, lab, edge, 32)))

    def build(x):
        return [PathModel(st, finder_groups(f, x, box, ab, ipot_of), x, nrows=1, box=box) for st, f, ab in edges]

    models, npaths = [], 0
    for (st, _f, _ab), model in zip(edges, build(pos)):
        npaths += model.batch.n
        S = st.linear_matrix(Q).double().contiguous()
        with torch.no_grad():
            target = model.rows(torch.tensor(hidden, device=dev), q, S)[0]
        models.append((model, q, S, RSpaceMisfit(NK, target, FitWindow(kmin=3.0, kmax=14.0, rmin=1.0, rmax=5.0),
                                                 device=dev)))

    def rebuild(x, old):
        return [(m, qq, SS, mis) for m, (_m, qq, SS, mis) in zip(build(x.cpu().numpy()), old)]

    g = GraphedRefinement(models, pos, lr=0.002, rebuild=rebuild, refresh_every=args.rmc_refresh)
    torch.cuda.synchronize(dev)
    g.step()
    torch.cuda.synchronize(dev)
    first = float(g.loss)
    g.reset()
    n = args.rmc_steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0 = _time.perf_counter()
    e0.record()
    for _ in range(n):
        g.step()
    e1.record()
    e1.synchronize()
    wall = (_time.perf_counter() - t0) * 1e3
    refresh_ms = [ms for _s, ms in g.refreshes]
    return {"steps": n, "ms_per_step": e0.elapsed_time(e1) / n, "wall_ms_per_step": wall / n,
            "wall_ms_per_step_between_refreshes": (wall - sum(refresh_ms)) / n, "atoms": len(pos),
            "paths_per_gpu": npaths, "paths_after_refresh": sum(m[0].batch.n for m in g.models),
            "refresh_every": args.rmc_refresh, "refreshes_ms": refresh_ms,
            "misfit_first_step": first, "misfit_final": float(g.loss),
            "launch_warps": [list(m[0].stage._launch) for m in g.models],
            "graph": "one CUDA graph replay per step; paths found again and the step re-captured at each refresh"}


# ------------------------------------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU work for the CPU baseline")
    ap.add_argument("--paths-scale", type=float, default=1.0, help="scale the paths per leg count (profiling runs)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--no-extras", action="store_true", help="only the headline forward (profiling runs)")
    ap.add_argument("--md-frames", type=int, default=500, help="frames of the MD-batch leg (0: skip it)")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes (profiling runs)")
    ap.add_argument("--rmc-steps", type=int, default=500, help="steps of the RMC leg (0: skip it)")
    ap.add_argument("--rmc-refresh", type=int, default=250, help="steps between path searches in the RMC leg")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference's own stage (GPU and host legs)")
    ap.add_argument("--frontends", action="store_true",
                    help="only time the reference's MD and RMC front ends on its own classes and after install()")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nthreads = os.cpu_count() or 1

    if args.frontends:
        import torch
        print(json.dumps({"frontends": frontends_leg(torch.device("cuda", 0))}))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        P, groups = workload(args.gpus, args.paths_scale, finder="oracle")
        vals, walls, timed_paths = [], [], 0
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            v, desc, smp = cpu_sample(P, groups, budget_s=max(2.0, args.cpu_budget / 3), nthreads=nthreads)
            wall = time.perf_counter() - t0
            if i >= args.warmup:
                vals.append(v)
                walls.append(wall)
                timed_paths = sum(len(x[0]) for x in smp.values())
        v = float(np.median(vals))
        n_paths = sum(len(g[0]) for g in groups)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.median(walls)) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
            "config": workload_config(groups, world=args.gpus),
            "reference_impl": "FP64 C port of the reference's path stage (oracle), all host cores",
            "timing": {"step": "one stratified sample of the batch (every leg count), timed per leg count; value = "
                               "the batch's path·k over the per-leg-count extrapolated time",
                       "timed_paths_per_step": timed_paths, "timed_s": float(np.sum(walls)),
                       "ms_full_batch_extrapolated": n_paths * NK / v * 1e3},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    import torch.distributed as dist
    from feffgpu_b200 import GPUPathStage, PathBatch, _lib
    from feffgpu_b200.roofline import batch_flops
    from feffgpu_b200.autotune import default_tuner, shape_key
    tuner = default_tuner()

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    P, all_groups = workload(world, args.paths_scale)
    stage = GPUPathStage(P, device=dev, dtype=torch.complex64, autotune=not args.no_autotune)
    from feffgpu_b200.sharded import chi_reduce_all_ranks, split_groups
    groups = split_groups(all_groups, world, rank, lmax=stage.lmax.cpu().numpy()) if world > 1 else all_groups
    batch = PathBatch(groups, nrows=2 * world, device=dev)
    n_total = sum(len(g[0]) for g in all_groups)

    def step_rows(**kw):
        # one rank: the fused call itself; several: each rank's share, exact row sums summed as integers
        return chi_reduce_all_ranks(stage, batch, Q, S, **kw) if world > 1 else stage.chi_reduce(batch, Q, S, **kw)
    S = stage.linear_matrix(Q)
    lib = _lib.load()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2, written between steps
    n_paths = batch.n

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(fn, steps, warmup, kernel_time=False):
        for _ in range(warmup):
            fn()
        barrier()
        total, kern = 0.0, []
        if kernel_time:
            lib.fg_set_kernel_timing(1)
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            total += e0.elapsed_time(e1)
            if kernel_time:
                import ctypes
                ms = ctypes.c_float()
                _lib.check(lib.fg_kernel_time_ms(ctypes.byref(ms)))
                kern.append(ms.value)
        if kernel_time:
            lib.fg_set_kernel_timing(0)
        barrier()
        t = torch.tensor([total], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()) / steps, kern

    # the headline: fused forward with the inputs resident
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    uuid = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    with torch.no_grad():
        with Clocks(uuid) as clk:
            ms, kern = timed(lambda: step_rows(), args.steps, args.warmup, kernel_time=True)
    value = n_total * NK / (ms * 1e-3)

    e2e = fwd_bwd = plain = md = rmc = pf = pairs = ref_gpu = saved = None
    if not args.no_extras:
        pf = finder_leg(args, dev, world, rank)
        pairs = pairs_leg(args, dev, world, rank)
        e2e, fwd_bwd, plain = extras(args, stage, batch, P, S, dev, timed, n_total, ms)
        if not args.no_ref_gpu and rank == 0:
            ref_gpu, saved = reference_gpu_leg(args, P, groups, dev, {
                "fwd": ms, "fwd64": plain["ms_per_step"], "fwd_bwd": (fwd_bwd or {}).get("ms_per_step")}, uuid)
        if args.md_frames > 0:
            md = md_extra(args, dev, timed, world, rank)
        if args.rmc_steps > 0:
            rmc = rmc_extra(args, dev, world, rank)
    # roofline of the dominant kernel (the fused per-path kernel): algorithmic FLOPs of the reference's loops
    import ctypes
    peak = ctypes.c_double()
    _lib.check(lib.fg_fp32_fma_peak(ctypes.byref(peak), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    flops = batch_flops(batch.nleg.cpu().numpy(), batch.ipots.cpu().numpy(), stage.lmax.cpu().numpy())
    kern_ms = float(np.mean(kern)) if kern else None
    achieved = flops / (kern_ms * 1e-3) / 1e12 if kern_ms else None
    traffic, traffic_src = None, None
    tf = ROOT / "profiles" / "k_fused_feopt_traffic.txt"
    if tf.exists():
        for line in tf.read_text().splitlines():
            if line.startswith("bytes_per_launch"):
                traffic = float(line.split("=")[1])
            if line.startswith("captured"):
                traffic_src = line.split("=", 1)[1].strip()
    pipe, pipe_src = None, None
    pf_ = ROOT / "profiles" / "k_fused_fma_pipe_full_size.md"
    if pf_.exists():
        for line in pf_.read_text().splitlines():
            if line.startswith("captured=") and "fma_pipe_pct=" in line:
                kv = dict(x.split("=", 1) for x in line.split())
                pipe, pipe_src = float(kv["fma_pipe_pct"]), kv["captured"]
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
            "frac": achieved / peak.value if achieved else None, "traffic": traffic,
            "traffic_source": f"not measured in this run: ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                              f"full-size launch, profiles/k_fused_feopt_traffic.txt ({traffic_src})",
            "fma_pipe_active_pct": pipe,
            "fma_pipe_source": f"not measured in this run: ncu sm__pipe_fma_cycles_active of one full-size launch, "
                               f"profiles/k_fused_fma_pipe_full_size.md ({pipe_src})",
            "kernel": "k_fused (per-path signal, all leg counts, one persistent launch)",
            "kernel_ms": kern_ms, "flops_per_launch": flops,
            "peak_source": "measured on this GPU by fg_fp32_fma_peak (FFMA chains on every SM); "
                           "MEASURED_PEAKS.json holds no FP32 figure"}

    cpu = ref_cpu = None
    parity = {}
    if rank == 0 and not args.no_cpu:
        v, desc, samples = cpu_sample(P, groups, budget_s=args.cpu_budget, nthreads=nthreads)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc}
        parity["oracle"] = parity_vs_oracle(P, samples, dev)
        if not args.no_ref_gpu:
            ref_cpu = reference_cpu_leg(P, groups)
    if saved is not None:
        parity["reference_gpu_stage"] = parity_vs_reference(P, saved, dev)

    # the figures beside the headline, gathered last so that they close the line
    def g(d, *k):
        for key in k:
            d = (d or {}).get(key) if isinstance(d, dict) else None
        return d
    summary = {
        "fwd_ms": ms, "fwd_bwd_ms": g(fwd_bwd, "ms_per_step"), "fwd_bwd_value": g(fwd_bwd, "value"),
        "plain_fp64_ms": g(plain, "ms_per_step"), "e2e_value": g(e2e, "value"),
        "roofline_frac": roof["frac"],
        "parity_R_mixed_vs_oracle": g(parity, "oracle", "R_mixed_vs_oracle"),
        "parity_R_fp64_vs_oracle": g(parity, "oracle", "R_fp64_vs_oracle"),
        "parity_R_mixed_vs_reference_fp64": g(parity, "reference_gpu_stage", "R_mixed_vs_ref_fp64"),
        "parity_R_fp64_vs_reference_fp64": g(parity, "reference_gpu_stage", "R_fp64_vs_ref_fp64"),
        "parity_max_rel_cchi_mixed": g(parity, "reference_gpu_stage", "max_rel_cchi_mixed"),
        "md_ms": g(md, "ms_per_step"), "md_fp64_ms": g(md, "fp64_ms_per_step"),
        "md_R_vs_fp64_max": g(md, "r_factor_vs_fp64_max"),
        "rmc_ms_per_step": g(rmc, "ms_per_step"), "path_finder_ms": g(pf, "ms"),
        "reference_gpu_fwd_c64_ms": g(ref_gpu, "fwd_c64", "ms_full_batch"),
        "reference_gpu_fwd_c128_ms": g(ref_gpu, "fwd_c128", "ms_full_batch"),
        "reference_gpu_fwd_bwd_c64_ms": g(ref_gpu, "fwd_bwd_c64", "ms_full_batch"),
    }
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 (complex chain) + fp64 (phase argument, sums)", "data": "synthetic",
        "config": workload_config(all_groups, world),
        "autotune": {"fwd_warps": stage._launch[0], "bwd_warps": stage._launch[1],
                     "fwd_regs_alt": stage._launch[2], "fwd_stage_t": stage._launch[3],
                     "timed": [{"kind": k, "shape": shape_key(w_) if k == "fwd" else w_, "ms": round(t_, 3)}
                               for sig, k, w_, t_ in tuner.log if sig.split("|")[1] == "p0"]},
        "reference_cpu": ref_cpu, "pair_tables": pairs, "path_finder": pf, "md_batch": md, "rmc_refinement": rmc,
        "reference_gpu": ref_gpu, "plain_fp64": plain, "fwd_bwd": fwd_bwd,
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "parity": parity,
        "gpu_launches": 3 * args.steps, "clocks": clk.summary(), "summary": summary,
    }
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
