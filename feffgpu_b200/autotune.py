"""Launch-shape autotuner of the persistent per-path kernels.

The forward (fused stage) and the adjoint kernels keep one path per warp and take their launch shape at launch.
The adjoint's shape is its warps per CTA, i.e. paths in flight per CTA.  The forward's has three parts:

* warps per CTA (1, 2, 4): the shared-memory granule of a CTA (the per-warp rotation tables grow with the batch's
  longest path and double in FP64) and with it how many paths an SM keeps resident;
* the register budget: the default (two CTAs of 128 threads per SM in FP32, one in FP64) or three CTAs per SM --
  more warps to hide latency against fewer registers for the partial-wave loop's instruction-level parallelism;
* the t-matrix source: read through L1, or each scatterer's column copied into a shared-memory tile per warp first
  (asynchronous copies), which takes shared memory from L1.

Which shape is fastest depends on the precision, the leg mix and the energy count.  The autotuner times every
candidate on the device (CUDA events on the current stream, one warm-up and three timed launches each, on a
stratified sample of the batch), keeps the fastest per workload signature, and persists the choice per GPU model in
a JSON file (``$FEFFGPU_B200_TUNE_CACHE``, default ``~/.cache/feffgpu_b200/autotune.json``), so a workload is tuned
once.  Results do not depend on the shape: the cross-path sums are exact and every path's arithmetic is the same
whatever the schedule.

``GPUPathStage(..., autotune=True)`` tunes on the first call of each new workload signature (never inside CUDA
graph capture: a signature first met during capture runs with the default shape); ``GPUPathStage.tune`` tunes
explicitly.
"""
from __future__ import annotations

import json
import os
import threading
from pathlib import Path

import numpy as np
import torch

from . import _lib

FWD_WARPS = (1, 2, 4)
BWD_WARPS = (1, 2, 4)
FWD_VARIANTS = ((0, 0), (1, 0), (0, 1))      # (register budget, t-matrix staging): default, 3 CTAs per SM, staged
FWD_SHAPES = tuple((w, r, t) for r, t in FWD_VARIANTS for w in FWD_WARPS)
SAMPLE_PATHS = 32768
_lock = threading.Lock()


def cache_path() -> Path:
    p = os.environ.get("FEFFGPU_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "feffgpu_b200" / "autotune.json"


def gpu_name(device) -> str:
    return torch.cuda.get_device_name(device).replace(" ", "_")


def signature(stage, batch, nk: int, prec: int) -> str:
    """Workload key: GPU model, precision, initial-state class, lambda-set order (other orders run other kernels),
    energies, k points, longest path and the leg mix (fraction of paths per leg count, to 0.05)."""
    name = gpu_name(stage.device)
    n = max(batch.n, 1)
    mix = ",".join(f"{k}:{round(20 * v / n) / 20:.2f}" for k, v in sorted(batch.counts.items()))
    order = "" if getattr(stage, "iorder", 2) == 2 else f"|o{stage.iorder}"
    return f"{name}|p{prec}|l{stage.ilinit}{order}|E{stage.E}|K{nk}|n{batch.nleg_max}|{mix}"


def shape_key(shape) -> str:
    """'w4r0t0' for a forward shape (warps, register budget, t staging)."""
    w, r, t = shape
    return f"w{w}r{r}t{t}"


class Autotuner:
    """Chooses the launch per workload signature: (forward warps, adjoint warps, forward register budget, forward t
    staging).  ``timer(kind, stage, batch, q, S, prec, shape)`` returns milliseconds for one candidate, ``shape`` a
    (warps, register budget, t staging) tuple for 'fwd' and the warps for 'bwd' (the default times the library's
    calls with CUDA events)."""

    def __init__(self, path: Path | None = None, timer=None, sample_paths: int = SAMPLE_PATHS):
        self.path = Path(path) if path is not None else cache_path()
        self.timer = timer or _time_candidate
        self.sample_paths = sample_paths
        self.table: dict = self._load()
        self.log: list = []          # (signature, kind, shape, ms) of the candidates timed by this process

    def _load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (OSError, ValueError):
            return {}

    def _save(self) -> None:
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            tmp = self.path.with_suffix(f".tmp{os.getpid()}")
            tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
            os.replace(tmp, self.path)
        except OSError:
            pass                     # a read-only home keeps the choice in memory only

    def lookup(self, sig: str, backward: bool):
        e = self.table.get(sig)
        if e is None or (backward and "bwd" not in e):
            return None
        f = e["fwd"]
        w, r, t = (int(f), 0, 0) if isinstance(f, int) else (int(x) for x in f)
        return w, int(e.get("bwd", 0)), r, t

    def tune(self, stage, batch, q, S, prec: int, backward: bool = True):
        """Times the candidates and records the fastest; returns (fwd_warps, bwd_warps, regs_alt, stage_t)."""
        nk = int(q.shape[0])
        sig = signature(stage, batch, nk, prec)
        with _lock:
            hit = self.lookup(sig, backward)
            if hit is not None:
                return hit
            sample = batch.sample(self.sample_paths)
            entry = self.table.get(sig, {})
            if "fwd" in entry and "ms_fwd" in entry:
                fwd = self.lookup(sig, False)
                fwd = (fwd[0], fwd[2], fwd[3])
            else:
                tf = {sh: self.timer("fwd", stage, sample, q, S, prec, sh) for sh in FWD_SHAPES}
                fwd = _pick(tf)
                entry = {"fwd": list(fwd), "ms_fwd": {shape_key(sh): round(ms, 4) for sh, ms in tf.items()},
                         "sample_paths": sample.n}
                self.log += [(sig, "fwd", sh, ms) for sh, ms in tf.items()]
            if backward:
                tb = {w: self.timer("bwd", stage, sample, q, S, prec, w) for w in BWD_WARPS}
                entry["bwd"] = _pick(tb)
                entry["ms_bwd"] = {str(w): round(ms, 4) for w, ms in tb.items()}
                self.log += [(sig, "bwd", w, ms) for w, ms in tb.items()]
            self.table[sig] = entry
            self._save()
            return fwd[0], entry.get("bwd", 0), fwd[1], fwd[2]


def _preference(shape):
    """Order among near-ties: the default variant first, then the widest CTA."""
    if isinstance(shape, tuple):
        w, r, t = shape
        return (r + t, -w)
    return (0, -shape)


def _pick(ms: dict, tol: float = 0.01):
    """The preferred shape within tol of the fastest (timing noise does not move the choice off the default)."""
    best = min(ms.values())
    return min((sh for sh, t in ms.items() if t <= best * (1 + tol)), key=_preference)


def _time_candidate(kind: str, stage, batch, q, S, prec: int, shape, reps: int = 3) -> float:
    """Milliseconds of the forward (kind 'fwd', shape = (warps, register budget, t staging)) or adjoint ('bwd',
    shape = warps) call on batch."""
    lib = stage._lib
    coords = batch.coords.contiguous()
    if kind == "fwd":
        fw, bw, r, t = shape[0], 0, shape[1], shape[2]
    else:
        fw, bw, r, t = 0, shape, 0, 0
    _lib.check(lib.fg_stage_set_launch(stage._h, fw, bw))
    _lib.check(lib.fg_stage_set_fused_variant(stage._h, r, t))
    try:
        with torch.no_grad():
            if kind == "fwd":
                def run():
                    stage._chi_reduce_forward(batch, coords, None, q, S, prec, save=False)
            else:
                _, cchi, reff = stage._chi_reduce_forward(batch, coords, None, q, S, prec, save=True)
                g = torch.ones(batch.nrows, int(q.shape[0]), device=stage.device, dtype=torch.float64)

                def run():
                    stage._chi_reduce_backward(batch, coords, None, q, S, prec, g, cchi, reff, False)
            run()
            ms = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                run()
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))
    finally:
        fw, bw, r, t = stage._launch
        _lib.check(lib.fg_stage_set_launch(stage._h, fw, bw))
        _lib.check(lib.fg_stage_set_fused_variant(stage._h, r, t))


_default = None


def default_tuner() -> Autotuner:
    global _default
    if _default is None:
        _default = Autotuner()
    return _default
