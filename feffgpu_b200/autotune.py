"""Launch-shape autotuner of the persistent per-path kernels.

The forward (fused stage) and the adjoint kernels keep one path per warp and take their launch shape -- warps per
CTA, i.e. paths in flight per CTA -- at launch.  The shape sets the shared-memory granule of a CTA (the per-warp
rotation tables grow with the batch's longest path and double in FP64) and with it how many paths an SM keeps
resident under the register and shared-memory limits; which shape is fastest depends on the precision, the leg mix
and the energy count.  The autotuner times every candidate shape on the device (CUDA events on the current stream,
one warm-up and three timed launches each, on a stratified sample of the batch), keeps the fastest per workload
signature, and persists the choice per GPU model in a JSON file (``$FEFFGPU_B200_TUNE_CACHE``, default
``~/.cache/feffgpu_b200/autotune.json``), so a workload is tuned once.  Results do not depend on the shape: the
cross-path sums run in a fixed order whatever the schedule.

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
SAMPLE_PATHS = 32768
_lock = threading.Lock()


def cache_path() -> Path:
    p = os.environ.get("FEFFGPU_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "feffgpu_b200" / "autotune.json"


def gpu_name(device) -> str:
    return torch.cuda.get_device_name(device).replace(" ", "_")


def signature(stage, batch, nk: int, prec: int) -> str:
    """Workload key: GPU model, precision, initial-state class, energies, k points, longest path and the leg mix
    (fraction of paths per leg count, to 0.05)."""
    name = gpu_name(stage.device)
    n = max(batch.n, 1)
    mix = ",".join(f"{k}:{round(20 * v / n) / 20:.2f}" for k, v in sorted(batch.counts.items()))
    return f"{name}|p{prec}|l{stage.ilinit}|E{stage.E}|K{nk}|n{batch.nleg_max}|{mix}"


class Autotuner:
    """Chooses (forward warps, adjoint warps) per workload signature.  ``timer(kind, stage, batch, q, S, prec, w)``
    returns milliseconds for one candidate (the default times the library's calls with CUDA events)."""

    def __init__(self, path: Path | None = None, timer=None, sample_paths: int = SAMPLE_PATHS):
        self.path = Path(path) if path is not None else cache_path()
        self.timer = timer or _time_candidate
        self.sample_paths = sample_paths
        self.table: dict = self._load()
        self.log: list = []          # (signature, kind, warps, ms) of the candidates timed by this process

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
        return int(e["fwd"]), int(e.get("bwd", 0))

    def tune(self, stage, batch, q, S, prec: int, backward: bool = True):
        """Times the candidates and records the fastest; returns (fwd_warps, bwd_warps)."""
        nk = int(q.shape[0])
        sig = signature(stage, batch, nk, prec)
        with _lock:
            hit = self.lookup(sig, backward)
            if hit is not None:
                return hit
            sample = batch.sample(self.sample_paths)
            times = {}
            for w in FWD_WARPS:
                times[("fwd", w)] = self.timer("fwd", stage, sample, q, S, prec, w)
            fwd = _pick({w: times[("fwd", w)] for w in FWD_WARPS})
            entry = {"fwd": fwd, "ms_fwd": {str(w): round(times[("fwd", w)], 4) for w in FWD_WARPS},
                     "sample_paths": sample.n}
            if backward:
                for w in BWD_WARPS:
                    times[("bwd", w)] = self.timer("bwd", stage, sample, q, S, prec, w)
                entry["bwd"] = _pick({w: times[("bwd", w)] for w in BWD_WARPS})
                entry["ms_bwd"] = {str(w): round(times[("bwd", w)], 4) for w in BWD_WARPS}
            for (kind, w), ms in times.items():
                self.log.append((sig, kind, w, ms))
            self.table[sig] = entry
            self._save()
            return entry["fwd"], entry.get("bwd", 0)


def _pick(ms: dict, tol: float = 0.01) -> int:
    """The widest shape within tol of the fastest (timing noise does not move the choice off the default)."""
    best = min(ms.values())
    return max(w for w, t in ms.items() if t <= best * (1 + tol))


def _time_candidate(kind: str, stage, batch, q, S, prec: int, warps: int, reps: int = 3) -> float:
    """Milliseconds of the forward (kind 'fwd') or adjoint ('bwd') call on batch with `warps` warps per CTA."""
    lib = stage._lib
    coords = batch.coords.contiguous()
    fw, bw = (warps, 0) if kind == "fwd" else (0, warps)
    _lib.check(lib.fg_stage_set_launch(stage._h, fw, bw))
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
        _lib.check(lib.fg_stage_set_launch(stage._h, *stage._launch))


_default = None


def default_tuner() -> Autotuner:
    global _default
    if _default is None:
        _default = Autotuner()
    return _default
