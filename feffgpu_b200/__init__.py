"""feffgpu_b200 -- the batched EXAFS path stage of nmarcella/feffGPU, built for NVIDIA B200 (sm_100a).

``GPUPathStage`` is a drop-in for the reference's class of the same name (``src/feffgpu/stage.py``); ``install()``
rebinds the reference's names to it so that its chain, MD-EXAFS and RMC-EXAFS front ends use this stage unchanged.
"""
from .pad import BOHR, HART, PhaseData, load_phase, read_phase_pad, resample_phase, save_phase
from .stage import GPUPathStage
from .batch import PathBatch
from .compare import hanning, r_factor

__all__ = ["GPUPathStage", "PathBatch", "PhaseData", "read_phase_pad", "load_phase", "resample_phase", "save_phase",
           "r_factor", "hanning", "install", "BOHR", "HART"]


def install() -> list[str]:
    """Point the reference package's GPUPathStage names at this implementation.

    The reference binds the class at import time in ``feffgpu/__init__.py:22``, ``feffgpu/chain.py:13`` and
    ``feffgpu/exafs/forward.py:27`` (besides ``feffgpu/stage.py`` itself); all present modules are rebound.  Returns
    the names that now refer to this stage.  The reference package must be importable."""
    import importlib
    done = []
    for mod in ("feffgpu.stage", "feffgpu", "feffgpu.chain", "feffgpu.exafs.forward"):
        try:
            m = importlib.import_module(mod)
        except ImportError:
            continue
        if hasattr(m, "GPUPathStage"):
            setattr(m, "GPUPathStage", GPUPathStage)
            done.append(f"{mod}.GPUPathStage")
    return done
