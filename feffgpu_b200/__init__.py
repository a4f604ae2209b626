"""feffgpu_b200 -- the batched EXAFS path stage of nmarcella/feffGPU, built for NVIDIA B200 (sm_100a).

``GPUPathStage`` is a drop-in for the reference's class of the same name (``src/feffgpu/stage.py``), and
``GPUPathFinder`` (``feffgpu_b200.pathfinder``) for its path finder (``src/feffgpu/pathfinder.py``); ``install()``
rebinds the reference's names to them so that its chain, MD-EXAFS and RMC-EXAFS front ends use them unchanged.
"""
from .pad import BOHR, HART, PhaseData, load_phase, read_phase_pad, resample_phase, save_phase
from .stage import GPUPathStage
from .batch import PathBatch

__all__ = ["GPUPathStage", "PathBatch", "PhaseData", "read_phase_pad", "load_phase", "resample_phase", "save_phase",
           "install", "BOHR", "HART"]


def install(finder: bool = True) -> list[str]:
    """Point the reference package's GPUPathStage (and, with finder, GPUPathFinder) names at this implementation.

    The reference binds the classes at import time: GPUPathStage in ``feffgpu/__init__.py:22``,
    ``feffgpu/chain.py:13`` and ``feffgpu/exafs/forward.py:27`` (besides ``feffgpu/stage.py`` itself), GPUPathFinder
    in ``feffgpu/__init__.py:21``, ``feffgpu/chain.py:12`` and ``feffgpu/exafs/forward.py:28`` (besides
    ``feffgpu/pathfinder.py``); all present modules are rebound.  Returns the names that now refer to this package.
    The reference package must be importable."""
    import importlib
    from .pathfinder import GPUPathFinder
    names = [("GPUPathStage", GPUPathStage, ("feffgpu.stage", "feffgpu", "feffgpu.chain", "feffgpu.exafs.forward"))]
    if finder:
        names.append(("GPUPathFinder", GPUPathFinder,
                      ("feffgpu.pathfinder", "feffgpu", "feffgpu.chain", "feffgpu.exafs.forward")))
    done = []
    for name, obj, mods in names:
        for mod in mods:
            try:
                m = importlib.import_module(mod)
            except ImportError:
                continue
            if hasattr(m, name):
                setattr(m, name, obj)
                done.append(f"{mod}.{name}")
    return done
