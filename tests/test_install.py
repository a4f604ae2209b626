"""install() rebinds the reference's GPUPathStage and GPUPathFinder names (fake reference modules, no GPU)."""
import sys
import types

import feffgpu_b200
from feffgpu_b200.pathfinder import GPUPathFinder


def test_install_rebinds_every_name(monkeypatch):
    mods = {}
    for name in ("feffgpu", "feffgpu.stage", "feffgpu.pathfinder", "feffgpu.chain", "feffgpu.exafs",
                 "feffgpu.exafs.forward"):
        m = types.ModuleType(name)
        mods[name] = m
        monkeypatch.setitem(sys.modules, name, m)
    for name in ("feffgpu", "feffgpu.stage", "feffgpu.chain", "feffgpu.exafs.forward"):
        mods[name].GPUPathStage = object
    for name in ("feffgpu", "feffgpu.pathfinder", "feffgpu.chain", "feffgpu.exafs.forward"):
        mods[name].GPUPathFinder = object
    done = feffgpu_b200.install()
    assert len(done) == 8
    for name in ("feffgpu", "feffgpu.stage", "feffgpu.chain", "feffgpu.exafs.forward"):
        assert mods[name].GPUPathStage is feffgpu_b200.GPUPathStage
    for name in ("feffgpu", "feffgpu.pathfinder", "feffgpu.chain", "feffgpu.exafs.forward"):
        assert mods[name].GPUPathFinder is GPUPathFinder
    assert not hasattr(mods["feffgpu.stage"], "GPUPathFinder")
