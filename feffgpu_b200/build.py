"""Builds the sm_100a shared library ``feffgpu_b200/_build/libfeffgpu_b200.so`` with nvcc.

Each translation unit of ``csrc/`` compiles in its own nvcc process (in parallel), then nvcc links them into one
shared library with the C ABI of ``include/feffgpu_b200.h``.  Rebuilds only what changed (by modification time
against every header).  ``python -m feffgpu_b200.build`` builds from the command line.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = OUT / "libfeffgpu_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build feffgpu_b200")
    return exe


def _headers_mtime() -> float:
    files = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return max(f.stat().st_mtime for f in files)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False, out: Path | None = None,
          defines: dict | None = None) -> Path:
    """Compile (if stale) and return the library path.  out/defines build a variant elsewhere (with preprocessor
    definitions) for offline comparisons."""
    out_dir = OUT if out is None else Path(out)
    lib = out_dir / LIB.name
    out_dir.mkdir(parents=True, exist_ok=True)
    extra = [f"-D{k}={v}" for k, v in (defines or {}).items()]
    sources = sorted(CSRC.glob("*.cu"))
    hdr = _headers_mtime()
    jobs = []
    for src in sources:
        obj = out_dir / (src.stem + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr):
            cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    if jobs:
        workers = max(1, min(len(jobs), os.cpu_count() or 1))
        with ThreadPoolExecutor(workers) as ex:
            for src, r in ex.map(run, jobs):
                if verbose or ptxas_info or r.returncode:
                    sys.stderr.write(r.stdout + r.stderr)
                if r.returncode:
                    raise RuntimeError(f"nvcc failed on {src.name}")
    objs = [str(out_dir / (s.stem + ".o")) for s in sources]
    if jobs or not lib.exists() or lib.stat().st_mtime < max(Path(o).stat().st_mtime for o in objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc link failed")
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
