"""Build ``libpystarc_b200.so`` in-tree with nvcc for sm_100a (no JIT, no torch extension cache).

Each source compiles to its own object in parallel (one nvcc process per file);
the objects are linked into the shared library.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libpystarc_b200.so"
SOURCES = ["bd_api.cu", "bd_noalloc.cu", "bd_mlp.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "pystarc_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = Path(tempfile.mkdtemp(prefix="pystarc_b200_build_"))
    procs = []
    objs = []
    for s in SOURCES:
        obj = objdir / (Path(s).stem + ".o")
        cmd = [nvcc(), *FLAGS, f"-I{ROOT / 'include'}", "-c", "-o", str(obj), str(CSRC / s)]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(str(obj))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = [nvcc(), *ARCH, "-shared", "-o", str(LIB) + ".tmp", *objs]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    shutil.rmtree(objdir, ignore_errors=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
