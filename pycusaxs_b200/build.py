"""Build the sm_100a shared library ``pycusaxs_b200/lib/libpycusaxs_b200.so``.

The library is compiled in-tree with nvcc (no JIT cache), so the built file
travels with the source tree.  ``python -m pycusaxs_b200.build`` rebuilds it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIBNAME = "libpycusaxs_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["setup.cpp", "plan.cu", "noalloc.cu", "trajectory.cpp"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build pycusaxs_b200")
    return exe


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    out = LIBDIR / LIBNAME
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [
        REPO / "include" / "pycusaxs_b200.h", Path(__file__)]
    if not force and not _stale(out, deps):
        return out
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
              "-ffp-contract=off", "-I", str(REPO / "include"), "-I", str(CSRC)] + ARCH
    objs = []
    for s in SOURCES:
        src = CSRC / s
        obj = objdir / (s + ".o")
        lang = ["-x", "cu"] if s.endswith(".cu") else ["-x", "c++"]
        cmd = [nvcc()] + common + lang + ["-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIBDIR / f".{LIBNAME}.{os.getpid()}"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)
