"""Builds libbfx.so (CUDA engines for sm_100a + host builders + C ABI) in-tree.

    python bf-new_b200/build.py [--force] [--verbose]

Objects go to bf-new_b200/_build/, the library to bf-new_b200/lib/libbfx.so.
nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libbfx.so"
INCLUDE = REPO / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-v"]
CXX_FLAGS = ["-O3", "-std=c++20", "-fPIC", "-Wall", "-Wextra", "-pthread"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cuda_include() -> Path:
    return Path(nvcc()).resolve().parent.parent / "include"


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return res.stdout + res.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    sources = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp"))
    if not force and not _stale(LIB, sources + headers):
        return LIB  # up to date (also where only the built library travelled)
    objs = []
    ptxas_log = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".cu.o")
        if force or _stale(obj, [src, *headers]):
            out = _run([nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)], verbose)
            ptxas_log.append(out)
        objs.append(obj)
    for src in sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.stem + ".cpp.o")
        if force or _stale(obj, [src, *headers]):
            _run(["g++", *CXX_FLAGS, "-I", str(INCLUDE), "-I", str(cuda_include()), "-c", str(src), "-o", str(obj)],
                 verbose)
        objs.append(obj)
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-lpthread"], verbose)
        os.replace(tmp, LIB)
    if ptxas_log:
        (BUILD / "ptxas.log").write_text("\n".join(ptxas_log))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
