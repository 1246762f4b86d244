"""Builds the libtorch autograd harness (torch_adjoint.cpp) in-tree.

    python bf-new_b200/harness/build_harness.py

Output: bf-new_b200/harness/_build/bfx_torch_harness*.so, linked against
bf-new_b200/lib/libbfx.so (rpath).  Gradient harness only; the product path
does not use torch.
"""
from __future__ import annotations

import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
REPO = PKG.parent


def load(verbose: bool = False):
    from torch.utils.cpp_extension import load as torch_load

    build_dir = HERE / "_build"
    build_dir.mkdir(exist_ok=True)
    lib_dir = PKG / "lib"
    return torch_load(
        name="bfx_torch_harness",
        sources=[str(HERE / "torch_adjoint.cpp")],
        extra_include_paths=[str(REPO / "include")],
        extra_ldflags=[f"-L{lib_dir}", "-lbfx", f"-Wl,-rpath,{lib_dir}"],
        build_directory=str(build_dir),
        verbose=verbose,
    )


if __name__ == "__main__":
    m = load(verbose="-v" in sys.argv)
    print(m.__file__)
