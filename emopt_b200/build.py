"""Build the B200 CUDA library ``emopt_b200/FDTD.so`` in-tree with nvcc.

The library is the drop-in replacement for the reference ``FDTD.so``: the same
C ABI (``include/emopt_fdtd.h``) implemented as a C++ host layer over
hand-written sm_100a kernels.  It is compiled for ``sm_100a`` only and links the
CUDA runtime statically, so it needs no torch or toolkit libraries at run time.

A second library, ``emopt_b200/FDTD_checked.so``, is the same code with
``FDTD_BOUNDS_CHECK`` defined in the sources that hold the production
stepping kernels (the vector pair and the serving kernel): every index those
kernels compute is checked against its array, an out-of-range lane records
where and skips the access, and the solve, slab and serving calls then fail
with the site.  It is a debugging build, selected by setting
``EMOPT_B200_LIB`` to its path before ``emopt_b200.fdtd_ctypes`` is imported.

Usage: ``python -m emopt_b200.build`` (also called by ``__graft_entry__.build``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "FDTD.so")
CHECKED = os.path.join(HERE, "FDTD_checked.so")
# sources whose kernels carry the index checks in the checked library
CHECKED_SOURCES = ["fdtd_abi.cu", "vec_kernels.cu", "serve_kernels.cu"]
BUILD = os.path.join(HERE, "_build")
SOURCES = ["fdtd_abi.cu", "step_kernels.cu", "vec_kernels.cu", "zmarch_kernels.cu", "aux_kernels.cu",
           "legacy_kernels.cu", "grad_kernels.cu", "serve_kernels.cu", "noalloc.cu", "structured.cu",
           "modes.cu", "fields_kernels.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, extra: list[str], headers: list[str], verbose: bool, force: bool) -> None:
    s = os.path.join(CSRC, src)
    if force or _stale(obj, [s] + headers):
        cmd = [nvcc()] + ARCH + FLAGS + extra + ["-c", s, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


def _link(out: str, objs: list[str], verbose: bool, force: bool) -> None:
    if force or _stale(out, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", out] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False, checked: bool = True) -> str:
    """Build FDTD.so (and, unless ``checked`` is False, FDTD_checked.so)."""
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "emopt_fdtd.h"))
    objs = []
    for src in SOURCES:
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        _compile(src, o, [], headers, verbose, force)
    _link(OUT, objs, verbose, force)
    if checked:
        cobjs = []
        for src, o in zip(SOURCES, objs):
            if src in CHECKED_SOURCES:
                o = os.path.join(BUILD, src.replace(".cu", ".checked.o"))
                _compile(src, o, ["-DFDTD_BOUNDS_CHECK"], headers, verbose, force)
            cobjs.append(o)
        _link(CHECKED, cobjs, verbose, force)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
