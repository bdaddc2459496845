"""Build libwavetoy_b200.so in-tree with nvcc for sm_100a.

Usage: python wavetoysecondorder.jl_b200/build.py [--force] [--ptxas-verbose] [--bounds-check]

Every .cu file under csrc/ is compiled to an object (in parallel, skipped when
up to date) and linked into wavetoysecondorder.jl_b200/libwavetoy_b200.so.
--bounds-check builds the debug variant libwavetoy_b200_bc.so instead
(-DWT_BOUNDS_CHECK: every index a kernel reads from the mesh's neighbour,
face-source and boundary-slot tables is range-checked; see wt_common.cuh).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwavetoy_b200.so")
OBJ_BC = os.path.join(HERE, "_build_bc")
LIB_BC = os.path.join(HERE, "libwavetoy_b200_bc.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def _deps_mtime() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def _compile(src: str, force: bool, verbose: bool, objdir: str = OBJ, extra=()) -> str:
    obj = os.path.join(objdir, os.path.basename(src).replace(".cu", ".o"))
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= _deps_mtime()):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, bounds_check: bool = False) -> str:
    objdir, lib = (OBJ_BC, LIB_BC) if bounds_check else (OBJ, LIB)
    extra = ("-DWT_BOUNDS_CHECK",) if bounds_check else ()
    os.makedirs(objdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose, objdir, extra), srcs))
    if force or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--ptxas-verbose" in sys.argv,
                bounds_check="--bounds-check" in sys.argv))
