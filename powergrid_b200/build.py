"""Build the sm_100a shared library in-tree (nvcc, no JIT cache).

Output: powergrid_b200/lib/libpowergrid_b200.so, linked against cuFFT and
the CUDA runtime.  Objects go to powergrid_b200/_build/.  A source is
recompiled when it or any header under csrc/ or include/ is newer than its
object.  build(checks=True) makes the PG_CHECKS variant,
libpowergrid_b200_checks.so (objects in _build_checks/): the gridding
kernels' device-side index checks compiled in (pg_checks_read reports them);
loaded instead of the product when PG_LIBRARY=checks.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
BUILD_CHECKS = os.path.join(HERE, "_build_checks")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpowergrid_b200.so")
LIB_CHECKS = os.path.join(LIBDIR, "libpowergrid_b200_checks.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
         "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def _compile(src: str, extra=(), build_dir: str = BUILD) -> str:
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    if _stale(obj, src):
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, ptxas_info: bool = False, checks: bool = False) -> str:
    bdir, lib = (BUILD_CHECKS, LIB_CHECKS) if checks else (BUILD, LIB)
    os.makedirs(bdir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    extra = (["-Xptxas", "-v"] if ptxas_info else []) + (["-DPG_CHECKS"] if checks else [])
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, bdir), srcs))
    if not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", lib, *objs, "-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(lib)
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, checks="--checks" in sys.argv)
