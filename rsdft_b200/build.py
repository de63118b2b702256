"""Build recipe of librsdft_gpu.so (sm_100a) from rsdft_b200/csrc.

``python -m rsdft_b200.build`` compiles every ``.cu`` file with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``rsdft_b200/_build`` and
links the shared library in-tree (``rsdft_b200/librsdft_gpu.so``) against
cuSOLVER.  Objects are rebuilt when their source or a header is
newer.  ``build(check=True)`` (``python -m rsdft_b200.build --check``) makes
the debug build ``librsdft_gpu_check.so`` with ``-DRSDFT_GPU_CHECK`` (in-kernel
index checks; objects under ``rsdft_b200/_build_check``), which
``rsdft_b200._lib`` loads when ``RSDFT_GPU_CHECK=1`` is set.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librsdft_gpu.so")
LIB_CHECK = os.path.join(HERE, "librsdft_gpu_check.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "-I", INCLUDE, "-I", CSRC]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib_dir() -> str:
    nvcc = _nvcc()
    root = os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))
    for d in ("lib64", os.path.join("targets", "x86_64-linux", "lib")):
        p = os.path.join(root, d)
        if os.path.exists(os.path.join(p, "libcusolver.so")):
            return p
    return os.path.join(root, "lib64")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + _headers())


def build(verbose: bool = False, extra_flags=None, check: bool = False) -> str:
    lib, objdir = (LIB_CHECK, BUILD + "_check") if check else (LIB, BUILD)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    if not extra_flags and os.path.exists(lib):
        # the linked library is newer than every source and header: nothing
        # to do, even where the object files did not travel with it
        t = os.path.getmtime(lib)
        if all(os.path.getmtime(d) <= t for d in srcs + _headers()):
            return lib
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    flags = NVCC_FLAGS + (["-DRSDFT_GPU_CHECK"] if check else []) + list(extra_flags or [])
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, s):
            jobs.append([nvcc, *ARCH, *flags, "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(run, jobs))
    if jobs or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        libdir = _cuda_lib_dir()
        link = [nvcc, *ARCH, "-shared", "-o", lib, *objs, "-L", libdir, "-lcusolver",
                "-Xlinker", "-rpath=" + libdir]
        run(link)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, check="--check" in sys.argv))
