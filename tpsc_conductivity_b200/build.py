"""Build the in-tree CUDA library ``libtpsc_b200.so`` for sm_100a.

    python -m tpsc_conductivity_b200.build          # or build() from Python

nvcc cross-compiles without a GPU.  The library is rebuilt only when a source
is newer than it (``force=True`` always rebuilds).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libtpsc_b200.so")
SOURCES = ["tpsc_kernels.cu", "tpsc_cond.cu", "tpsc_al.cu", "tpsc_mixed.cu", "tpsc_roots.cu", "tpsc_engine.cpp",
           "tpsc_batch.cpp", "tpsc_tangent.cu", "tpsc_noalloc.cu", "tpsc_files.cpp",
           "tpsc_lattice.cu", "tpsc_peaks.cu", "tpsc_adjoint.cu", "tpsc_direct.cu", "tpsc_tcdct.cu"]
HEADERS = ["tpsc_fft.cuh", "tpsc_kernels.cuh", "tpsc_device.cuh", "tpsc_dct.cuh", "tpsc_tc.cuh", "tpsc_host.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found (set NVCC or install the CUDA toolkit)")


def host_compiler() -> list[str]:
    # prefer the distribution g++ (another g++ on the image comes without libgomp)
    for cand in ("/usr/bin/g++",):
        if os.path.exists(cand):
            return ["-ccbin", cand]
    return []


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "tpsc_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc_path(), *ARCH, *host_compiler(), "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
              "-I", os.path.join(ROOT, "include")]
    if verbose:
        common.insert(1, "-Xptxas=-v")

    def compile_one(src: str) -> str:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [*common, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    # the translation units compile independently (one nvcc each), then one link
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    subprocess.run([nvcc_path(), *ARCH, *host_compiler(), "-shared", "-cudart", "static", *objs, "-o", LIB + ".tmp"],
                   check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
