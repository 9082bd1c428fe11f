"""Build libvoronota_b200.so (sm_100a) in-tree with nvcc.

The FP64 translation units are compiled with --fmad=false so that the device arithmetic
matches the reference's uncontracted f64 expressions; the FP32 contact kernel keeps FMA
contraction.  Usage: ``python voronota-ltr_b200/build.py`` (or ``build()`` from Python).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libvoronota_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xcompiler", "-Wall"]
UNITS = {
    "vt_pipeline.cu": ["--fmad=false"],
    "vt_contact64.cu": ["--fmad=false"],
    # FP32 bulk kernel: every decision is banded, so approximate division / square root
    # (a few ulps) are safe; 64 registers per thread for 8 resident blocks per SM
    "vt_contact32.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false", "-DVT_C32_MINB=8"],
    "vt_engine.cu": ["--fmad=false"],
    "vt_noalloc.cu": ["--fmad=false"],
    "vt_frontier.cu": ["--fmad=false"],
    "vt_batch.cu": ["--fmad=false"],
    "vt_adjoint.cu": ["--fmad=false"],
    "vt_network.cu": ["--fmad=false"],
    "vt_solvent.cu": ["--fmad=false"],
    "vt_updateable.cu": ["--fmad=false"],
}


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    # one build at a time: two concurrent builds could link objects compiled against
    # different versions of the shared headers (struct layouts passed to kernels by value)
    import fcntl

    with open(os.path.join(BUILD, ".lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        return _build_locked(verbose, ptxas_info)


def _build_locked(verbose: bool, ptxas_info: bool) -> str:
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "voronota_b200.h"))
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [src, __file__] + headers) or ptxas_info:
            cmd = [_nvcc(), *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
