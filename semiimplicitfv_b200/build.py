"""Build the CUDA library in-tree: semiimplicitfv_b200/libsifv_b200.so.

nvcc -gencode arch=compute_100a,code=sm_100a, FP64 kernels compiled with
--fmad=false so the parity path evaluates every expression exactly as the
reference writes it (no contraction into FMA).
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libsifv_b200.so")
# (source, extra flags): the reference-ordered kernels are compiled without
# FMA contraction; the fused sweep path (sifv_fast.cu) with it.
SOURCES = [("sifv_capi.cu", ["--fmad=false"]), ("sifv_noalloc.cu", ["--fmad=false"]),
           ("sifv_fast.cu", ["--fmad=true"]), ("sifv_ensemble.cu", ["--fmad=false"]),
           ("sifv_ensemble_mixed.cu", ["--fmad=true", "--use_fast_math"]), ("sifv_adjoint.cu", ["--fmad=true"]),
           ("sifv_vtk.cpp", []), ("sifv_ib.cpp", ["-Xcompiler", "-ffp-contract=off"])]
HEADERS = ["sifv_device.cuh", "sifv_common.cuh", "sifv_kernels.cuh", "sifv_sweep.cuh", "sifv_sweep_api.h",
           "sifv_ensemble.cuh", "sifv_ensemble_api.h", "sifv_adjoint.cuh", "sifv_adjoint_api.h", "sifv_dual.cuh", "sifv_march2d.cuh", "sifv_fastmath.cuh", "sifv_vtk_api.h", "sifv_ib_api.h",
           "sifv_mg.cuh", "sifv_gs_march.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f, _ in SOURCES] + [os.path.join(CSRC, f) for f in HEADERS] + \
        [os.path.join(ROOT, "include", "sifv.h"), os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    import concurrent.futures as cf
    objdir = os.path.join(ROOT, "_build", "csrc")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    cmds, objs = [], []
    for src, extra in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmds.append([_nvcc(), *NVCC_FLAGS, *extra, *inc, "-c", os.path.join(CSRC, src), "-o", obj])
    with cf.ThreadPoolExecutor(len(cmds)) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
        list(ex.map(lambda c: subprocess.run(c, check=True), cmds))
    link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
