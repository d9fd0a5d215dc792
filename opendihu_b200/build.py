"""Build libfdm_b200.so in-tree with nvcc for sm_100a.

The CUDA translation units are compiled in parallel into ``_build/`` at the repository root and
linked into ``opendihu_b200/libfdm_b200.so`` (the file the ctypes loader opens).  Device code uses
the default FMA contraction; host code is compiled with ``-ffp-contract=off`` because it evaluates
the reference's time arithmetic, whose discrete stimulation decisions must match the C expressions
exactly.  FP32 division/sqrt use the fast approximate forms (FP32 is only used by the reaction
right-hand side in the FP32-reaction mode).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libfdm_b200.so")

SOURCES = ["fdm_host.cu", "fdm_kernels_split.cu", "fdm_fused.cu", "fdm_fused_f64_exact.cu", "fdm_fused_f64_approx.cu",
           "fdm_fused_f32_exact.cu", "fdm_fused_f32_approx.cu", "fdm_fused_f64_exact_gate.cu",
           "fdm_fused_f64_approx_gate.cu", "fdm_fused_f32_exact_gate.cu", "fdm_fused_f32_approx_gate.cu",
           "fdm_fused_cluster_f32.cu", "fdm_fused_cluster_f64.cu", "fdm_noalloc.cu", "fdm_emg.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                     "-prec-div=false", "-prec-sqrt=false", "-ftz=true",
                     "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libfdm_b200.so")


def _deps(src: str) -> List[str]:
    out = [os.path.join(CSRC, src)]
    for d in (CSRC, os.path.join(CSRC, "generated")):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "fdm_b200.h"))
    return out


def _stale(target: str, deps: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    if not _stale(obj, _deps(src)):
        return obj
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for src in SOURCES:
            obj = os.path.join(BUILD, src.replace(".cu", ".o"))
            if os.path.exists(obj):
                os.remove(obj)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
