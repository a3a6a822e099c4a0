"""Build the in-tree shared library ``tbfsolver_b200/lib/libtbfp.so`` for sm_100a.

    python -m tbfsolver_b200.build [--force]

nvcc cross-compiles without a GPU.  Each source compiles to an object in
parallel (the transform kernels are specialised per length, so the files are
heavy), then nvcc links the shared library.  The CUDA runtime is linked
statically (nvcc's default), so the library does not depend on the CUDA
runtime that a host process (e.g. PyTorch) has loaded.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib", "libtbfp.so")
SOURCES = ["tbfp_api.cu", "tbfp_xfft.cu", "tbfp_yz.cu", "tbfp_correct.cu", "tbfp_mg.cu", "tbfp_noalloc.cu", "tbfp_vof.cu", "tbfp_momentum.cu", "tbfp_flow.cu", "tbfp_ensemble.cu", "tbfp_surface.cu", "tbfp_correct_tma.cu"]
HEADERS = ["tbfp_kernels.cuh", "tbfp_stages.cuh", "fft_smem.cuh", "tbfp_mg.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
OBJ_DIR = os.path.join(PKG, "_build")


def _inputs():
    return [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "tbfp.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include")]
    objs = [os.path.join(OBJ_DIR, os.path.splitext(f)[0] + ".o") for f in SOURCES]

    def compile_one(src_obj):
        src, obj = src_obj
        cmd = [NVCC, *ARCH, *FLAGS, *inc, "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, zip(SOURCES, objs)))
    for src, r in zip(SOURCES, results):
        if r.stdout or r.stderr:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, f"nvcc {src}")
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
