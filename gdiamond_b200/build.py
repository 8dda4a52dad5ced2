"""Builds gdiamond_b200/libgdiamond_b200.so in-tree with nvcc for sm_100a.

    python -m gdiamond_b200.build            # incremental
    python -m gdiamond_b200.build --force    # rebuild everything
    python -m gdiamond_b200.build --verbose  # also print ptxas register/spill reports
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgdiamond_b200.so")
SOURCES = ["fdtd_capi.cu", "k_naive.cu", "k_tiled.cu", "k_tiled2.cu", "k_tiled2_f32.cu", "k_tiled2_f16.cu", "k_tiled2_bf16.cu", "k_tiled2_f16e.cu", "convert.cu", "coefs.cu", "materials.cu", "materials_noalloc.cu", "mlp.cu", "mlp_tc.cu", "dft_fold.cu", "flux.cu", "cpml.cu"]
HEADERS = ["fdtd_common.cuh", "fdtd_kernels.cuh", "k_tiled2.cuh", "mlp.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> tuple[str, str]:
    obj = os.path.join(OBJ, src.replace(".cu", ".o"))
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
        ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "fdtd_capi.h")]
    todo = []
    for s in SOURCES:
        obj = os.path.join(OBJ, s.replace(".cu", ".o"))
        if force or verbose or _stale(obj, [os.path.join(CSRC, s)] + hdrs):
            todo.append(s)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for obj, log in ex.map(lambda s: _compile(s, verbose), todo):
            if verbose and log:
                sys.stderr.write(log)
    objs = [os.path.join(OBJ, s.replace(".cu", ".o")) for s in SOURCES]
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
