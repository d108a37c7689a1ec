"""Build recipe for the C-ABI library lettuce_b200/liblettuce_b200.so (sm_100a).

Each translation unit is compiled by nvcc in parallel and linked into one shared library
with the CUDA runtime linked statically, so the library has no dependency beyond the driver.

Usage: python -m lettuce_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblettuce_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-I", CSRC, "-I", INCLUDE]

SOURCES = ["lt_impl_fp64.cu", "lt_impl_fp32.cu", "lt_impl_fp32_12.cu", "lt_capi.cu", "lt_ensemble.cu", "lt_host.cpp",
           "lt_noalloc.cu", "lt_bmw.cu", "lt_selftest.cu"]
HEADERS = ["lt_math.cuh", "lt_field.cuh", "lt_kernels.cuh", "lt_impl.cuh", "lt_backend.h", "lt_host.h", "lt_handle.h"]


def _newest_input() -> float:
    paths = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    paths.append(os.path.join(INCLUDE, "lettuce_b200.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(lambda s: _compile(s, verbose), SOURCES))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
