"""Build recipe for the reference harness (test infrastructure, not product).

Copies the reference's ``LettuceGauge/`` headers from the read-only reference checkout into
``oracle/_ref/src/`` (git-ignored), replaces the compile-time lattice extents of
``LettuceGauge/defines.hpp:34-37`` by the macros ``LT_NT``..``LT_NZ``, and compiles
``oracle/ref_harness.cpp`` once per extent tuple into ``oracle/_ref/liblt_ref_<T>x<X>x<Y>x<Z>.so``.
The reference's own build system (Makefile) is not used.  Eigen and PCG are taken from
where they lie in the reference checkout.

Besides these parity builds (``-ffp-contract=off``, a fixed x86-64-v3 target), the CPU
baseline is timed on ``oracle/_ref/liblt_ref_fast_<ext>_<isa>.so``: the same harness compiled
with the optimisation of the reference Makefile (``Makefile:89``: ``-O3 -DNDEBUG
-fno-math-errno -fopenmp``, ``-march=native``) with floating-point contraction on.  The GPU
hosts are not this machine, so ``-march=native`` is built for both x86-64-v4 (AVX-512) and
x86-64-v3 (AVX2) and the bench loads the best one the running host supports.

The reference checkout is found at ``$LETTUCE_REFERENCE`` (default: the read-only checkout
of this build environment).

Usage: python oracle/build_ref.py [--ref DIR] [--extents 4x4x4x4 8x8x8x8 ...] [--fast]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")

# 4^4 and 4x6x8x10: golden fixtures; 8^4: the CPU-runnable plain config; 16^4: the MetaD
# config; 12^4: the tempering streams; 32^4: the large plain-vs-FP32 config (CPU baseline).
DEFAULT_EXTENTS = ["4x4x4x4", "4x6x8x10", "8x8x8x8", "12x12x12x12", "16x16x16x16", "32x32x32x32"]

# Flags follow the reference Makefile's optimisation level (Makefile:89: -O3 -fno-math-errno),
# with an explicit x86-64-v3 target instead of -march=native so the library also runs on
# the GPU hosts, and -ffp-contract=off so results do not depend on FMA contraction.
CXXFLAGS = ["-std=c++20", "-O3", "-DNDEBUG", "-fno-math-errno", "-march=x86-64-v3",
            "-ffp-contract=off", "-fopenmp", "-DFIXED_SEED", "-fPIC", "-shared", "-w"]

# The timing builds: the reference Makefile's optimisation with contraction on, per ISA level
FAST_EXTENTS = ["32x32x32x32", "16x16x16x16"]
FAST_ISAS = {"v4": "-march=x86-64-v4", "v3": "-march=x86-64-v3"}
FAST_CXXFLAGS = ["-std=c++20", "-O3", "-DNDEBUG", "-fno-math-errno", "-ffp-contract=fast", "-fopenmp",
                 "-DFIXED_SEED", "-fPIC", "-shared", "-w"]


def default_reference() -> str:
    return os.environ.get("LETTUCE_REFERENCE", "/root/reference")


def lib_name(ext: str) -> str:
    return os.path.join(OUT, f"liblt_ref_{ext}.so")


def stage_sources(ref: str) -> None:
    dst = os.path.join(SRC, "LettuceGauge")
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    os.makedirs(SRC, exist_ok=True)
    shutil.copytree(os.path.join(ref, "LettuceGauge"), dst)
    for sub in ("PCG", "Eigen_3.4"):
        link = os.path.join(SRC, sub)
        if os.path.islink(link) or os.path.exists(link):
            os.remove(link) if os.path.islink(link) else shutil.rmtree(link)
        os.symlink(os.path.join(ref, sub), link)
    defines = os.path.join(dst, "defines.hpp")
    os.chmod(defines, 0o644)
    text = open(defines).read()
    for name, macro in (("Nt", "LT_NT"), ("Nx", "LT_NX"), ("Ny", "LT_NY"), ("Nz", "LT_NZ")):
        text, n = re.subn(r"inline constexpr int %s\s*\{\d+\};" % name,
                          "inline constexpr int %s {%s};" % (name, macro), text)
        if n != 1:
            raise RuntimeError(f"could not patch extent {name} in defines.hpp")
    open(defines, "w").write(text)


def fast_lib_name(ext: str, isa: str) -> str:
    return os.path.join(OUT, f"liblt_ref_fast_{ext}_{isa}.so")


def build_one(job) -> str:
    ext, isa = job
    t, x, y, z = (int(v) for v in ext.split("x"))
    flags = CXXFLAGS if isa is None else [*FAST_CXXFLAGS, FAST_ISAS[isa]]
    out = lib_name(ext) if isa is None else fast_lib_name(ext, isa)
    cmd = ["g++", *flags, f"-DLT_NT={t}", f"-DLT_NX={x}", f"-DLT_NY={y}", f"-DLT_NZ={z}",
           "-I", SRC, "-I", os.path.join(SRC, "Eigen_3.4"),
           os.path.join(HERE, "ref_harness.cpp"), "-o", out]
    subprocess.run(cmd, check=True)
    return out


def build(ref: str | None = None, extents=None, force: bool = False, fast: bool = True) -> list[str]:
    ref = ref or default_reference()
    extents = list(extents or DEFAULT_EXTENTS)
    if not os.path.isdir(os.path.join(ref, "LettuceGauge")):
        raise FileNotFoundError(f"reference checkout not found at {ref}")
    harness = os.path.join(HERE, "ref_harness.cpp")
    jobs = [(e, None) for e in extents]
    if fast:
        jobs += [(e, isa) for e in FAST_EXTENTS if e in extents for isa in FAST_ISAS]
    outs = [lib_name(e) if isa is None else fast_lib_name(e, isa) for e, isa in jobs]
    todo = [j for j, o in zip(jobs, outs) if force or not os.path.exists(o)
            or os.path.getmtime(o) < os.path.getmtime(harness)]
    if not todo:
        return outs
    stage_sources(ref)
    with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 1)) as pool:
        list(pool.map(build_one, todo))
    return outs


def reference_present() -> bool:
    return os.path.isdir(os.path.join(default_reference(), "LettuceGauge"))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    ap.add_argument("--extents", nargs="*", default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-fast", action="store_true", help="skip the timing builds")
    a = ap.parse_args()
    for p in build(a.ref, a.extents, a.force, fast=not a.no_fast):
        print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
