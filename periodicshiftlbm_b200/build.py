"""Build the CUDA library (sm_100a) in-tree, plus the CPU checkers under oracle/.

    python -m periodicshiftlbm_b200.build

* ``periodicshiftlbm_b200/libpsl_b200.so`` -- every kernel and the C ABI of include/psl.h,
  compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a`` (cross-compiles without
  a GPU).
* ``oracle/liboracle.so`` and, when the reference checkout is present,
  ``oracle/_ref/libpsl_ref.so`` (``make -C oracle``): test infrastructure only.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpsl_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-shared", "-Xcompiler", "-fPIC",
]
SOURCES = [os.path.join(CSRC, "psl_capi.cu"), os.path.join(CSRC, "psl_noalloc.cu"), os.path.join(CSRC, "psl_batch.cu"),
           os.path.join(CSRC, "psl_learned.cu"),
           os.path.join(CSRC, "psl_train.cu"),
           os.path.join(CSRC, "psl_reports.cu"),
           os.path.join(CSRC, "psl_rowmap.cu")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the library")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile each translation unit to an object in parallel (one nvcc per file), then
    link the shared library."""
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", "psl.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    incs = ["-I", os.path.join(REPO, "include"), "-I", CSRC]

    def compile_one(src: str) -> str:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [_nvcc(), *compile_flags, *incs, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def reference_checkout() -> str | None:
    """The reference checkout the CPU checker is compiled from: PSL_REFERENCE_DIR, else the
    location the build machine keeps it at; None where neither exists (a GPU box uses the
    prebuilt oracle/_ref)."""
    for cand in (os.environ.get("PSL_REFERENCE_DIR"), "/root/reference"):
        if cand and os.path.isdir(os.path.join(cand, "include")):
            return cand
    return None


def build_oracle(verbose: bool = False) -> None:
    """The CPU checkers (test infrastructure): liboracle.so and, if the reference
    checkout exists on this machine, oracle/_ref/libpsl_ref.so."""
    cmd = ["make", "-s", "-C", os.path.join(REPO, "oracle"), "all"]
    ref = reference_checkout()
    if ref:
        cmd.append(f"REF={ref}")
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> None:
    build_library(force=force, verbose=verbose)
    build_oracle(verbose=verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
