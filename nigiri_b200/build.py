"""Builds the engine library nigiri_b200/libb2r.so (sm_100a) in-tree.

    python -m nigiri_b200.build [--oracle]

The CUDA sources are compiled for sm_100a only; host sources with the same
nvcc driver.  The CUDA runtime is linked statically so the library has no
run-time dependency beyond the driver.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++20", "-O3", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
          "-I" + CSRC]
CU_FLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(out, deps):
    return os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps)


def build_lib(force=False, verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith((".cc", ".cu")))
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(ROOT, "include", "b2r.h"))
    objs = []
    for f in srcs:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if not force and _newer(obj, [src] + hdrs):
            continue
        flags = COMMON + (CU_FLAGS if f.endswith(".cu") else ["-x", "c++"])
        if verbose_ptxas and f.endswith(".cu"):
            flags = flags + ["-Xptxas", "-v"]
        _run([NVCC] + flags + ["-c", src, "-o", obj])
    out = os.path.join(HERE, "libb2r.so")
    if force or not _newer(out, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", out] + objs + ["-lpthread"])
    return out


def build_oracle(force=False):
    """The CPU oracle (test infrastructure): oracle/liboracle.so."""
    src = os.path.join(ROOT, "oracle", "oracle.cc")
    out = os.path.join(ROOT, "oracle", "liboracle.so")
    deps = [src, os.path.join(ROOT, "oracle", "oracle.h"), os.path.join(ROOT, "include", "b2r.h")]
    if force or not _newer(out, deps):
        _run(["g++", "-std=c++20", "-O3", "-ffp-contract=off", "-fPIC", "-shared",
              "-I" + os.path.join(ROOT, "include"), "-o", out, src, "-lpthread"])
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    build_lib(force=force, verbose_ptxas="--ptxas-v" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle(force=force)
