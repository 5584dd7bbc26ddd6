"""Build libfsi_b200.so (the C ABI declared in include/fsi_b200.h) in-tree.

The library is compiled for sm_100a only, with nvcc, into
mpm_lbm_b200/_build/libfsi_b200.so; it travels with the repository snapshot
(it is git-ignored, not copied anywhere else).  Usage::

    python -m mpm_lbm_b200.build [--force]
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libfsi_b200.so")
SOURCES = ["fsi_abi.cu", "lbm_kernels.cu", "mpm_kernels.cu", "mpm_binned.cu"]
HEADERS = ["common.cuh", "d3q19.cuh", "polar3.cuh", "mpm_common.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "fsi_b200.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [_nvcc(), *ARCH, *FLAGS, "-c", s, "-o", o + ".tmp"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            os.replace(o + ".tmp", o)
    if force or _stale(LIB, objs):
        tmp = LIB + f".tmp{os.getpid()}"
        cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=True))


if __name__ == "__main__":
    sys.exit(main())
