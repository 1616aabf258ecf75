"""Builds libgsw.so (the C ABI of include/gsw.h) for sm_100a, in-tree."""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(HERE, "libgsw.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "**", "*.cu*"), recursive=True) +
                  glob.glob(os.path.join(HERE, "csrc", "**", "*.h"), recursive=True) +
                  [os.path.join(ROOT, "include", "gsw.h")])


def stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if force or stale(SO):
        cmd = [NVCC, *ARCH, *FLAGS, "-o", SO + ".tmp", os.path.join(HERE, "csrc", "gsw_capi.cu"),
               os.path.join(HERE, "csrc", "gsw_noalloc.cu")]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        os.replace(SO + ".tmp", SO)
    return SO


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
