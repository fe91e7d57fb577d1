"""Build libexciting_b200.so in-tree with nvcc for sm_100a.

The library is a plain C-ABI shared object (no Python or torch types in its
interface); Python reaches it through ctypes (exciting_b200/abi.py), a Fortran
host through iso_c_binding.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libexciting_b200.so")

SOURCES = ["exs_api.cu", "match.cu", "setup_f64.cu", "ozaki.cu", "forcek.cu", "noalloc.cu", "interstitial.cu", "solve.cu", "mtint.cu", "rttddft.cu", "pmat.cu", "wavefmt.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"]


LIBS = ["-lcusolver", "-lcublas"]          # the device eigen-solve (solve.cu)


def nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.sep not in p or os.path.exists(p)):
            return p
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "exciting_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, extra=None) -> str:
    cmd = [nvcc(), *ARCH, *FLAGS, *(extra or []), "-o", LIB, *sources(), *LIBS]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(verbose=True, extra=extra))
