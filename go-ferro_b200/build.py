"""Build libgoferro_b200.so in-tree for sm_100a with nvcc.

    python go-ferro_b200/build.py

The FP64 parity kernels are compiled with -fmad=false (no contraction of
multiply-add pairs) so that every operation is rounded as in the reference's
host build; the library links cuFFT for the magnetostatic transforms.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgoferro_b200.so")

SOURCES = ["gf_engine.cu", "gf_deck.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-O2", "-shared",
         "-I" + os.path.join(ROOT, "include")]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def newest_input_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "goferro_b200.h"), __file__]
    return max(os.path.getmtime(p) for p in paths)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest_input_mtime():
        return OUT
    cmd = [nvcc()] + ARCH + FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcufft", "-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
