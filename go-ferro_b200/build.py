"""Build libgoferro_b200.so in-tree for sm_100a with nvcc.

    python go-ferro_b200/build.py

Two CUDA translation units: gf_engine.cu (the FP64 parity kernels, the host
engine and the C ABI) is compiled with -fmad=false, so that every multiply
and add is rounded as in the reference's host build; gf_mixed.cu (the FP32
mixed-form stage kernels) is compiled with FMA contraction.  The library
links cuFFT for the magnetostatic transforms.
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

# (source, extra flags): each compiled to its own object, then linked
UNITS = [("gf_engine.cu", ["-fmad=false"]), ("gf_mixed.cu", ["-fmad=true"]), ("gf_deck.cpp", [])]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I" + os.path.join(ROOT, "include")]


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
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    cmds, objs = [], []
    for src, extra in UNITS:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        cmds.append([nvcc()] + ARCH + FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj])
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
    if any(p.wait() != 0 for p in procs):
        raise subprocess.CalledProcessError(1, "nvcc")
    link = [nvcc()] + ARCH + ["-shared"] + objs + ["-lcufft", "-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
