"""Run the reference oracle (GO-Ferro's own sources built into
oracle/_ref/goferro_ref by oracle/Makefile) on a deck directory and read back
its full-precision traces and final fields.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker / the timed CPU reference.
"""
from __future__ import annotations

import json
import os
import subprocess
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "goferro_ref")

TRACE_COLS = ["step", "mx", "my", "mz", "m1x", "m1y", "m1z", "m2x", "m2y", "m2z",
              "px", "py", "pz", "ux", "uy", "uz", "Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]


def available() -> bool:
    return os.path.exists(REF_BIN)


def build(ref_dir: Optional[str] = None) -> None:
    """Compile the oracle (needs the reference sources; run where they exist).
    ref_dir: the reference source tree; default $GOFERRO_REF_DIR, else the
    Makefile's default."""
    ref_dir = ref_dir or os.environ.get("GOFERRO_REF_DIR")
    args = [f"REF_DIR={ref_dir}"] if ref_dir else []
    subprocess.run(["make", "-C", HERE] + args + ["-j8"], check=True,
                   stdout=subprocess.DEVNULL)


def run(deck_dir: str, out_dir: str, steps: Optional[int] = None, trace_every: int = 1,
        probe: Optional[Sequence[int]] = None, dump: bool = False, timeout: float = 3600.0,
        warmup: int = 0, outputs: bool = False) -> Dict:
    """Run the reference on `deck_dir`; returns {"trace": (K,22) array,
    "timing": {...}, "fields": {name: flat float64 array}}.  With outputs,
    the reference's own text outputs (its deck's if_output_* schedule) are
    written into out_dir as well."""
    if not available():
        raise RuntimeError(f"oracle binary missing: {REF_BIN}")
    os.makedirs(out_dir, exist_ok=True)
    cmd = [REF_BIN, os.path.abspath(deck_dir), os.path.abspath(out_dir), "--trace-every", str(trace_every)]
    if steps is not None:
        cmd += ["--steps", str(int(steps))]
    if warmup:
        cmd += ["--warmup", str(int(warmup))]
    if probe is not None:
        cmd += ["--probe"] + [str(int(x)) for x in probe]
    if dump:
        cmd += ["--dump"]
    if outputs:
        cmd += ["--outputs"]
    subprocess.run(cmd, check=True, timeout=timeout, stdout=subprocess.DEVNULL)
    trace = np.loadtxt(os.path.join(out_dir, "trace.txt"), ndmin=2)
    with open(os.path.join(out_dir, "timing.json")) as f:
        timing = json.load(f)
    fields = {}
    if dump:
        for fn in os.listdir(out_dir):
            if fn.endswith(".bin"):
                fields[fn[:-4]] = np.fromfile(os.path.join(out_dir, fn), dtype=np.float64)
    return {"trace": trace, "timing": timing, "fields": fields}
