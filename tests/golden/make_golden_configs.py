"""Generate the named-configuration parity fixtures of tests/golden/ by running
GO-Ferro's own solver (the oracle build, oracle/_ref/goferro_ref, compiled
from the reference sources, serial on the host) on the benchmark workloads at
their own sizes and horizons, or on reduced copies of them run for the full
horizon:

* fm_demag 64x64x16, 4000 steps: the CPU-runnable FM LLG + FFT
  magnetostatics workload in full (trace every step, final m);
* magnetoelastic 32x32x24 (the 56/32/8 layer stack scaled to 14/8/2),
  10000 steps, and the full 128x128x96 grid for its first 200 steps;
* ferroelectric 16x16x32, 40000 steps (the 20000-step relaxation from
  +-1e-3 random P plus 20000 further steps under the type-4 sheet current),
  and the full 128^3 grid for its first 200 steps.

    python tests/golden/make_golden_configs.py [name ...]   # default: all

Each fixture <name>.npz holds the full-precision trace (columns as
oracle/refrun.TRACE_COLS, every `trace_every`-th step) and, for the grids
small enough to commit, the final fields listed in the case.  The serial
reference needs about 40 minutes for the 64x64x16 run and about an hour for
each of the others; cases run in parallel processes.
"""
import json
import os
import sys
import tempfile
import multiprocessing
from concurrent.futures import ProcessPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# name -> (preset, kwargs, steps, trace_every, probe, kept final fields)
CONFIGS = {
    "cfg_fm_demag_64x64x16_4000": (
        "fm_demag", dict(), 4000, 1, None, ["mx", "my", "mz"]),
    "cfg_magnetoelastic_32x32x24_10000": (
        "magnetoelastic", dict(nx=32, ny=32, nz=24, sub=14, film=8, steps=10000), 10000, 10, (16, 16, 18),
        ["mx", "my", "mz", "ux", "uy", "uz"]),
    "cfg_magnetoelastic_128x128x96_200": (
        "magnetoelastic", dict(steps=200), 200, 1, (64, 64, 70), []),
    "cfg_ferroelectric_16x16x32_40000": (
        "ferroelectric", dict(nx=16, ny=16, nz=32, steps=40000), 40000, 10, (8, 8, 16),
        ["px", "py", "pz", "ux", "uy", "uz"]),
    "cfg_ferroelectric_128x128x128_200": (
        "ferroelectric", dict(steps=200), 200, 1, (64, 64, 64), []),
}


def make_deck(gf, name):
    preset, kw, steps, every, probe, keep = CONFIGS[name]
    return gf.decks.PRESETS[preset](**kw), steps, every, probe, keep


def run_case(name):
    import __graft_entry__
    from oracle import refrun
    gf = __graft_entry__.import_package()
    d, steps, every, probe, keep = make_deck(gf, name)
    with tempfile.TemporaryDirectory() as tmp:
        gf.decks.write_deck(d, os.path.join(tmp, "deck"))
        r = refrun.run(os.path.join(tmp, "deck"), os.path.join(tmp, "out"), steps=steps, trace_every=every,
                       probe=probe, dump=bool(keep), timeout=6 * 3600.0)
    fields = {k: r["fields"][k] for k in keep}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), trace=r["trace"], **fields)
    return name, r["trace"].shape, r["timing"]


def main(names):
    names = names or list(CONFIGS)
    with ProcessPoolExecutor(max_workers=len(names), mp_context=multiprocessing.get_context("spawn")) as ex:
        for name, shape, timing in ex.map(run_case, names):
            print(name, shape, timing, flush=True)
    with open(os.path.join(HERE, "configs.json"), "w") as f:
        json.dump({k: list(v) for k, v in CONFIGS.items()}, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
