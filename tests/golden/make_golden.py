"""Generate the golden fixtures of tests/golden/ by running GO-Ferro's own
solver (the oracle build, oracle/_ref/goferro_ref, compiled from the
reference sources) on small seeded decks.

    python tests/golden/make_golden.py

Each fixture <name>.npz holds the full-precision trace (step, <m>, <m_AFM1>,
<m_AFM2>, <p>, <u>, E_cell and H_cell at the probe cell) and the final
fields the oracle dumps; the deck itself is regenerated from the preset
parameters stored alongside (decks.py is deterministic).
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402
from oracle import refrun  # noqa: E402

gf = __graft_entry__.import_package()

# name -> (preset, kwargs, steps, probe, source scale)
CASES = {
    "fm_demag_16x16x8": ("fm_demag", dict(nx=16, ny=16, nz=8, steps=60), 60, None, 1.0),
    "magnetoelastic_8x16x12": ("magnetoelastic", dict(nx=8, ny=16, nz=12, sub=5, film=4, steps=40), 40, (4, 8, 7), 1e6),
    "magnetoelastic_quirk_8x8x12": ("magnetoelastic", dict(nx=8, ny=8, nz=12, sub=5, film=4, steps=40), 40, (4, 4, 7), 1e6),
    "ferroelectric_8x8x10": ("ferroelectric", dict(nx=8, ny=8, nz=10, steps=40), 40, (4, 4, 5), 1.0),
}


def make_deck(name):
    preset, kw, steps, probe, scale = CASES[name]
    d = gf.decks.PRESETS[preset](**kw)
    d.amp_gauss *= scale
    d.jf_amp *= scale
    return d, steps, probe


def main():
    for name in CASES:
        d, steps, probe = make_deck(name)
        with tempfile.TemporaryDirectory() as tmp:
            gf.decks.write_deck(d, os.path.join(tmp, "deck"))
            r = refrun.run(os.path.join(tmp, "deck"), os.path.join(tmp, "out"), steps=steps, probe=probe, dump=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), trace=r["trace"], **r["fields"])
        print(name, r["trace"].shape, sorted(r["fields"]))
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump({k: [v[0], v[1], v[2], v[3], v[4]] for k, v in CASES.items()}, f, indent=1)


if __name__ == "__main__":
    main()
