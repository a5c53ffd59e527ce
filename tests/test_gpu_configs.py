"""GPU parity on the benchmark workloads at their own sizes and horizons.

The fixtures (tests/golden/cfg_*.npz, made by tests/golden/make_golden_configs.py
from GO-Ferro's own solver, serial on the host) cover:

* the FM LLG + FFT magnetostatics workload, 64x64x16, all 4000 steps;
* the coupled magnetoelastic + elastodynamics + FDTD workload: a 32x32x24
  copy of its layer stack over all 10000 steps, and the full 128x128x96 grid
  over its first 200 steps;
* the ferroelectric TDGL + electrostriction + elastodynamics + FDTD workload:
  a 16x16x32 copy over the 20000-step relaxation plus 20000 steps under the
  sheet current, and the full 128^3 grid over its first 200 steps.

FP64 form: every traced observable (<m>, <p>, <u>, the probed cell's E and H)
within 1e-10 of the reference relative to that observable's largest
component over the trace, and the committed final fields within 1e-10 of
their largest component.

FP32 mixed form: the same traces within 1e-5 relative to the magnitude of
the field each observable samples: for <m>, <p> and <u> the largest cell
value of the field (the average of +-1e-3 random P is ~1e-5, and an FP32
field's rounding is relative to its cells, not to their mean); for the probed
E and H the electromagnetic field's scale max(|E|, eta0 |H|) over the trace
(in a quasi-static E of 1e6 V/m the probed H is a few A/m, a small
difference of FP32 E values).  The error relative to each observable's own
trace magnitude is printed beside it.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CONFIGS = json.load(open(os.path.join(GOLDEN, "configs.json")))
TOL = {"fp64": 1e-10, "mixed": 1e-5}
ETA0 = 376.730313668

# trace columns of each vector observable (oracle/refrun.TRACE_COLS)
GROUPS = {"m": (1, 4), "m_afm1": (4, 7), "m_afm2": (7, 10), "p": (10, 13), "u": (13, 16), "E": (16, 19), "H": (19, 22)}
FIELDS = {"m": ("mx", "my", "mz"), "p": ("px", "py", "pz"), "u": ("ux", "uy", "uz")}


def make_deck(gf, name):
    preset, kw, steps, every, probe, keep = CONFIGS[name]
    return gf.decks.PRESETS[preset](**kw), steps, every, probe, keep


def engine_trace(eng, steps, every, probe):
    """Trace rows at steps 0, every, 2*every, ... in the oracle's columns."""
    rows = []
    for s in range(0, steps + 1, every):
        if s:
            eng.advance(every)
        row = np.zeros(22)
        row[0] = s
        if eng.info.fm:
            row[1:4] = eng.average("m")
        if eng.info.afm:
            row[4:7] = eng.average("m_afm1")
            row[7:10] = eng.average("m_afm2")
        if eng.info.fe:
            row[10:13] = eng.average("p")
        if eng.info.elastic:
            row[13:16] = eng.average("u")
        if eng.info.em:
            e, h = eng.probe_em(*probe)
            row[16:19] = e
            row[19:22] = h
        rows.append(row)
    return np.array(rows)


def field_scale_errors(mine, ref, field_max):
    """{observable: max error relative to the sampled field's magnitude}"""
    out = {}
    em = float(np.max(np.maximum(np.max(np.abs(ref[:, 16:19]), axis=1), ETA0 * np.max(np.abs(ref[:, 19:22]), axis=1))))
    for name, (a, b) in GROUPS.items():
        own = float(np.max(np.abs(ref[:, a:b])))
        if own == 0.0:
            continue
        if name in ("E",):
            scale = em
        elif name == "H":
            scale = em / ETA0
        else:
            scale = max(own, field_max.get(name, 0.0))
        out[name] = float(np.max(np.abs(mine[:, a:b] - ref[:, a:b]))) / scale
    return out


def trace_errors(mine, ref):
    """{observable: (max relative error, first traced step above 1e-10)}"""
    assert mine.shape == ref.shape, (mine.shape, ref.shape)
    assert np.array_equal(mine[:, 0], ref[:, 0])
    out = {}
    for name, (a, b) in GROUPS.items():
        scale = float(np.max(np.abs(ref[:, a:b])))
        if scale == 0.0:
            assert float(np.max(np.abs(mine[:, a:b]))) == 0.0, f"{name}: expected zeros"
            continue
        err = np.max(np.abs(mine[:, a:b] - ref[:, a:b]), axis=1) / scale
        above = np.nonzero(err > 1e-10)[0]
        out[name] = (float(err.max()), int(ref[above[0], 0]) if above.size else None)
    return out


@pytest.mark.parametrize("form", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_config_matches_reference(gf, tmp_path, name, form):
    d, steps, every, probe, keep = make_deck(gf, name)
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    ref = g["trace"]
    init = {}
    # the initial state is uploaded, not written as text, for the large grids
    if d.m0 is not None and d.n > 300_000:
        init["m"], d.m0 = d.m0, None
    if d.p0 is not None and d.n > 300_000:
        init["p"], init["q"], d.p0 = d.p0, d.q0, None
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0, precision=form) as eng:
        for k, v in init.items():
            eng.upload(k, v)
        mine = engine_trace(eng, steps, every, tuple(probe) if probe else (0, 0, 0))
        errs = trace_errors(mine, ref)
        print(name, form, "own scale:", {k: f"{v[0]:.2e} (first step > 1e-10: {v[1]})" for k, v in errs.items()})
        if form == "fp64":
            for obs, (e, _) in errs.items():
                assert e <= TOL[form], f"{name} {form} <{obs}>: rel err {e:.3e}"
        else:
            fmax = {}
            for obs, on in (("m", eng.info.fm), ("p", eng.info.fe), ("u", eng.info.elastic)):
                if on:
                    fmax[obs] = float(np.max(np.abs(eng.download(obs))))
            ferr = field_scale_errors(mine, ref, fmax)
            print(name, form, "field scale:", {k: f"{v:.2e}" for k, v in ferr.items()})
            for obs, e in ferr.items():
                assert e <= TOL[form], f"{name} {form} <{obs}>: error {e:.3e} of the field's magnitude"
        if form == "fp64":
            for fld, parts in FIELDS.items():
                if parts[0] not in g.files:
                    continue
                mf = eng.download(fld)
                scale = max(float(np.max(np.abs(g[p]))) for p in parts)
                for c, p in enumerate(parts):
                    err = float(np.max(np.abs(mf[c].ravel() - g[p]))) / scale
                    assert err <= TOL[form], f"{name} final {p}: rel err {err:.3e}"
        eng.check_finite()
