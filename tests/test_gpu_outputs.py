"""GPU tests of the reference's text outputs (gf_write_outputs / gf_run_deck).

The reference writes its outputs with inoutput.cpp on main.cpp's schedule;
the oracle does the same with the reference's own writers (--outputs), so
each deck is run both ways and every file the reference writes must exist
with the same name, the same lines and columns in the same printf layout,
and values that agree to the %.7e print resolution of each column (the
FP64 engine follows the reference to ~1e-12, so a printed value differs at
most in its last digit when the two sides straddle a rounding boundary)."""
import dataclasses
import os
import re

import numpy as np
import pytest

from test_gpu_parity import _variants

pytestmark = pytest.mark.gpu
NUM = re.compile(r"[-+]?\d+(\.\d+)?(e[-+]\d+)?")


def _decks(gf):
    D = gf.decks
    v = {}
    d = D.preset_ferroelectric(nx=6, ny=5, nz=12, steps=8)
    d.outputs = {"ave": 2, "p": 4, "q": 4, "em": 4, "em_onecell": 2, "emYee": 8, "strain": 4, "uv": 8,
                 "force": 8, "Estat": 8, "eig0": 8}
    d.em_onecell_index = 37
    v["ferroelectric"] = d
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=8)
    d.amp_gauss *= 1e6
    d.outputs = {"ave": 1, "m": 4, "magcell": 8, "Hstat": 4, "uv": 8, "strain": 8, "em": 8, "emYee": 8}
    v["magnetoelastic"] = d
    var = _variants(gf)
    d = dataclasses.replace(var["afm_film_demag"][0], steps=6)
    d.outputs = {"ave": 3, "AFMm": 6, "m": 6, "Hstat": 6}
    v["afm"] = d
    d = dataclasses.replace(var["drude_metal_layer"][0], steps=6)
    d.outputs = {"Jp": 3, "em": 6, "ave": 2}
    v["drude"] = d
    # the 1-D magnetostatic model's cell H_z in the EM outputs
    d = dataclasses.replace(var["mag_1d_maxwell"][0], steps=8)
    d.outputs = {"ave": 2, "em": 4, "em_onecell": 2, "m": 8}
    d.em_onecell_index = 703     # (3, 10, 6), inside the film
    v["mag_1d_maxwell"] = d
    return v


def _compare(path_ref, path_mine):
    with open(path_ref) as f:
        ref = f.read().splitlines()
    with open(path_mine) as f:
        mine = f.read().splitlines()
    assert len(ref) == len(mine), (path_ref, len(ref), len(mine))
    # the same layout: each line with its numbers blanked is identical
    for a, b in zip(ref[:50], mine[:50]):
        assert NUM.sub("N", a) == NUM.sub("N", b), (path_ref, a, b)
    A = np.array([[float(x) for x in l.split()] for l in ref])
    B = np.array([[float(x) for x in l.split()] for l in mine])
    assert A.shape == B.shape
    scale = np.max(np.abs(A), axis=0)
    err = np.max(np.abs(A - B), axis=0)
    bad = err > 2e-7 * scale + 1e-300
    assert not bad.any(), (os.path.basename(path_ref), err, scale)


@pytest.mark.parametrize("name", ["ferroelectric", "magnetoelastic", "afm", "drude", "mag_1d_maxwell"])
def test_text_outputs_match_the_reference(gf, refrun, tmp_path, name):
    d = _decks(gf)[name]
    gf.decks.write_deck(d, str(tmp_path / "deck"))
    refrun.run(str(tmp_path / "deck"), str(tmp_path / "ref"), outputs=True)
    out = tmp_path / "mine"
    out.mkdir()
    with gf.Engine(str(tmp_path / "deck"), device=0) as eng:
        eng.run_deck(str(out))
        assert eng.get_info().step == d.steps
    ref_files = sorted(f for f in os.listdir(tmp_path / "ref") if f.endswith(".dat") and not f.startswith("J_ISHE"))
    mine_files = sorted(os.listdir(out))
    assert ref_files == mine_files
    assert len(ref_files) >= 4
    for f in ref_files:
        _compare(str(tmp_path / "ref" / f), str(out / f))


def test_restart_inputs_force_store_and_drude_currents(gf, refrun, tmp_path):
    """elastoforce.in and Jp1-3.in (if_input_elastoforce, if_input_Jp) are
    read as the reference reads them (inoutput.cpp:220-237, 283-328): the
    stiffness damping of the first step uses the restored force store and
    the Drude update starts from the restored pole currents."""
    from test_gpu_parity import assert_trace_close, engine_trace
    var = _variants(gf)
    d = dataclasses.replace(var["drude_metal_layer"][0], steps=10)
    rng = np.random.default_rng(41)
    shape = (3, d.nx, d.ny, d.nz)
    solid = (d.material_cell() != 0)[None]
    metal = (d.material_cell() == 3)[None]
    d.materials = [dataclasses.replace(m, stiff_damping=0.2 * d.dt / m.density) for m in d.materials]
    d.force0 = rng.uniform(-1e9, 1e9, size=shape) * solid
    d.jp0 = [rng.uniform(-1e8, 1e8, size=shape) * metal for _ in range(3)]
    probe = (4, 4, 2)
    gf.decks.write_deck(d, str(tmp_path / "deck"))
    r = refrun.run(str(tmp_path / "deck"), str(tmp_path / "ref"), steps=10, probe=probe)
    with gf.Engine(str(tmp_path / "deck"), device=0) as eng:
        got = eng.download("force_store").reshape(shape)
        assert np.array_equal(got, d.force0)
        mine = engine_trace(eng, 10, probe)
    assert_trace_close(mine, r["trace"])
    # without the restored values the run differs (the inputs matter)
    d.force0, d.jp0 = None, None
    gf.decks.write_deck(d, str(tmp_path / "deck2"))
    with gf.Engine(str(tmp_path / "deck2"), device=0) as eng:
        other = engine_trace(eng, 10, probe)
    assert np.max(np.abs(other - mine)) > 0.0
