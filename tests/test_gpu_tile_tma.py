"""GPU tests of the elastic tile's TMA staging (cp.async.bulk.tensor of each
staged plane).  Blocks whose staged box lies inside the grid in every
periodic direction load it with TMA, the others with per-thread cp.async;
both write the same shared-memory layout, so a run equals the run with every
block on cp.async (GOFERRO_TILE_TMA=0) bit for bit, and the reference to
1e-10."""
import os

import numpy as np
import pytest

from test_gpu_parity import assert_fields_close, assert_trace_close, engine_trace

pytestmark = pytest.mark.gpu


def _deck(gf):
    # ny = 32: tiles at j0 = 8, 16 stage by TMA, j0 = 0, 24 wrap (cp.async);
    # nz = 48 (a multiple of 16) so the maps exist
    d = gf.decks.preset_magnetoelastic(nx=8, ny=32, nz=48, sub=20, film=16, steps=10)
    d.amp_gauss *= 1e6
    return d, (4, 16, 30)


def _run(gf, ddir, precision, tma, steps, probe):
    old = os.environ.get("GOFERRO_TILE_TMA")
    os.environ["GOFERRO_TILE_TMA"] = "1" if tma else "0"
    try:
        with gf.Engine(ddir, device=0, precision=precision) as eng:
            tr = engine_trace(eng, steps, probe)
            fields = {f: eng.download(f) for f in ("m", "u", "v")}
            eng.check_finite()
    finally:
        if old is None:
            del os.environ["GOFERRO_TILE_TMA"]
        else:
            os.environ["GOFERRO_TILE_TMA"] = old
    return tr, fields


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tma_staging_equals_cp_async_staging(gf, tmp_path, precision):
    d, probe = _deck(gf)
    gf.decks.write_deck(d, str(tmp_path))
    a = _run(gf, str(tmp_path), precision, True, 10, probe)
    b = _run(gf, str(tmp_path), precision, False, 10, probe)
    assert np.array_equal(a[0], b[0])
    for f in a[1]:
        assert np.array_equal(a[1][f], b[1][f]), f


def test_tma_staging_matches_reference(gf, refrun, tmp_path):
    d, probe = _deck(gf)
    gf.decks.write_deck(d, str(tmp_path / "deck"))
    r = refrun.run(str(tmp_path / "deck"), str(tmp_path / "ref"), steps=10, probe=probe, dump=True)
    with gf.Engine(str(tmp_path / "deck"), device=0) as eng:
        assert_trace_close(engine_trace(eng, 10, probe), r["trace"])
        assert_fields_close(eng, r["fields"])
