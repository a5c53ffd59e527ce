"""GPU tests of gf_save_state / gf_load_state: a run restarted from a
checkpoint continues bit for bit (Liao history, stiffness-damping force
store, step counter and external-field clock included), in both forms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _deck(gf, kind):
    D = gf.decks
    if kind == "magnetoelastic":
        d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=40)
        d.amp_gauss *= 1e6
        return d, ("m", "u", "v", "Ex", "Hz")
    d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=40)
    d.jf_type, d.jf_freq, d.jf_sigma, d.jf_amp = 6, 3e15, 5e-18, 1e12
    return d, ("p", "q", "u", "Ez")


@pytest.mark.parametrize("kind", ["magnetoelastic", "ferroelectric"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_continues_bit_for_bit(gf, tmp_path, kind, precision):
    d, fields = _deck(gf, kind)
    ddir = str(tmp_path / "deck")
    gf.decks.write_deck(d, ddir)
    ck = str(tmp_path / "state.ck")
    with gf.Engine(ddir, device=0, precision=precision) as a:
        a.advance(13)               # odd: the restart must follow the step parity
        a.save_state(ck)
        a.advance(11)
        ref = [a.download(f) for f in fields]
        t_ref = a.get_info().time
    with gf.Engine(ddir, device=0, precision=precision) as b:
        b.load_state(ck)
        assert b.info.step == 13
        b.advance(11)
        got = [b.download(f) for f in fields]
        assert b.get_info().time == t_ref
    for f, x, y in zip(fields, ref, got):
        assert np.array_equal(x, y), f


def test_checkpoint_rejects_other_grids(gf, tmp_path):
    d, _ = _deck(gf, "ferroelectric")
    gf.decks.write_deck(d, str(tmp_path / "a"))
    d2 = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=12, steps=5)
    gf.decks.write_deck(d2, str(tmp_path / "b"))
    ck = str(tmp_path / "a.ck")
    with gf.Engine(str(tmp_path / "a"), device=0) as a:
        a.save_state(ck)
    with gf.Engine(str(tmp_path / "b"), device=0) as b:
        with pytest.raises(gf.GFError):
            b.load_state(ck)
    with gf.Engine(str(tmp_path / "a"), device=0, precision="mixed") as c:
        with pytest.raises(gf.GFError):
            c.load_state(ck)


def test_elastic_mur_boundary_rejects_single_layer(gf, tmp_path):
    """The elastic Mur boundary reads the plane below the top one, so a deck
    with nz = 1 is refused instead of reading outside the grid."""
    d = gf.decks.preset_ferroelectric(nx=4, ny=4, nz=1, steps=2)
    assert d.abc_1D and d.elastic
    gf.decks.write_deck(d, str(tmp_path))
    with pytest.raises(gf.GFError) as ei:
        gf.Engine(str(tmp_path), device=0)
    assert ei.value.code == -7
    assert "Mur boundary needs nz >= 2" in str(ei.value)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_with_elastostatic_solve(gf, tmp_path, precision):
    """Without elastodynamics the static strain is solved again after every
    step from the last iterate; a restart carries the static fields and the
    iterate, so the continued run equals the uninterrupted one bit for bit."""
    D = gf.decks
    d = D.Deck(nx=6, ny=6, nz=16, dx=1e-9, dy=1e-9, dz=1e-9, periodic=(True, True, True),
               layers=[(5, 2), (8, 1), (3, 2)], steps=20, dt=2e-14, materials=[D.pto(), D.ggg()], name="es_ck")
    d.elastostatic, d.elasto_limit, d.elasto_tol = True, 3, 1e-12
    rng = np.random.default_rng(11)
    d.p0 = rng.uniform(-0.2, 0.2, size=(3, 6, 6, 16)) * (d.material_cell() == 1)
    d.q0 = np.zeros_like(d.p0)
    ddir = str(tmp_path / "deck")
    gf.decks.write_deck(d, ddir)
    ck = str(tmp_path / "state.ck")
    with gf.Engine(ddir, device=0, precision=precision) as a:
        a.set_elastostatics(True)
        a.advance(5)
        a.save_state(ck)
        a.advance(4)
        ref = [a.download(f) for f in ("p", "q", "strain_static", "eigenstrain_static")]
    with gf.Engine(ddir, device=0, precision=precision) as b:
        b.set_elastostatics(True)
        b.load_state(ck)
        b.advance(4)
        got = [b.download(f) for f in ("p", "q", "strain_static", "eigenstrain_static")]
    for x, y in zip(ref, got):
        assert np.array_equal(x, y)
