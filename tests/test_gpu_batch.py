"""GPU tests of batched runs (gf_batch_*): instances of uneven grids and both
precisions advanced by one CUDA graph per step give, bit for bit, what each
engine gives when advanced alone; the elastic-tile autotuner changes the
x-chunk only, which does not change results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _decks(gf):
    D = gf.decks
    fe = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=30)
    fe.jf_type, fe.jf_freq, fe.jf_sigma, fe.jf_amp = 6, 3e15, 5e-18, 1e12
    me = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=30)
    me.amp_gauss *= 1e6
    fe2 = D.preset_ferroelectric(nx=12, ny=8, nz=16, steps=30)
    fm = D.preset_fm_demag(nx=16, ny=16, nz=8, steps=30)
    return [(fe, "mixed", "p"), (me, "mixed", "u"), (fe2, "fp64", "p"), (me, "fp64", "v"), (fm, "fp64", "m")]


def test_batch_matches_engines_advanced_alone(gf, tmp_path):
    cases = _decks(gf)
    dirs = []
    for i, (d, _, _) in enumerate(cases):
        p = str(tmp_path / f"d{i}")
        gf.decks.write_deck(d, p)
        dirs.append(p)
    solo = []
    for p, (_, prec, field) in zip(dirs, cases):
        with gf.Engine(p, device=0, precision=prec) as e:
            e.advance(17)
            solo.append([e.download(field), e.download("Ex") if e.info.em else None])
    engines = [gf.Engine(p, device=0, precision=prec) for p, (_, prec, _) in zip(dirs, cases)]
    try:
        with gf.Batch(engines, autotune=True) as b:
            chunks = [b.tuned_chunk(i) for i in range(len(engines))]
            assert all(c >= 1 for c in chunks)
            b.advance(10)
            b.advance(7)
            b.synchronize()
        for e, (_, _, field), ref in zip(engines, cases, solo):
            assert e.get_info().step == 17
            assert np.array_equal(e.download(field), ref[0])
            if ref[1] is not None:
                assert np.array_equal(e.download("Ex"), ref[1])
        # the engines keep working alone after the batch is gone
        engines[0].advance(1)
        engines[0].check_finite()
    finally:
        for e in engines:
            e.close()


def test_batch_rejects_engines_at_different_parity(gf, tmp_path):
    d = gf.decks.preset_fm_demag(nx=8, ny=8, nz=4, steps=5)
    gf.decks.write_deck(d, str(tmp_path))
    a = gf.Engine(str(tmp_path), device=0)
    b = gf.Engine(str(tmp_path), device=0)
    try:
        b.advance(1)
        with pytest.raises(gf.GFError):
            gf.Batch([a, b])
    finally:
        a.close()
        b.close()


# ---------------------------------------------------------------------------
# phase mode: mixed-form TDGL / elastodynamics / FDTD engines, each RK stage
# three launches over the work items of every engine (the per-engine
# kernels' bodies on per-item block coordinates)
# ---------------------------------------------------------------------------
def _phase_decks(gf):
    D = gf.decks
    out = []
    for k, (nx, ny, nz) in enumerate([(8, 8, 10), (12, 20, 40), (6, 9, 33), (16, 16, 16)]):
        d = D.preset_ferroelectric(nx=nx, ny=ny, nz=nz, steps=30)
        d.jf_type, d.jf_freq, d.jf_sigma, d.jf_amp = 6, (1 + k) * 1e15, 5e-18, (1 + k) * 1e12
        out.append(d)
    # open x and y faces (Mur boundaries of E in all three directions), a
    # dielectric substrate and no elastodynamics in one of them
    d = D.preset_ferroelectric(nx=10, ny=12, nz=20, steps=30)
    d.periodic = (False, False, False)
    d.materials = [D.pto(), D.ggg()]
    d.layers = [(6, 2), (14, 1)]
    out.append(d)
    d = D.preset_ferroelectric(nx=8, ny=8, nz=12, steps=30)
    d.elastic = d.elasto_back = d.elasto_on = False
    out.append(d)
    return out


@pytest.mark.parametrize("autotune,mode", [(False, "phases"), (True, "phases"), (False, "persistent"), (True, "persistent")])
def test_batch_phases_match_engines_advanced_alone(gf, tmp_path, autotune, mode):
    """The phase mode (launches per stage phase) and the persistent mode
    (the whole step as one cooperative launch with grid barriers between the
    phases) run the per-engine kernels' bodies on the same work lists: each
    engine's fields equal its own run bit for bit."""
    decks = _phase_decks(gf)
    dirs = []
    for i, d in enumerate(decks):
        p = str(tmp_path / f"d{i}")
        gf.decks.write_deck(d, p)
        dirs.append(p)
    fields = [("p", "q", "u", "Ex", "Hz") if d.elastic else ("p", "q", "Ex", "Hz") for d in decks]
    solo = []
    for p, fl in zip(dirs, fields):
        with gf.Engine(p, device=0, precision="mixed") as e:
            e.advance(13)
            solo.append({f: e.download(f) for f in fl})
    engines = [gf.Engine(p, device=0, precision="mixed") for p in dirs]
    try:
        with gf.Batch(engines, autotune=autotune, mode=mode) as b:
            assert b.plan().startswith(mode + ":"), b.plan()
            assert all(b.tuned_chunk(i) >= 1 for i in range(len(engines)))
            b.advance(6)
            b.advance(7)
            b.synchronize()
        for i, (e, ref) in enumerate(zip(engines, solo)):
            assert e.get_info().step == 13
            e.check_finite()
            for f in ref:
                a = e.download(f)
                assert np.array_equal(a, ref[f]), (i, f, float(np.max(np.abs(a - ref[f]))))
        engines[0].advance(1)
        engines[0].check_finite()
    finally:
        for e in engines:
            e.close()


def test_batch_mode_choice(gf, tmp_path):
    fe = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=10, steps=5)
    fm = gf.decks.preset_fm_demag(nx=8, ny=8, nz=4, steps=5)
    gf.decks.write_deck(fe, str(tmp_path / "fe"))
    gf.decks.write_deck(fm, str(tmp_path / "fm"))
    a = gf.Engine(str(tmp_path / "fe"), device=0, precision="mixed")
    b = gf.Engine(str(tmp_path / "fe"), device=0)
    c = gf.Engine(str(tmp_path / "fm"), device=0, precision="mixed")
    try:
        with pytest.raises(gf.GFError) as ei:
            gf.Batch([a, b], autotune=False, mode="phases")
        assert ei.value.code == -7 and "FP64" in str(ei.value)
        with pytest.raises(gf.GFError):
            gf.Batch([a, c], autotune=False, mode="phases")
        with gf.Batch([a, b], autotune=False) as bb:
            assert bb.plan().startswith("branches"), bb.plan()
        with gf.Batch([a], autotune=False) as bb:
            assert bb.plan().startswith("phases:"), bb.plan()
    finally:
        for e in (a, b, c):
            e.close()


def test_batch_auto_mode_times_both_and_undoes_its_trial_steps(gf, tmp_path):
    """GF_BATCH_AUTO with autotune times steps of the phase and branch modes
    on the engines' own state and restores it: the batch then gives what each
    engine gives alone, whichever mode it kept."""
    decks = _phase_decks(gf)[:4]
    dirs = []
    for i, d in enumerate(decks):
        p = str(tmp_path / f"d{i}")
        gf.decks.write_deck(d, p)
        dirs.append(p)
    solo = []
    for p in dirs:
        with gf.Engine(p, device=0, precision="mixed") as e:
            e.advance(3)
            solo.append({f: e.download(f) for f in ("p", "u", "Ex")})
    engines = [gf.Engine(p, device=0, precision="mixed") for p in dirs]
    try:
        with gf.Batch(engines, autotune=True) as b:
            assert "timed steps: phases" in b.plan() and "persistent" in b.plan(), b.plan()
            assert all(e.get_info().step == 0 for e in engines)
            b.advance(3)
            b.synchronize()
        for e, ref in zip(engines, solo):
            assert e.get_info().step == 3
            for f, v in ref.items():
                assert np.array_equal(e.download(f), v), f
    finally:
        for e in engines:
            e.close()
