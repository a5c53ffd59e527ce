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
