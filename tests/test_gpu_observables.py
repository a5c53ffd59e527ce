"""GPU tests of the observable reads of the C ABI (gf_average, gf_probe_em)
against the full fields downloaded through gf_download, both forms.

gf_average sums the three components in one deterministic reduction (8192
strided partials, then 64, then 1); its result is compared with an FP64
numpy sum of the downloaded field divided by the cell count of the
observable, to 1e-13 relative (the two sums are taken in different orders).
gf_probe_em centres only the probed cell; it must equal the same cell of the
whole-grid centring (E_cell, H_cell) bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_average_and_probe_match_full_fields(gf, tmp_path, precision):
    d = gf.decks.preset_magnetoelastic(nx=12, ny=10, nz=16, sub=6, film=6, steps=12)
    d.amp_gauss *= 1e6
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0, precision=precision) as eng:
        eng.advance(12)
        u = eng.download("u")
        avg_u = eng.average("u")
        ref_u = u.reshape(3, -1).sum(axis=1) / d.n
        assert np.allclose(avg_u, ref_u, rtol=1e-13, atol=1e-13 * np.max(np.abs(ref_u)))
        m = eng.download("m")
        nfm = int((np.sqrt((m ** 2).sum(axis=0)) > 0.5).sum())
        avg_m = eng.average("m")
        ref_m = m.reshape(3, -1).sum(axis=1) / nfm
        assert np.allclose(avg_m, ref_m, rtol=1e-13, atol=1e-15)
        ec = eng.download("E_cell")
        hc = eng.download("H_cell")
        for cell in [(0, 0, 0), (5, 3, 9), (11, 9, 15)]:
            e, h = eng.probe_em(*cell)
            assert np.array_equal(e, ec[(slice(None),) + cell])
            assert np.array_equal(h, hc[(slice(None),) + cell])
