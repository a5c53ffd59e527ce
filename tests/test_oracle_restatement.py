"""The numpy restatement of the ferromagnetic LLG + magnetostatics step
(oracle/restate_fm.py) against the compiled reference: the committed golden
fixture of the CPU-runnable configuration and, when the reference build is
present, the live reference on a two-material deck with DMI and uniaxial
anisotropy.  Tolerance 1e-11 relative to the vector's magnitude: the two
differ only by FFT, transcendental-function and summation-order rounding."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import restate_fm  # noqa: E402

TOL = 1e-11


def _mats(deck):
    return [dict(fm=m.fm, Ms=m.Ms, Aex=m.Aex, iDMI=m.iDMI, aniso_type=m.aniso_type, K1=m.K1, K2=m.K2,
                 alpha=m.alpha, gyro=m.gyro) for m in deck.materials]


def _run(deck, steps):
    mid = deck.material_cell()
    m0 = deck.m0 if deck.m0 is not None else None
    assert m0 is not None
    return restate_fm.run(mid, _mats(deck), deck.dx, deck.dy, deck.dz, deck.periodic, m0, deck.dt, steps,
                          magnetostatics=deck.magnetostatics, Hext_table=deck.Hext_table,
                          Hext_stat=deck.Hext_stat, Hext_altr=deck.Hext_altr, H_altr_freq=deck.H_altr_freq)


def _close(a, b, what, scale=None):
    scale = np.max(np.abs(b)) if scale is None else scale
    err = np.max(np.abs(a - b))
    assert err <= TOL * max(scale, 1e-300), f"{what}: rel err {err / scale:.3e}"


def test_restatement_matches_golden_fm_demag(gf):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    deck, steps, _ = mg.make_deck("fm_demag_16x16x8")
    g = np.load(os.path.join(ROOT, "tests", "golden", "fm_demag_16x16x8.npz"))
    trace, m, hs = _run(deck, steps)
    # <m> is a vector: its components are compared on the scale of |<m>|
    vs = np.max(np.abs(g["trace"][:, 1:4]))
    for c in range(3):
        _close(trace[:, c], g["trace"][:, 1 + c], f"<m>{'xyz'[c]}", vs)
    ms = max(np.max(np.abs(g[n])) for n in ("mx", "my", "mz"))
    for c, name in enumerate(("mx", "my", "mz")):
        _close(m[c].ravel(), g[name], name, ms)
    hsc = max(np.max(np.abs(g[n])) for n in ("Hx_stat", "Hy_stat", "Hz_stat"))
    for c, name in enumerate(("Hx_stat", "Hy_stat", "Hz_stat")):
        _close(hs[c].ravel(), g[name], name, hsc)


def test_restatement_matches_live_reference_dmi_uniaxial(gf, refrun, tmp_path):
    D = gf.decks
    d = D.preset_fm_demag(nx=12, ny=8, nz=6, steps=15)
    d.Hext_table = None
    d.Hext_stat, d.Hext_altr, d.H_altr_freq = (0, 0, 8e4), (2e3, 0, 0), (2e11, 0, 0)
    m2 = D.yig(0.02)
    m2.Aex, m2.iDMI, m2.aniso_type, m2.K1 = 2.0e-12, 1e-3, 2, 3e3
    d.materials.append(m2)
    d.layers = [(3, 1), (3, 2)]
    d.periodic = (True, False, False)
    D.write_deck(d, str(tmp_path / "deck"))
    r = refrun.run(str(tmp_path / "deck"), str(tmp_path / "ref"), steps=15, dump=True)
    trace, m, hs = _run(d, 15)
    vs = np.max(np.abs(r["trace"][:, 1:4]))
    for c in range(3):
        _close(trace[:, c], r["trace"][:, 1 + c], f"<m>{'xyz'[c]}", vs)
    ms = max(np.max(np.abs(r["fields"][n])) for n in ("mx", "my", "mz"))
    for c, name in enumerate(("mx", "my", "mz")):
        _close(m[c].ravel(), r["fields"][name], name, ms)
