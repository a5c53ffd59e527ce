"""GPU parity: the B200 engine, called through the C ABI, against GO-Ferro's
own solver (golden fixtures made by the oracle build, and the oracle binary
run live on extra decks).

Tolerance (FP64 form): every traced observable and every final field agrees
with the reference to 1e-10 relative to the observable's largest magnitude.
"""
import importlib.util
import dataclasses
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
TOL = 1e-10

FIELDS = {"m": ("mx", "my", "mz"), "m_afm1": ("mx_AFM1", "my_AFM1", "mz_AFM1"),
          "m_afm2": ("mx_AFM2", "my_AFM2", "mz_AFM2"), "u": ("ux", "uy", "uz"), "v": ("vx", "vy", "vz"),
          "p": ("px", "py", "pz"), "q": ("qx", "qy", "qz"), "Hstat": ("Hx_stat", "Hy_stat", "Hz_stat")}
YEE = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def engine_trace(eng, steps, probe, graph=True):
    rows = []
    for s in range(steps + 1):
        if s:
            eng.advance(1, graph=graph)
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


def assert_trace_close(mine, ref, tol=TOL):
    for c in range(1, 22):
        scale = np.max(np.abs(ref[:, c]))
        err = np.max(np.abs(mine[:, c] - ref[:, c]))
        if scale == 0.0:
            assert err == 0.0, f"column {c}: expected zeros, got {err}"
        else:
            assert err <= tol * scale, f"column {c}: rel err {err / scale:.3e}"


def assert_fields_close(eng, ref_fields, tol=TOL):
    checked = 0
    for name, parts in FIELDS.items():
        if parts[0] not in ref_fields:
            continue
        mine = eng.download(name)
        # scale of a vector field = its largest component: each component of
        # the FFT magnetostatic field mixes all components of M through the
        # demag tensor, so its rounding error is relative to the whole field
        vscale = max(float(np.max(np.abs(ref_fields[p]))) for p in parts)
        for c, p in enumerate(parts):
            r = ref_fields[p]
            scale = vscale
            err = np.max(np.abs(mine[c].ravel() - r))
            assert err <= tol * max(scale, 1e-300) or (scale == 0 and err == 0), f"{p}: {err / max(scale, 1e-300):.3e}"
            checked += 1
    for p in YEE:
        if p not in ref_fields:
            continue
        mine = eng.download(p).ravel()
        r = ref_fields[p]
        scale = np.max(np.abs(r))
        err = np.max(np.abs(mine - r))
        assert err <= tol * max(scale, 1e-300) or (scale == 0 and err == 0), f"{p}: {err / max(scale, 1e-300):.3e}"
        checked += 1
    assert checked > 0


@pytest.mark.parametrize("name", json.load(open(os.path.join(GOLDEN, "cases.json"))).keys())
def test_engine_matches_golden(gf, tmp_path, name):
    mg = _mg()
    d, steps, probe = mg.make_deck(name)
    gf.decks.write_deck(d, str(tmp_path))
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    with gf.Engine(str(tmp_path), device=0) as eng:
        mine = engine_trace(eng, steps, probe)
        assert_trace_close(mine, g["trace"])
        assert_fields_close(eng, {k: g[k] for k in g.files if k != "trace"})
        eng.check_finite()


def test_graph_and_eager_paths_are_identical(gf, tmp_path):
    d = gf.decks.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=9)
    d.amp_gauss *= 1e6
    gf.decks.write_deck(d, str(tmp_path))
    out = []
    for graph in (True, False):
        with gf.Engine(str(tmp_path), device=0) as eng:
            eng.advance(9, graph=graph)
            out.append([eng.download(f) for f in ("m", "u", "v", "Ex", "Hz")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_upload_download_roundtrip(gf, tmp_path):
    d = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=10, steps=2)
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0) as eng:
        p = eng.download("p")
        assert p.shape == (3, 8, 8, 10)
        assert np.array_equal(p, d.p0)
        new = np.random.default_rng(0).standard_normal(p.shape) * 1e-3
        eng.upload("p", new)
        assert np.array_equal(eng.download("p"), new)
        dims, cnt = eng.field_dims("Ez")
        assert dims == (9, 9, 10) and cnt == 810


# ---------------------------------------------------------------------------
# live oracle on deck variants that exercise further branches
# ---------------------------------------------------------------------------
def _variants(gf):
    D = gf.decks
    v = {}
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=25)
    d.abc_1D = True
    d.strain_type, d.sigma_gauss, d.amp_gauss, d.strain_z = 1, 2e-16, 1e-3, 1
    v["mur_elastic_gauss_source"] = (d, 25, (4, 8, 7))
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=25)
    d.strain_type, d.sigma_gauss, d.amp_gauss, d.strain_z = 3, 2e-16, 1e7, 8
    d.layers = [(5, 1), (4, 2), (3, 1)]
    d.periodic = (False, False, False)
    v["traction_source_open_box"] = (d, 25, (4, 8, 7))
    d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=25)
    d.jf_type, d.jf_freq, d.jf_sigma, d.jf_amp = 6, 3e15, 5e-18, 1e12
    d.planeEM, d.planeEM_E, d.planeEM_freq = True, (1e5, 0.0, 0.0), (1e15, 1e15, 1e15)
    d.Eext_altr, d.E_altr_freq = (1e6, 0.0, 2e6), (1e14, 0.0, 3e14)
    v["fe_jf6_plane_wave_eext"] = (d, 25, (4, 4, 5))
    d = D.preset_fm_demag(nx=12, ny=8, nz=6, steps=25)
    d.Hext_table = None
    d.Hext_stat, d.Hext_altr, d.H_altr_freq = (0, 0, 8e4), (2e3, 0, 0), (2e11, 0, 0)
    m2 = D.yig(0.02)
    m2.Aex, m2.iDMI, m2.aniso_type, m2.K1 = 2.0e-12, 1e-3, 2, 3e3
    d.materials.append(m2)
    d.layers = [(3, 1), (3, 2)]
    d.periodic = (True, False, False)
    v["two_fm_materials_dmi_uniaxial"] = (d, 25, None)
    d = D.preset_fm_demag(nx=8, ny=8, nz=4, steps=15)
    d.demag_factor, d.demag_fac = True, (0.1, 0.2, 0.7)
    v["demag_factor"] = (d, 15, None)
    # several (j,k) tiles of the elastic kernel, partial tiles in j and k
    d = D.preset_magnetoelastic(nx=6, ny=20, nz=40, sub=20, film=12, steps=8)
    d.amp_gauss *= 1e6
    v["elastic_multi_tile"] = (d, 8, (3, 10, 30))
    # ny-1 < nz-1 with k = ny-1 = 35 in the second z tile: the +z neighbour
    # of that layer (k = 0) lies outside the tile
    d = D.preset_magnetoelastic(nx=4, ny=36, nz=40, sub=20, film=12, steps=6)
    d.amp_gauss *= 1e6
    v["elastic_quirk_far_tile"] = (d, 6, (2, 10, 30))
    # ferromagnetic film on a non-magnetic substrate with vacuum above:
    # magnetostatics every stage with non-magnetic cells in the FFT input
    d = D.preset_fm_demag(nx=8, ny=8, nz=10, steps=15)
    d.materials = [D.ggg(), D.yig(0.01)]
    d.layers = [(4, 1), (4, 2), (2, 0)]
    d.m0 = D.tilt_m0((8, 8, 10), 5, d.material_cell() == 2)
    v["fm_film_demag_substrate"] = (d, 15, None)
    # two-sublattice antiferromagnet film: uniaxial anisotropy, inter-sublattice
    # exchange, magnetostatics every stage, external pulse, seeded tilted m1/m2
    d = D.preset_fm_demag(nx=8, ny=8, nz=10, steps=20)
    d.materials = [D.ggg(), D.afm_uniaxial(0.02)]
    d.layers = [(4, 1), (4, 2), (2, 0)]
    d.m0 = None
    d.afm0 = D.tilt_afm0((8, 8, 10), 99, d.material_cell() == 2)
    v["afm_film_demag"] = (d, 20, None)
    # antiferromagnet with magnetoelastic coupling and eigenstrain, elastic
    # source, Maxwell fields driven by and acting on the sublattices
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=20)
    d.materials = [D.ggg(), D.afm_uniaxial(0.01, magnetoelastic=True)]
    d.m0 = None
    d.afm0 = D.tilt_afm0((8, 16, 12), 11, d.material_cell() == 2)
    d.amp_gauss *= 1e6
    v["afm_magnetoelastic_em"] = (d, 20, (4, 8, 7))
    # ferromagnet on an antiferromagnet with a prescribed H table and a static
    # + alternating field: the antiferromagnet recomputes the shared external
    # field every stage and the ferromagnet's later stages see that value
    d = D.preset_fm_demag(nx=8, ny=8, nz=10, steps=20)
    d.materials = [D.afm_uniaxial(0.02), D.yig(0.01)]
    d.layers = [(4, 1), (4, 2), (2, 0)]
    mc = d.material_cell()
    d.m0 = D.tilt_m0((8, 8, 10), 21, mc == 2)
    d.afm0 = D.tilt_afm0((8, 8, 10), 22, mc == 1)
    d.Hext_stat, d.Hext_altr, d.H_altr_freq = (0.0, 0.0, 4e4), (3e3, 0.0, 0.0), (5e11, 0.0, 0.0)
    v["fm_on_afm_prescribed_h"] = (d, 20, None)
    # metal layer with two Drude poles under the ferroelectric, sheet-current source in the metal
    d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=20)
    metal = D.Material(title="metal", c11=2.3e11, c12=1.0e11, c44=1.2e11, density=8.9e3, er=1.0,
                       drude=((0.6, 2e16, 1e-14), (0.4, 5e15, 5e-15), (0.0, 0.0, 1.0)))
    d.materials.append(metal)
    d.layers = [(3, 2), (7, 1)]
    v["drude_metal_layer"] = (d, 20, (4, 4, 2))
    # the same stack with a perfect-conductor bottom layer
    d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=20)
    d.materials.append(D.Material(title="pec", c11=2.3e11, c12=1.0e11, c44=1.2e11, density=8.9e3, pec=True))
    d.layers = [(3, 2), (7, 1)]
    d.jf_lo, d.jf_hi = (0, 0, 5), (7, 7, 5)
    v["pec_layer"] = (d, 20, (4, 4, 6))
    # spin pumping: a heavy-metal layer under a YIG film, inverse-spin-Hall
    # current from m x dm/dt of the film's bottom plane driving the Yee E field
    d = D.preset_fm_demag(nx=8, ny=8, nz=12, steps=20)
    d.dt = 4e-18
    metal = D.Material(title="Pt", c11=3.47e11, c12=2.51e11, c44=0.765e11, density=21450.0, er=1.0, cond=1e5,
                       spin_pump=True, spin=(0.1, 1e19, 2e-9))
    d.materials = [metal, D.yig(0.01)]
    # no vacuum layer: with spin pumping on, the reference reads the material
    # of every layer's first cell without a vacuum test (global.cpp:185)
    d.layers = [(4, 1), (8, 2)]
    d.m0 = D.tilt_m0((8, 8, 12), 31, d.material_cell() == 2, max_deg=5.0)
    d.em, d.em_fromM, d.em_back_M = True, True, True
    d.spin_pumping = True
    d.periodic = (True, True, False)
    v["spin_pumping_ishe"] = (d, 20, (4, 4, 2))
    # materials scattered cell by cell (struct.in): the ferroelectric and
    # dielectrics of different permittivity and conductivity.  With three
    # materials every E edge's four-cell quadruple is one of at most 3^4 = 81
    # classes (the Yee kernel's class table); with six there are more than
    # 256 and the kernel reads the four cells' materials itself.
    for nmat in (3, 6):
        d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=20)
        for q in range(1, nmat):
            d.materials.append(dataclasses.replace(D.ggg(), title=f"diel{q}", er=4.0 + 3.0 * q,
                                                   cond=(0.0, 1e3, 1e4, 5e4, 2e4)[q - 1]))
        rng = np.random.default_rng(100 + nmat)
        d.struct = rng.integers(1, nmat + 1, size=(8, 8, 10)).astype(np.uint8)
        v[f"random_struct_{nmat}mat"] = (d, 20, (4, 4, 5))
    # crystal frame rotated against the grid (if_OrientRotate): the rotated
    # stiffness has no cubic pattern, magnetostriction / electrostriction and
    # anisotropy act in the crystal frame (mathlib.cpp:45-135, global.cpp:365-441)
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=20)
    d.amp_gauss *= 1e6
    d.Tg2c = D.rotation(20.0, 30.0)
    v["rotated_magnetoelastic"] = (d, 20, (4, 8, 7))
    d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=20)
    d.Tg2c = D.rotation(-35.0, 15.0)
    v["rotated_ferroelectric"] = (d, 20, (4, 4, 5))
    # sheet-current source types 0-3 and 5 (update_Jf_input,
    # EMdynamic_solver.cpp:3885-4000): sine, sine x sin / cos of the depth in
    # the box, sine for a number of cycles, Gaussian derivative
    for jt in (0, 1, 2, 3, 5):
        d = D.preset_ferroelectric(nx=8, ny=8, nz=12, steps=20)
        d.jf_type, d.jf_comp = jt, ("x", "y", "z", "x", "y")[jt if jt < 5 else 4]
        d.jf_lo, d.jf_hi = (1, 2, 3), (6, 5, 6)
        # type 5 reads its width from Jf_input_freq; type 3 stops after one cycle
        d.jf_freq = {5: 5e-17, 3: 4e16}.get(jt, 4e15)
        d.jf_cycles = 1 if jt == 3 else 0
        d.jf_amp = 1e14
        v[f"jf_type{jt}"] = (d, 20, (4, 4, 5))
    # 1-D magnetostatics (if_mag_1Dmodel: H_z = -Ms m_z, magnetostatic_solver.cpp:221-249)
    d = D.preset_fm_demag(nx=8, ny=8, nz=10, steps=15)
    d.materials = [D.ggg(), D.yig(0.01)]
    d.layers = [(4, 1), (4, 2), (2, 0)]
    d.m0 = D.tilt_m0((8, 8, 10), 41, d.material_cell() == 2, max_deg=10.0)
    d.mag_1D = True
    v["mag_1d_model"] = (d, 15, None)
    # the 1-D model with M-sourced Maxwell fields acting back on m: the
    # cell-centred Maxwell H_z is the 1-D field -Ms m_z - H_stat,z of the
    # stage state (update_DH_cell, EMdynamic_solver.cpp:3793-3804), for a
    # ferromagnetic and an antiferromagnetic film
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=20)
    d.m0 = D.tilt_m0((8, 16, 12), 61, d.material_cell() == 2, max_deg=15.0)
    d.amp_gauss *= 1e6
    d.mag_1D = True
    v["mag_1d_maxwell"] = (d, 20, (4, 8, 7))
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=20)
    d.materials = [D.ggg(), D.afm_uniaxial(0.01, magnetoelastic=True)]
    d.m0 = None
    d.afm0 = D.tilt_afm0((8, 16, 12), 63, d.material_cell() == 2)
    d.amp_gauss *= 1e6
    d.mag_1D = True
    v["afm_mag_1d_maxwell"] = (d, 20, (4, 8, 7))
    # prescribed-m test mode: the k = 0 plane of a ferromagnetic film on a
    # magnetoelastic, Maxwell-coupled deck precesses on a 20-degree cone at
    # 5e12 Hz (stage outputs and the step value of that plane overwritten)
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=2, film=6, steps=20)
    d.layers = [(6, 2), (6, 0)]
    d.m0 = D.tilt_m0((8, 16, 12), 51, d.material_cell() == 2)
    d.amp_gauss *= 1e6
    d.prescribed_m, d.precess_angle, d.precess_freq = True, 20.0, 5e12
    v["prescribed_m_film"] = (d, 20, (4, 8, 3))
    # flexoelectric coupling (if_flexo): polarisation- and strain-gradient
    # terms of the TDGL field (ferroelectric_solver.cpp:800-833), the
    # p-gradient eigenstrain (elastic_dynamic_solver.cpp:63-70), with the
    # ferroelectric film between an elastic dielectric substrate and vacuum
    # so the mirror (p) and stress-free (strain) surface rules both act
    for vn, rot, elastic in (("flexo_fe_film", None, True), ("flexo_rotated", (25.0, -40.0), True),
                             ("flexo_no_elastic", None, False)):
        d = D.preset_ferroelectric(nx=8, ny=8, nz=12, steps=20, pulse=elastic)
        d.materials = [dataclasses.replace(D.pto(), f11=6.0, f12=3.5, f44=2.5), D.ggg()]
        d.layers = [(3, 2), (6, 1), (3, 0)]
        r = D.splitmix64(20240917, 3 * d.n).reshape(d.n, 3)
        d.p0 = (0.1 * r - 0.05).T.reshape(3, 8, 8, 12).copy() * (d.material_cell() == 1)
        d.q0 = np.zeros_like(d.p0)
        d.flexo = True
        if rot:
            d.Tg2c = D.rotation(*rot)
        if not elastic:
            d.elastic = d.elasto_back = d.elasto_on = d.abc_1D = False
            d.em = d.em_fromP = d.em_back_P = False
        v[vn] = (d, 20, (4, 4, 5) if elastic else None)
    return v


def edge_quadruples(mc):
    """Distinct four-cell material quadruples of the interior x-directed E
    edges (cells (i, j-1|j, k-1|k)), a lower bound of the Yee kernel's class
    count."""
    q = np.stack([mc[:, :-1, :-1], mc[:, :-1, 1:], mc[:, 1:, :-1], mc[:, 1:, 1:]], axis=-1).reshape(-1, 4)
    return len({tuple(r) for r in q})


def test_random_struct_variants_cover_both_yee_paths(gf):
    v = _variants(gf)
    assert edge_quadruples(v["random_struct_3mat"][0].material_cell()) <= 81
    assert edge_quadruples(v["random_struct_6mat"][0].material_cell()) > 256


@pytest.mark.parametrize("vname", ["mur_elastic_gauss_source", "traction_source_open_box",
                                   "fe_jf6_plane_wave_eext", "two_fm_materials_dmi_uniaxial", "demag_factor",
                                   "elastic_multi_tile", "elastic_quirk_far_tile", "fm_film_demag_substrate",
                                   "afm_film_demag", "afm_magnetoelastic_em", "fm_on_afm_prescribed_h",
                                   "drude_metal_layer", "pec_layer", "spin_pumping_ishe", "random_struct_3mat",
                                   "random_struct_6mat", "rotated_magnetoelastic", "rotated_ferroelectric",
                                   "jf_type0", "jf_type1", "jf_type2", "jf_type3", "jf_type5", "mag_1d_model",
                                   "mag_1d_maxwell", "afm_mag_1d_maxwell",
                                   "flexo_fe_film", "flexo_rotated", "flexo_no_elastic", "prescribed_m_film"])
def test_engine_matches_live_oracle(gf, refrun, tmp_path, vname):
    d, steps, probe = _variants(gf)[vname]
    gf.decks.write_deck(d, str(tmp_path / "deck"))
    r = refrun.run(str(tmp_path / "deck"), str(tmp_path / "ref"), steps=steps, probe=probe, dump=True)
    with gf.Engine(str(tmp_path / "deck"), device=0) as eng:
        mine = engine_trace(eng, steps, probe if probe else (0, 0, 0))
        assert_trace_close(mine, r["trace"])
        assert_fields_close(eng, r["fields"])
