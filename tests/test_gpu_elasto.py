"""GPU tests of the static-strain paths and the 1-D electrostatic model.

* Static strain inputs (strain_stat.in, eigenstraint0_crt.in) and
  if_elastostatic: the coupled step against the reference's solver, which
  reads the same files (FP64 1e-10, mixed 1e-5).
* The elastostatic solve (gf_set_elastostatics): the reference declares
  get_strain_static but its sources do not define it, so the solve is pinned
  to closed-form microelasticity (laminates, where the spectral operator is
  exact) and to a numpy restatement of the same iteration on a 3-D case;
  its coupling is pinned by feeding its solution to the reference through the
  input files.
* The 1-D electrostatic model (if_elec_1Dmodel; get_E_static_1D is also
  undefined in the reference): equal to the spectral solve for a laterally
  uniform polarisation, and its closed form with compensation.
"""
import dataclasses

import numpy as np
import pytest

from test_gpu_mixed import assert_mixed_close, trace_errors
from test_gpu_parity import assert_fields_close, assert_trace_close, engine_trace

pytestmark = pytest.mark.gpu
E0 = 8.854187817e-12


def smooth6(shape, seed, amp):
    """Six smooth random fields (sum of a few low Fourier modes)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x, y, z = np.meshgrid(np.arange(nx) / nx, np.arange(ny) / ny, np.arange(nz) / nz, indexing="ij")
    out = np.zeros((6,) + shape)
    for a in range(6):
        for _ in range(3):
            kx, ky, kz = rng.integers(0, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi)
            out[a] += rng.uniform(-1, 1) * np.cos(2 * np.pi * (kx * x + ky * y + kz * z) + ph)
    return amp * out


def static_decks(gf):
    D = gf.decks
    v = {}
    # ferroelectric film on a dielectric substrate under vacuum, with static
    # strain and eigenstrain inputs and if_elastostatic (the TDGL field adds
    # both; the dynamic eigenstrain subtracts the static one)
    d = D.preset_ferroelectric(nx=8, ny=8, nz=12, steps=15)
    d.materials = [D.pto(), D.ggg()]
    d.layers = [(3, 2), (6, 1), (3, 0)]
    r = D.splitmix64(4242, 3 * d.n).reshape(d.n, 3)
    d.p0 = (0.1 * r - 0.05).T.reshape(3, 8, 8, 12).copy() * (d.material_cell() == 1)
    d.q0 = np.zeros_like(d.p0)
    d.elastostatic = True
    d.strain_t0 = smooth6((8, 8, 12), 1, 2e-3)
    d.eig_t0 = smooth6((8, 8, 12), 2, 1e-3)
    v["static_inputs_fe"] = (d, 15, (4, 4, 5))
    # the same in a rotated crystal frame (strain_stat.in is rotated to it)
    d = dataclasses.replace(d, Tg2c=D.rotation(30.0, -20.0))
    v["static_inputs_fe_rotated"] = (d, 15, (4, 4, 5))
    # if_elastostatic without inputs: the static fields are zeros
    d = dataclasses.replace(v["static_inputs_fe"][0], strain_t0=None, eig_t0=None)
    v["elastostatic_flag_only"] = (d, 15, (4, 4, 5))
    # magnetoelastic film: the LLG adds the static strain, the elastic
    # solver's eigenstrain subtracts the static eigenstrain
    d = D.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=15)
    d.amp_gauss *= 1e6
    d.strain_t0 = smooth6((8, 16, 12), 3, 1e-3)
    d.eig_t0 = smooth6((8, 16, 12), 4, 5e-4)
    v["static_inputs_magnetoelastic"] = (d, 15, (4, 8, 7))
    # the 1-D electrostatic flag alone (the reference's model is undefined:
    # E_stat stays zero until the engine's model is enabled)
    d = D.preset_ferroelectric(nx=8, ny=8, nz=10, steps=15)
    d.elec_1D, d.elec_1D_comp = True, True
    v["elec_1d_flag"] = (d, 15, (4, 4, 5))
    return v


@pytest.mark.parametrize("vname", ["static_inputs_fe", "static_inputs_fe_rotated", "elastostatic_flag_only",
                                   "static_inputs_magnetoelastic", "elec_1d_flag"])
def test_static_inputs_match_reference(gf, refrun, tmp_path, vname):
    d, steps, probe = static_decks(gf)[vname]
    gf.decks.write_deck(d, str(tmp_path / "deck"))
    r = refrun.run(str(tmp_path / "deck"), str(tmp_path / "ref"), steps=steps, probe=probe, dump=True)
    with gf.Engine(str(tmp_path / "deck"), device=0) as eng:
        mine = engine_trace(eng, steps, probe)
        # each vector observable against its largest component: <u_y> of the
        # magnetoelastic film is a cancellation-level 1e-27 beside <u_z>
        for name, e in trace_errors(mine, r["trace"]).items():
            assert e <= 1e-10, f"{name}: {e:.3e}"
        assert_fields_close(eng, r["fields"])
    with gf.Engine(str(tmp_path / "deck"), device=0, precision="mixed") as eng:
        assert_mixed_close(engine_trace(eng, steps, probe), r["trace"])


def test_static_input_is_rotated_to_the_crystal_frame(gf, tmp_path):
    d = static_decks(gf)["static_inputs_fe_rotated"][0]
    gf.decks.write_deck(d, str(tmp_path))
    T = np.asarray(d.Tg2c)
    with gf.Engine(str(tmp_path), device=0) as eng:
        eps = eng.download("strain_static")
        eig = eng.download("eigenstrain_static")
    assert np.array_equal(eig, d.eig_t0)
    g = d.strain_t0
    full = np.array([[g[0], g[5], g[4]], [g[5], g[1], g[3]], [g[4], g[3], g[2]]])
    rot = np.einsum("ik,jl,kl...->ij...", T, T, full)
    solid = d.material_cell() != 0
    want = np.array([rot[0, 0], rot[1, 1], rot[2, 2], rot[1, 2], rot[0, 2], rot[0, 1]]) * solid
    assert np.max(np.abs(eps - want)) <= 1e-15


# ---------------------------------------------------------------------------
# the elastostatic solve
# ---------------------------------------------------------------------------
def laminate_deck(gf, layers, mats, nz, limit=3000, tol=1e-14, vacuum=False):
    D = gf.decks
    d = D.Deck(nx=4, ny=4, nz=nz, dx=1e-9, dy=1e-9, dz=1e-9, periodic=(True, True, True), layers=layers,
               steps=4, dt=1e-15, materials=mats, name="laminate")
    d.elastostatic = True
    d.elasto_limit, d.elasto_tol = limit, tol
    mc = d.material_cell()
    z = np.arange(nz)
    pz = (0.2 + 0.3 * np.sin(2 * np.pi * z / nz) + 0.1 * np.cos(6 * np.pi * z / nz))[None, None, :] * np.ones((4, 4, 1))
    fe = np.zeros_like(mc, dtype=bool)
    for i, m in enumerate(mats):
        if m.fe:
            fe |= mc == i + 1
    d.p0 = np.zeros((3, 4, 4, nz))
    d.p0[2] = pz * fe
    d.q0 = np.zeros_like(d.p0)
    return d


def laminate_exact(d):
    """Exact static strain of a laminate along z (clamped box, zero mean
    strain): in-plane strains 0, sigma_zz = S uniform,
    e_zz = e0_zz + (S + c12 (e0_xx + e0_yy)) / c11, S from <e_zz> = 0; in
    vacuum cells S = 0 forces the film's e_zz and the vacuum takes the mean."""
    mc = d.material_cell()[0, 0, :]
    pz = d.p0[2][0, 0, :]
    c11 = np.array([0.0] + [m.c11 for m in d.materials])[mc]
    c12 = np.array([0.0] + [m.c12 for m in d.materials])[mc]
    Q11 = np.array([0.0] + [m.Q11 for m in d.materials])[mc]
    Q12 = np.array([0.0] + [m.Q12 for m in d.materials])[mc]
    e0 = np.zeros((6, len(mc)))
    e0[0] = Q12 * pz ** 2
    e0[1] = Q12 * pz ** 2
    e0[2] = Q11 * pz ** 2
    solid = mc != 0
    ezz = np.zeros(len(mc))
    if solid.all():
        S = -np.mean(e0[2] + c12 * (e0[0] + e0[1]) / c11) / np.mean(1.0 / c11)
        ezz = e0[2] + (S + c12 * (e0[0] + e0[1])) / c11
    else:
        ezz[solid] = e0[2][solid] + c12[solid] * (e0[0] + e0[1])[solid] / c11[solid]
    out = np.zeros((6, len(mc)))
    out[2] = ezz
    return out, e0, solid


@pytest.mark.parametrize("case", ["homogeneous", "two_materials", "film_in_vacuum"])
def test_elastostatic_laminate_closed_form(gf, tmp_path, case):
    D = gf.decks
    if case == "homogeneous":
        d = laminate_deck(gf, [(32, 1)], [D.pto()], 32)
    elif case == "two_materials":
        d = laminate_deck(gf, [(12, 2), (14, 1), (6, 2)], [D.pto(), D.ggg()], 32)
    else:
        d = laminate_deck(gf, [(10, 2), (12, 1), (10, 0)], [D.pto(), D.ggg()], 32)
    gf.decks.write_deck(d, str(tmp_path))
    want, e0, solid = laminate_exact(d)
    with gf.Engine(str(tmp_path), device=0) as eng:
        used = eng.set_elastostatics(True)
        eps = eng.download("strain_static")[:, 0, 0, :]
        eig = eng.download("eigenstrain_static")[:, 0, 0, :]
        full = eng.download("strain_static")
    # laterally uniform
    assert np.max(np.abs(full - full[:, :1, :1, :])) <= 1e-15 * np.max(np.abs(full))
    assert np.max(np.abs(eig[:, solid] - e0[:, solid])) <= 1e-15 * np.max(np.abs(e0))
    scale = np.max(np.abs(want))
    tol = {"homogeneous": 1e-13, "two_materials": 1e-9, "film_in_vacuum": 1e-6}[case]
    err = np.max(np.abs(eps[:, solid] - want[:, solid])) / scale
    assert err <= tol, f"{case}: {err:.3e} after {used} iterations"
    if case == "homogeneous":
        assert used <= 3


def numpy_khachaturyan(d, e0, iters):
    """The same iteration restated with numpy FFTs (crystal frame, zero mean
    strain, the operator averaged over both signs of a Nyquist component),
    for a 3-D check of the device kernels."""
    nx, ny, nz = d.nx, d.ny, d.nz
    mc = d.material_cell()
    cs = np.array([[0, 0, 0]] + [[m.c11, m.c12, m.c44] for m in d.materials], dtype=np.float64)
    ch = cs.max(axis=0) * d.scale_elasto
    c11, c12, c44 = ch
    T = np.eye(3) if d.Tg2c is None else np.asarray(d.Tg2c)
    ks = [2 * np.pi * np.fft.fftfreq(nn, h) for nn, h in ((nx, d.dx), (ny, d.dy), (nz, d.dz))]
    K = np.array(np.meshgrid(*ks, indexing="ij"))
    nyq = np.array(np.meshgrid(*[(np.arange(nn) == nn // 2) & (nn % 2 == 0) for nn in (nx, ny, nz)], indexing="ij"))
    vi = [[0, 5, 4], [5, 1, 3], [4, 3, 2]]
    pairs = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]

    def green_apply(Kg, tk):
        Kq = np.einsum("ij,j...->i...", T, Kg)
        A = np.zeros((3, 3) + Kq.shape[1:])
        for i in range(3):
            for j in range(3):
                A[i, j] = (c11 * Kq[i] ** 2 + c44 * (np.sum(Kq ** 2, axis=0) - Kq[i] ** 2)) if i == j \
                    else (c12 + c44) * Kq[i] * Kq[j]
        Am = np.moveaxis(A, (0, 1), (-2, -1)).copy()
        zero = np.sum(Kg ** 2, axis=0) == 0
        Am[zero] = np.eye(3)
        G = np.linalg.inv(Am)
        G[zero] = 0.0
        f = np.array([sum(tk[vi[i][j]] * Kq[j] for j in range(3)) for i in range(3)])
        nvec = np.einsum("...ij,j...->i...", G, f)
        return np.array([0.5 * (Kq[j] * nvec[i] + Kq[i] * nvec[j]) for i, j in pairs])

    dc = cs[mc] - ch
    e = np.zeros_like(e0)
    for _ in range(iters):
        d_ = e - e0
        tau = np.empty_like(e0)
        for a, (b, c) in enumerate([(1, 2), (0, 2), (0, 1)]):
            tau[a] = (c11 * e0[a] + c12 * (e0[b] + e0[c])) - (dc[..., 0] * d_[a] + dc[..., 1] * (d_[b] + d_[c]))
        for a in range(3, 6):
            tau[a] = 2 * c44 * e0[a] - 2 * dc[..., 2] * d_[a]
        tk = np.array([np.fft.fftn(t) for t in tau])
        acc = np.zeros_like(tk)
        cnt = np.zeros(K.shape[1:])
        for sgn in range(8):
            flip = np.array([(sgn >> a) & 1 for a in range(3)], dtype=bool)
            use = np.all(nyq[flip], axis=0) if flip.any() else np.ones(K.shape[1:], dtype=bool)
            Kf = K.copy()
            for a in range(3):
                if flip[a]:
                    Kf[a] = np.where(nyq[a], -K[a], K[a])
            acc += green_apply(Kf, tk) * use
            cnt += use
        e = np.array([np.real(np.fft.ifftn(acc[a] / cnt)) for a in range(6)])
    return e


def test_elastostatic_matches_numpy_restatement_3d(gf, tmp_path):
    """Random 3-D polarisation in a rotated two-material box (no vacuum):
    the device solve equals the numpy restatement of the iteration."""
    D = gf.decks
    d = laminate_deck(gf, [(5, 2), (7, 1), (4, 2)], [D.pto(), D.ggg()], 16, limit=60, tol=1e-30)
    d.nx = d.ny = 8
    d.Tg2c = D.rotation(25.0, 40.0)
    d.scale_elasto = 1.2
    rng = np.random.default_rng(7)
    fe = d.material_cell() == 1
    d.p0 = rng.uniform(-0.3, 0.3, size=(3, 8, 8, 16)) * fe
    d.q0 = np.zeros_like(d.p0)
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0) as eng:
        used = eng.set_elastostatics(True)
        eps = eng.download("strain_static")
        eig = eng.download("eigenstrain_static")
    assert used == 60
    ref = numpy_khachaturyan(d, eig, 60)
    solid = d.material_cell() != 0
    assert np.max(np.abs((eps - ref)[:, solid])) <= 1e-11 * np.max(np.abs(ref))


def test_elastostatic_coupling_through_the_reference(gf, refrun, tmp_path):
    """The solved static strain and eigenstrain, handed to the reference as
    its restart inputs, give the same coupled run as the engine that solved
    them (the engine with the solve, bit for bit against the engine reading
    the files; the reference at 1e-10)."""
    d, steps, probe = static_decks(gf)["elastostatic_flag_only"]
    d.elasto_limit, d.elasto_tol = 400, 1e-13
    gf.decks.write_deck(d, str(tmp_path / "a"))
    with gf.Engine(str(tmp_path / "a"), device=0) as eng:
        eng.set_elastostatics(True)
        eps = eng.download("strain_static")
        eig = eng.download("eigenstrain_static")
        solved = engine_trace(eng, steps, probe)
    assert np.max(np.abs(eps)) > 1e-5
    # strain_stat.in holds the global frame: the deck has no rotation
    d2 = dataclasses.replace(d, strain_t0=eps, eig_t0=eig)
    gf.decks.write_deck(d2, str(tmp_path / "b"))
    with gf.Engine(str(tmp_path / "b"), device=0) as eng:
        from_files = engine_trace(eng, steps, probe)
    assert np.array_equal(solved, from_files)
    r = refrun.run(str(tmp_path / "b"), str(tmp_path / "ref"), steps=steps, probe=probe, dump=False)
    assert_trace_close(from_files, r["trace"])


def test_elastostatic_per_step_without_elastodynamics(gf, tmp_path):
    """Without elastodynamics the solve runs again after every step (from the
    last solution): after a step the static eigenstrain is that of the new
    p, and the strain that of the closed form."""
    D = gf.decks
    d = laminate_deck(gf, [(32, 1)], [D.pto()], 32, limit=4, tol=1e-14)
    d.dt = 2e-14                      # p moves by about 1e-2 per step under the Landau drive
    gf.decks.write_deck(d, str(tmp_path))
    p_start = d.p0.copy()
    with gf.Engine(str(tmp_path), device=0) as eng:
        eng.set_elastostatics(True)
        eng.advance(3)
        p = eng.download("p")
        eps = eng.download("strain_static")[:, 0, 0, :]
    assert np.max(np.abs(p[2] - p_start[2])) > 1e-4
    d.p0 = p
    want, _, _ = laminate_exact(d)
    assert np.max(np.abs(eps - want)) <= 1e-13 * np.max(np.abs(want))


# ---------------------------------------------------------------------------
# 1-D electrostatics
# ---------------------------------------------------------------------------
def elec_deck(gf, one_d, comp=False):
    D = gf.decks
    m = D.pto()
    m.er = 25.0
    d = D.Deck(nx=4, ny=4, nz=32, dx=1e-9, dy=1e-9, dz=1e-9, periodic=(True, True, True),
               layers=[(8, 2), (14, 1), (10, 0)], steps=4, dt=1e-16, materials=[m, D.ggg()], name="elec1d")
    d.elec_limit, d.elec_tol = 3000, 1e-14
    d.elec_1D, d.elec_1D_comp = one_d, comp
    z = np.arange(32)
    fe = d.material_cell() == 1
    d.p0 = np.zeros((3, 4, 4, 32))
    d.p0[2] = (0.25 + 0.05 * np.sin(2 * np.pi * z / 14))[None, None, :] * fe
    d.q0 = np.zeros_like(d.p0)
    return d


def test_elec_1d_equals_spectral_solve_for_uniform_layers(gf, tmp_path):
    out = {}
    for one_d in (False, True):
        d = elec_deck(gf, one_d)
        gf.decks.write_deck(d, str(tmp_path / str(one_d)))
        with gf.Engine(str(tmp_path / str(one_d)), device=0) as eng:
            eng.set_electrostatics(True)
            out[one_d] = eng.download("Estat")
    e1, es = out[True], out[False]
    assert np.max(np.abs(e1[:2])) == 0.0
    assert np.max(np.abs(e1 - es)) <= 1e-9 * np.max(np.abs(es))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
def test_elec_1d_compensated_closed_form(gf, tmp_path, precision, tol):
    d = elec_deck(gf, True, comp=True)
    d.dt = 2e-14
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0, precision=precision) as eng:
        p0 = eng.download("p")
        eng.set_electrostatics(True)
        assert np.max(np.abs(eng.download("Estat"))) == 0.0     # compensated: P = P(t0)
        eng.advance(3)
        p = eng.download("p")
        E = eng.download("Estat")
    mc = d.material_cell()
    er = np.array([1.0, d.materials[0].er, d.materials[1].er])[mc]
    dp = (p[2] - p0[2]) * (mc == 1)
    D_ = np.sum(dp / er, axis=2, keepdims=True) / np.sum(1.0 / er, axis=2, keepdims=True)
    want = -(dp - D_) / (E0 * er)
    assert np.max(np.abs(dp)) > 0
    assert np.max(np.abs(E[2] - want)) <= tol * np.max(np.abs(want))
