"""GPU tests of the discrete adjoint of the ferromagnetic RK4 step
(gf_adjoint_*), called through the C ABI.

The loss is the spectral power of the <m_x>(t) trace in a band of rfft bins;
the gradient is taken with respect to an x-directed excitation waveform
(piecewise constant over the run) and the per-cell damping alpha, through a
torch.autograd.Function that wraps the adjoint (test harness only).  The
check is FP64 central finite differences of the adjoint's own forward run.

Finite-difference steps (relative 1e-4): 1e-4 of the largest waveform sample
per waveform entry; for alpha, directional derivatives over all cells (the
uniform direction and a seeded +-1 pattern) with a step of 1e-4 of the mean
alpha (a single cell's damping moves the cell-averaged trace of a ~1 ps run
too little to difference it alone).  Tolerance 1e-4 relative; measured on the
B200: 8e-12 (waveform) and 4e-11 (alpha directions).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MU0 = 1.256637061e-6
BAND = slice(1, 9)


def film(gf, tmp_path, nx=32, ny=32, nz=8, steps=300):
    d = gf.decks.preset_fm_demag(nx=nx, ny=ny, nz=nz, steps=steps)
    d.Hext_table = None
    d.Hext_stat = (0.0, 0.0, 1.0 / MU0)
    d.materials[0].alpha = 0.02
    gf.decks.write_deck(d, str(tmp_path))
    return d


def spectral_loss_np(trace):
    return float(np.sum(np.abs(np.fft.rfft(trace)[BAND]) ** 2))


def test_adjoint_forward_matches_engine(gf, tmp_path):
    """With zero waveform and the material damping, the adjoint's forward run
    follows the engine's own FP64 RK4 step."""
    d = film(gf, tmp_path, nx=16, ny=16, nz=8, steps=40)
    with gf.Engine(str(tmp_path), device=0) as eng:
        with gf.Adjoint(eng, n_wave=4, checkpoint_every=16) as adj:
            tr = adj.forward(40)
            mfin = adj.final_m()
        ref = [eng.average("m")[0]]
        for _ in range(40):
            eng.advance(1)
            ref.append(eng.average("m")[0])
        m_eng = eng.download("m")
    assert np.max(np.abs(tr - np.array(ref))) <= 1e-12
    assert np.max(np.abs(mfin - m_eng)) <= 1e-12
    assert d.n == 16 * 16 * 8


def test_adjoint_gradients_match_finite_differences(gf, tmp_path):
    torch = pytest.importorskip("torch")
    steps, nw = 300, 8
    d = film(gf, tmp_path, steps=steps)
    mc = d.material_cell() == 1
    rng = np.random.default_rng(7)
    alpha0 = (0.02 * (1.0 + 0.1 * rng.random(d.n)) * mc.ravel()).astype(np.float64)
    tt = (np.arange(nw) + 0.5) / nw
    wave0 = (1e-2 / MU0) * np.sin(2 * np.pi * tt) * np.exp(-4.0 * (tt - 0.4) ** 2)

    with gf.Engine(str(tmp_path), device=0) as eng:
        with gf.Adjoint(eng, n_wave=nw, checkpoint_every=64) as adj:

            class Trace(torch.autograd.Function):
                @staticmethod
                def forward(ctx, wave, alpha):
                    adj.set_waveform(wave.detach().numpy())
                    adj.set_alpha(alpha.detach().numpy())
                    return torch.from_numpy(adj.forward(steps))

                @staticmethod
                def backward(ctx, g):
                    gw, ga = adj.backward(g.detach().contiguous().numpy())
                    return torch.from_numpy(gw), torch.from_numpy(ga)

            def loss_of(wave, alpha):
                adj.set_waveform(wave)
                adj.set_alpha(alpha)
                return spectral_loss_np(adj.forward(steps))

            w = torch.tensor(wave0, dtype=torch.float64, requires_grad=True)
            a = torch.tensor(alpha0, dtype=torch.float64, requires_grad=True)
            tr = Trace.apply(w, a)
            L = (torch.fft.rfft(tr)[BAND].abs() ** 2).sum()
            L.backward()
            gw = w.grad.numpy().copy()
            ga = a.grad.numpy().copy()
            Lv = float(L.detach())
            assert abs(Lv - loss_of(wave0, alpha0)) <= 1e-12 * abs(Lv)

            # waveform: every sample
            h = 1e-4 * np.max(np.abs(wave0))
            fd_w = np.empty(nw)
            for j in range(nw):
                wp, wm = wave0.copy(), wave0.copy()
                wp[j] += h
                wm[j] -= h
                fd_w[j] = (loss_of(wp, alpha0) - loss_of(wm, alpha0)) / (2 * h)
            err_w = np.max(np.abs(gw - fd_w)) / np.max(np.abs(fd_w))
            assert err_w <= 1e-4, f"waveform gradient vs FD: {err_w:.2e}"

            # damping: directional derivatives over all cells
            dirs = [mc.ravel().astype(np.float64),
                    np.where(rng.random(d.n) < 0.5, 1.0, -1.0) * mc.ravel()]
            for v in dirs:
                ha = 1e-4 * float(np.mean(alpha0[mc.ravel()]))
                fd = (loss_of(wave0, alpha0 + ha * v) - loss_of(wave0, alpha0 - ha * v)) / (2 * ha)
                ad = float(ga @ v)
                assert abs(ad - fd) <= 1e-4 * abs(fd), f"alpha directional gradient {ad:.6e} vs FD {fd:.6e}"
            # no gradient on non-magnetic cells, and none from cells outside the film
            assert np.all(ga[~mc.ravel()] == 0.0)


def test_adjoint_checkpoint_interval_does_not_change_gradients(gf, tmp_path):
    steps, nw = 50, 5
    film(gf, tmp_path, nx=16, ny=16, nz=8, steps=steps)
    out = []
    with gf.Engine(str(tmp_path), device=0) as eng:
        for every in (7, 1000):
            with gf.Adjoint(eng, n_wave=nw, checkpoint_every=every) as adj:
                adj.set_waveform(np.linspace(-3e3, 5e3, nw))
                tr = adj.forward(steps)
                g = np.cos(0.3 * np.arange(steps + 1))
                out.append((tr,) + adj.backward(g))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["fm_film", "magnetoelastic"])
def test_adjoint_stage_store_and_recompute_layouts_agree(gf, tmp_path, case, precision):
    """The backward run with every step's stages kept (stage store) and with
    the stages recomputed per step from the stored step values gives the same
    gradients bit for bit, over blocks that do not divide the run (23 steps,
    checkpoints every 7), and a byte limit below one block's store selects
    the recompute layout."""
    steps, nw = 23, 5
    if case == "fm_film":
        film(gf, tmp_path, nx=16, ny=16, nz=8, steps=steps)
    else:
        me_film(gf, tmp_path, nx=16, ny=16, nz=8, steps=steps)
    n = 16 * 16 * 8
    slot = (48 if case == "magnetoelastic" else 24) * n * (4 if precision == "mixed" else 8)
    out, layouts = [], []
    with gf.Engine(str(tmp_path), device=0, precision=precision) as eng:
        eng.advance(3)
        for limit in (-1, 0, 7 * slot - 1, 7 * slot):
            with gf.Adjoint(eng, n_wave=nw, checkpoint_every=7) as adj:
                adj.set_store_limit(limit)
                adj.set_waveform(np.linspace(-3e3, 5e3, nw))
                tr = adj.forward(steps)
                g = np.cos(0.3 * np.arange(steps + 1))
                out.append((tr,) + adj.backward(g))
                layouts.append(adj.store_info())
    assert [u for u, _ in layouts] == [True, False, False, True]
    assert layouts[0][1] == 7 * slot and layouts[3][1] == 7 * slot
    assert np.max(np.abs(out[0][1])) > 0.0 and np.max(np.abs(out[0][2])) > 0.0
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert np.array_equal(a, b)


def test_adjoint_rejects_unsupported_decks(gf, tmp_path):
    d = gf.decks.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=5)
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0) as eng:
        with pytest.raises(gf.GFError) as ei:
            gf.Adjoint(eng, n_wave=4)
        assert ei.value.code == -7


# ---------------------------------------------------------------------------
# magnetoelastic coupling with elastodynamics (the adjoint configuration's
# physics): the stress divergence with the magnetostrictive eigenstrain, the
# magnetoelastic field of the cell strain, the elastic RK4 with step-start
# mass damping and the stiffness-damping force store, and the Liao boundary
# at k = 0 are transposed.  The film's magnetostriction is raised 100x so the
# elastic path changes the gradients by far more than the FD tolerance.
# ---------------------------------------------------------------------------
def me_film(gf, tmp_path, nx=16, ny=16, nz=8, steps=200, boost=100.0):
    D = gf.decks
    d = D.preset_fm_demag(nx=nx, ny=ny, nz=nz, steps=steps)
    d.Hext_table = None
    d.Hext_stat = (0.0, 0.0, 1.0 / MU0)
    m = D.yig(0.02, magnetoelastic=True)
    m.lam100 *= boost
    m.lam111 *= boost
    d.materials = [m]
    d.elastic, d.elasto_back, d.elasto_on = True, True, True
    d.abc_1D, d.liao_w = False, 0.5
    gf.decks.write_deck(d, str(tmp_path))
    return d


def test_adjoint_forward_matches_engine_magnetoelastic(gf, tmp_path):
    me_film(gf, tmp_path, steps=40)
    with gf.Engine(str(tmp_path), device=0) as eng:
        with gf.Adjoint(eng, n_wave=4, checkpoint_every=16) as adj:
            tr = adj.forward(40)
            mfin = adj.final_m()
        ref = [eng.average("m")[0]]
        for _ in range(40):
            eng.advance(1)
            ref.append(eng.average("m")[0])
        m_eng = eng.download("m")
        u_eng = eng.download("u")
    assert np.max(np.abs(u_eng)) > 0.0
    assert np.max(np.abs(tr - np.array(ref))) <= 1e-12
    assert np.max(np.abs(mfin - m_eng)) <= 1e-12


def _grads(gf, tmp_path, d, steps, nw, wave0, alpha0, fd, precision="fp64"):
    with gf.Engine(str(tmp_path), device=0, precision=precision) as eng:
        with gf.Adjoint(eng, n_wave=nw, checkpoint_every=64) as adj:
            def loss_of(wave, alpha):
                adj.set_waveform(wave)
                adj.set_alpha(alpha)
                return spectral_loss_np(adj.forward(steps))
            adj.set_waveform(wave0)
            adj.set_alpha(alpha0)
            tr = adj.forward(steps)
            X = np.fft.rfft(tr)
            n = np.arange(tr.size)
            g = np.zeros(tr.size)
            for k in range(BAND.start, BAND.stop):
                g += 2.0 * np.real(np.conj(X[k]) * np.exp(-2j * np.pi * k * n / tr.size))
            gw, ga = adj.backward(g)
            if not fd:
                return gw, ga, None
            h = 1e-4 * np.max(np.abs(wave0))
            fd_w = np.empty(nw)
            for j in range(nw):
                wp, wm = wave0.copy(), wave0.copy()
                wp[j] += h
                wm[j] -= h
                fd_w[j] = (loss_of(wp, alpha0) - loss_of(wm, alpha0)) / (2 * h)
            mc = d.material_cell().ravel() == 1
            rng = np.random.default_rng(3)
            v = np.where(rng.random(d.n) < 0.5, 1.0, -1.0) * mc
            ha = 1e-4 * float(np.mean(alpha0[mc]))
            fd_a = (loss_of(wave0, alpha0 + ha * v) - loss_of(wave0, alpha0 - ha * v)) / (2 * ha)
            return gw, ga, (fd_w, v, fd_a)


def test_adjoint_gradients_magnetoelastic_match_finite_differences(gf, tmp_path):
    steps, nw = 200, 8
    d = me_film(gf, tmp_path / "me", steps=steps)
    mc = d.material_cell().ravel() == 1
    rng = np.random.default_rng(5)
    alpha0 = 0.02 * (1.0 + 0.1 * rng.random(d.n)) * mc
    tt = (np.arange(nw) + 0.5) / nw
    wave0 = (1e-2 / MU0) * np.sin(2 * np.pi * tt) * np.exp(-4.0 * (tt - 0.4) ** 2)
    gw, ga, (fd_w, v, fd_a) = _grads(gf, tmp_path / "me", d, steps, nw, wave0, alpha0, True)
    err_w = np.max(np.abs(gw - fd_w)) / np.max(np.abs(fd_w))
    assert err_w <= 1e-4, f"waveform gradient vs FD: {err_w:.2e}"
    ad = float(ga @ v)
    assert abs(ad - fd_a) <= 1e-4 * abs(fd_a), f"alpha directional gradient {ad:.6e} vs FD {fd_a:.6e}"
    # the elastic path matters: without magnetostriction the gradients differ
    d0 = me_film(gf, tmp_path / "plain", steps=steps, boost=0.0)
    gw0, _, _ = _grads(gf, tmp_path / "plain", d0, steps, nw, wave0, alpha0, False)
    assert np.max(np.abs(gw - gw0)) > 1e-2 * np.max(np.abs(gw))


# ---------------------------------------------------------------------------
# the FP32 mixed adjoint: on a mixed-form engine the adjoint's forward run,
# stage fields and cotangents are FP32 (step values compensated, the
# engine's own FP32 elastic kernels), the damping and waveform gradients are
# accumulated in FP64.  Gradients are checked against FP64 central finite
# differences (the FP64 engine's adjoint forward run, relative step 1e-4)
# at the same 1e-4 tolerance.
# ---------------------------------------------------------------------------
def test_mixed_adjoint_forward_follows_the_engines(gf, tmp_path):
    """The FP32 adjoint's <m_x> trace and final m follow the mixed engine's
    step (which also renormalises |m| every stage) and the FP64 engine's to
    FP32 resolution."""
    me_film(gf, tmp_path, steps=40)
    out = {}
    for prec in ("mixed", "fp64"):
        with gf.Engine(str(tmp_path), device=0, precision=prec) as eng:
            if prec == "mixed":
                with gf.Adjoint(eng, n_wave=4, checkpoint_every=16) as adj:
                    out["adj_tr"] = adj.forward(40)
                    out["adj_m"] = adj.final_m()
            ref = [eng.average("m")[0]]
            for _ in range(40):
                eng.advance(1)
                ref.append(eng.average("m")[0])
            out[prec + "_tr"] = np.array(ref)
            out[prec + "_m"] = eng.download("m")
    for prec in ("mixed", "fp64"):
        e_tr = np.max(np.abs(out["adj_tr"] - out[prec + "_tr"]))
        e_m = np.max(np.abs(out["adj_m"] - out[prec + "_m"]))
        assert e_tr <= 1e-6 and e_m <= 1e-6, f"{prec}: trace {e_tr:.2e}, m {e_m:.2e}"


@pytest.mark.parametrize("case", ["fm_film", "magnetoelastic"])
def test_mixed_adjoint_gradients_match_fp64_finite_differences(gf, tmp_path, case):
    nw = 8
    if case == "fm_film":
        steps = 300
        d = film(gf, tmp_path, steps=steps)
    else:
        steps = 200
        d = me_film(gf, tmp_path, steps=steps)
    mc = d.material_cell().ravel() == 1
    rng = np.random.default_rng(11)
    alpha0 = 0.02 * (1.0 + 0.1 * rng.random(d.n)) * mc
    tt = (np.arange(nw) + 0.5) / nw
    wave0 = (1e-2 / MU0) * np.sin(2 * np.pi * tt) * np.exp(-4.0 * (tt - 0.4) ** 2)
    gw, ga, _ = _grads(gf, tmp_path, d, steps, nw, wave0, alpha0, False, precision="mixed")
    gw64, ga64, (fd_w, v, fd_a) = _grads(gf, tmp_path, d, steps, nw, wave0, alpha0, True)
    err_w = np.max(np.abs(gw - fd_w)) / np.max(np.abs(fd_w))
    assert err_w <= 1e-4, f"FP32 waveform gradient vs FP64 FD: {err_w:.2e}"
    ad = float(ga @ v)
    assert abs(ad - fd_a) <= 1e-4 * abs(fd_a), f"FP32 alpha directional gradient {ad:.6e} vs FP64 FD {fd_a:.6e}"
    # per cell against the FP64 adjoint (FP32 resolution of each cell's share)
    err_a = np.max(np.abs(ga - ga64)) / np.max(np.abs(ga64))
    assert err_a <= 1e-3, f"FP32 per-cell alpha gradient vs FP64 adjoint: {err_a:.2e}"
    print(f"{case}: waveform {err_w:.2e}, alpha direction {abs(ad - fd_a) / abs(fd_a):.2e}, per cell {err_a:.2e}")
