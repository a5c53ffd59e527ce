"""CPU restatement (numpy) of GO-Ferro's ferromagnetic LLG + FFT
magnetostatics RK4 time step — the CPU-runnable benchmark configuration
(FM LLG + demag, no elasticity, no Maxwell fields).

TEST INFRASTRUCTURE ONLY: imported by tests/ as an independent checker of
the compiled reference (oracle/_ref) and of the CUDA engine.  Nothing in the
product path uses it.

It restates, array-wise, the algorithm of these reference functions:
  * Newell demag tensor tables    magnetic_initialize.cpp:1176-1402 (windowed,
    wrapped, 1/n pre-applied) with F2/F1/A/G2/G1/B :1404-1557
  * get_H_static                  magnetostatic_solver.cpp:114-187
    (M = Ms m, forward FFT, N_k . M_k, inverse FFT, / (-dx dy dz))
  * get_dm_RK{1..4}               magnetic_solver.cpp:3-229 (anisotropy types
    1 and 2, harmonic-mean exchange, interfacial DMI, static + external field)
  * get_m_spatial_derivative_local magnetic_solver.cpp:1639-1831 (one-sided
    slopes, DMI interface slope +-D/2A m, zero slope on z interfaces)
  * update_m_RK{1,2,3}, get_dm, update_m magnetic_solver.cpp:1131-1146, 1515-1636
    (no |m| renormalisation; the increment is summed before it is added)
  * time_marching_device_serial   global.cpp:512-549 (prescribed H table) and
    update_external_Hfield*       magnetic_solver.cpp:1834-1861
  * get_averagem                  magnetic_solver.cpp:1863-1888 (sum over all
    cells / number of FM cells)

Inputs are plain arrays and scalars (see run()); the frame rotation is taken
as the identity (if_OrientRotate false).  Results agree with the compiled
reference to rounding: the FFT and numpy's transcendental functions differ
from the reference's host build by a few ulps.
"""
from __future__ import annotations

import math

import numpy as np

MU0 = 1.256637061e-6        # magnetic_system.h:14
PI = 3.14159265358979323846
S = 1.0e-33                 # threshold of the Newell branches


def _f2(x, y, z):
    """Newell F2 (magnetic_initialize.cpp:1427-1476), vectorised."""
    u, v, w = x * x, y * y, z * z
    r = np.sqrt(u + v + w)
    ax, ay, az = np.abs(x), np.abs(y), np.abs(z)
    with np.errstate(all="ignore"):
        b0 = z * (u - v) * np.log(r - z) / 2. + y * (u - w) * np.log(r - y) / 2. \
            - x * y * z * np.arctan(y * z / (x * r)) + (2. * u - v - w) * r / 6.
        b1 = -(z * v / 2.) * np.log(r - z) - (y * w / 2.) * np.log(r - y) - r * r * r / 6.
        b2 = (z * u / 2.) * np.log(r - z) + (2. * u - w) * r / 6.
        b3 = (y * u / 2.) * np.log(r - y) + (2. * u - v) * r / 6.
    f = np.zeros_like(x)
    conds = [(ax > S) & (ay > S) & (az > S), (ax < S) & (ay > S) & (az > S), (ax > S) & (ay < S) & (az > S),
             (ax > S) & (ay > S) & (az < S), (ax < S) & (ay < S) & (az > S), (ax < S) & (ay > S) & (az < S),
             (ax > S) & (ay < S) & (az < S)]
    vals = [b0, b1, b2, b3, -az * az * az / 6., -ay * ay * ay / 6., ax * ax * ax / 3.]
    done = np.zeros(x.shape, dtype=bool)
    for c, val in zip(conds, vals):
        sel = c & ~done
        f = np.where(sel, val, f)
        done |= sel
    return f


def _f1(x, y, z, dy):
    """Newell F1 (magnetic_initialize.cpp:1419-1425)."""
    return 2. * _f2(x, y, z) - _f2(x, y - dy, z) - _f2(x, y + dy, z)


def _a(x, y, z, dx, dy, dz):
    """Newell A (magnetic_initialize.cpp:1404-1417)."""
    xp, xm, zp, zm = x + dx, x - dx, z + dz, z - dz
    return (4. * _f1(x, y, z, dy) - 2. * _f1(x, y, zp, dy) - 2. * _f1(x, y, zm, dy) - 2. * _f1(xp, y, z, dy)
            + _f1(xp, y, zp, dy) + _f1(xp, y, zm, dy) - 2. * _f1(xm, y, z, dy) + _f1(xm, y, zp, dy) + _f1(xm, y, zm, dy))


def _g2(x, y, z):
    """Newell G2 (magnetic_initialize.cpp:1507-1557), vectorised."""
    u, v, w = x * x, y * y, z * z
    r = np.sqrt(u + v + w)
    with np.errstate(all="ignore"):
        b0 = (y * y * y / 6. - y * w / 2.) * np.log(r + x) + (x / 6.) * (3. * w - u) * np.log(r - y) + x * y * r / 3. \
            + x * y * z * np.log(r - z) + (v * z / 2.) * np.arctan(x * z / (r * y)) \
            + (z * z * z / 6.) * np.arctan(x * y / (r * z)) + (u * z / 2.) * np.arctan(y * z / (r * x))
        b1 = (y * y * y / 6. - y * w / 2.) * np.log(r)
        b2 = (x * w / 2. - x * x * x / 6.) * np.log(r)
        b3 = ((y * y * y) / 6.) * np.log(r + x) - (x * x * x / 6.) * np.log(r - y) + x * y * r / 3.
        b5 = (y * y * y) / 12. * np.log(v)
        b6 = -((x * x * x) / 12.) * np.log(u)
    conds = [np.abs(x * y * z) > S, (np.abs(x) < S) & (np.abs(y * z) > S), (np.abs(x * z) > S) & (np.abs(y) < S),
             (np.abs(x * y) > S) & (np.abs(z) < S), ((np.abs(x) + np.abs(y)) < S) & (np.abs(z) > S),
             ((np.abs(x) + np.abs(z)) < S) & (np.abs(y) > S), (np.abs(x) > S) & ((np.abs(y) + np.abs(z)) < S)]
    vals = [b0, b1, b2, b3, np.zeros_like(x), b5, b6]
    g = np.zeros_like(x)
    done = np.zeros(x.shape, dtype=bool)
    for c, val in zip(conds, vals):
        sel = c & ~done
        g = np.where(sel, val, g)
        done |= sel
    return g


def _g1(x, y, z, dx, dy, dz):
    """Newell G1 (magnetic_initialize.cpp:1486-1505)."""
    xp, xm, yp, ym, zp, zm = x + dx, x - dx, y + dy / 2., y - dy / 2., z + dz, z - dz
    return (4. * _g2(x, yp, z) - 4. * _g2(x, ym, z) - 2. * _g2(x, yp, zp) + 2. * _g2(x, ym, zp)
            - 2. * _g2(x, yp, zm) + 2. * _g2(x, ym, zm) - 2. * _g2(xm, yp, z) + 2. * _g2(xm, ym, z)
            + _g2(xm, yp, zp) - _g2(xm, ym, zp) + _g2(xm, yp, zm) - _g2(xm, ym, zm)
            - 2. * _g2(xp, yp, z) + 2. * _g2(xp, ym, z) + _g2(xp, yp, zp) - _g2(xp, ym, zp)
            + _g2(xp, yp, zm) - _g2(xp, ym, zm))


def _b(x, y, z, dx, dy, dz):
    """Newell B (magnetic_initialize.cpp:1478-1484)."""
    return _g1(x, y + dy / 2., z, dx, dy, dz) - _g1(x, y - dy / 2., z, dx, dy, dz)


def _offsets(n):
    """Signed offset of each wrapped index (the reference's window of
    n/2-1 on each side, entries outside it zero), and the in-window mask."""
    a = np.arange(n)
    h = n // 2
    off = np.where(a <= h - 1, a, a - n)
    ok = (a <= h - 1) | (a >= n - h + 1)
    return off, ok


def demag_spectra(nx, ny, nz, dx, dy, dz):
    """Forward FFTs of the nine tables Axyz, Ayzx, Azxy, Bxyz, Byzx, Bzxy,
    Byxz, Bzyx, Bxzy (magnetic_initialize.cpp:1176-1402), each divided by
    4 pi and by n."""
    oi, mi = _offsets(nx)
    oj, mj = _offsets(ny)
    ok, mk = _offsets(nz)
    X, Y, Z = np.meshgrid(oi * dx, oj * dy, ok * dz, indexing="ij")
    inside = mi[:, None, None] & mj[None, :, None] & mk[None, None, :]
    fourpi, nn = 2. * (2. * PI), float(nx * ny * nz)
    tabs = [_a(X, Y, Z, dx, dy, dz), _a(Y, Z, X, dy, dz, dx), _a(Z, X, Y, dz, dx, dy),
            _b(X, Y, Z, dx, dy, dz), _b(Y, Z, X, dy, dz, dx), _b(Z, X, Y, dz, dx, dy),
            _b(Y, X, Z, dy, dx, dz), _b(Z, Y, X, dz, dy, dx), _b(X, Z, Y, dx, dz, dy)]
    return [np.fft.rfftn(np.where(inside, t / fourpi / nn, 0.)) for t in tabs]


def h_static(Nk, M, dx, dy, dz):
    """get_H_static (magnetostatic_solver.cpp:114-187): unnormalised forward
    transform of M, tensor product, unnormalised inverse, / (-dx dy dz)."""
    shape = M[0].shape
    n = M[0].size
    mx, my, mz = (np.fft.rfftn(c) for c in M)
    hx = mx * Nk[0] + my * Nk[3] + mz * Nk[8]
    hy = my * Nk[1] + mz * Nk[4] + mx * Nk[6]
    hz = mz * Nk[2] + mx * Nk[5] + my * Nk[7]
    vol_neg = -dx * dy * dz
    return np.stack([np.fft.irfftn(h / vol_neg, s=shape, axes=(0, 1, 2)) * n for h in (hx, hy, hz)])


def _shift(a, d, s):
    """a at the neighbour +1 (s=+1) or -1 (s=-1) along axis d, periodic wrap."""
    return np.roll(a, -s, axis=d)


def dm_fm(m, mid, mats, dx, dy, dz, periodic, Hstat, Hext, dt):
    """get_dm_RK* for every FM cell (magnetic_solver.cpp:3-229 with
    get_m_spatial_derivative_local :1639-1831); 0 elsewhere."""
    tab = lambda key: np.array([0.] + [float(mt.get(key, 0.)) for mt in mats])
    isfm = np.array([False] + [bool(mt.get("fm", False)) for mt in mats])[mid]
    Ms, A, D = tab("Ms")[mid], tab("Aex")[mid], tab("iDMI")[mid]
    K1, K2, alpha, gyro = tab("K1")[mid], tab("K2")[mid], tab("alpha")[mid], tab("gyro")[mid]
    aniso = np.array([0] + [int(mt.get("aniso_type", 0)) for mt in mats])[mid]
    with np.errstate(all="ignore"):
        dA = np.where(isfm, D / 2. / A, 0.)
        K1c, K2c = K1 / MU0 / Ms, K2 / MU0 / Ms
        exc, dmic = 2. / MU0 / Ms, 2. * D / MU0 / Ms
        prec = -gyro / (1 + alpha * alpha) * dt
    Avals = tab("Aex")
    with np.errstate(all="ignore"):
        Apair = np.where(Avals[:, None] + Avals[None, :] != 0.,
                         2. * Avals[:, None] * Avals[None, :] / (Avals[:, None] + Avals[None, :]), 0.)
    h = (dx, dy, dz)
    shape = mid.shape
    idx = [np.arange(shape[d]).reshape([-1 if e == d else 1 for e in range(3)]) for d in range(3)]
    slopes_b, slopes_f, Aface_b, Aface_f = [], [], [], []
    for d in range(3):
        n = shape[d]
        nb_b, nb_f = _shift(mid, d, -1), _shift(mid, d, +1)
        isfm_b = np.array([False] + [bool(mt.get("fm", False)) for mt in mats])[nb_b]
        isfm_f = np.array([False] + [bool(mt.get("fm", False)) for mt in mats])[nb_f]
        sb = ((idx[d] == 0) & (not periodic[d])) | ~isfm_b
        sf = ((idx[d] == n - 1) & (not periodic[d])) | ~isfm_f
        mb = [_shift(m[a], d, -1) for a in range(3)]
        mf = [_shift(m[a], d, +1) for a in range(3)]
        # interface slopes: x faces (-dA mz, 0, dA mx), y faces (0, -dA mz, dA my), z faces 0
        surf = [np.zeros(shape) for _ in range(3)]
        if d == 0:
            surf = [-dA * m[2], np.zeros(shape), dA * m[0]]
        elif d == 1:
            surf = [np.zeros(shape), -dA * m[2], dA * m[1]]
        gb = [np.where(sb, surf[a], (m[a] - mb[a]) / h[d]) for a in range(3)]
        gf = [np.where(sf, surf[a], (mf[a] - m[a]) / h[d]) for a in range(3)]
        slopes_b.append(gb)
        slopes_f.append(gf)
        Aface_b.append(np.where(sb, A, Apair[mid, nb_b]))
        Aface_f.append(np.where(sf, A, Apair[mid, nb_f]))
    Hex = []
    for a in range(3):
        acc = (Aface_f[0] * (slopes_f[0][a] / dx) + Aface_b[0] * (-slopes_b[0][a] / dx)
               + Aface_f[1] * (slopes_f[1][a] / dy) + Aface_b[1] * (-slopes_b[1][a] / dy)
               + Aface_f[2] * (slopes_f[2][a] / dz) + Aface_b[2] * (-slopes_b[2][a] / dz))
        Hex.append(exc * acc)
    mx, my, mz = m
    cub = aniso == 1
    uni = aniso == 2
    hax = np.where(cub, -2. * (K1c * (my * my + mz * mz) + K2c * my * my * mz * mz) * mx, 0.)
    hay = np.where(cub, -2. * (K1c * (mx * mx + mz * mz) + K2c * mx * mx * mz * mz) * my, 0.)
    haz = np.where(cub, -2. * (K1c * (mx * mx + my * my) + K2c * mx * mx * my * my) * mz, np.where(uni, 2. * K1c * mz, 0.))
    dmxdx = (slopes_b[0][0] + slopes_f[0][0]) * 0.5
    dmzdx = (slopes_b[0][2] + slopes_f[0][2]) * 0.5
    dmydy = (slopes_b[1][1] + slopes_f[1][1]) * 0.5
    dmzdy = (slopes_b[1][2] + slopes_f[1][2]) * 0.5
    Hd = [dmic * dmzdx, dmic * dmzdy, -dmic * (dmxdx + dmydy)]
    Ha = [hax, hay, haz]
    H = [Hstat[a] + Ha[a] + 0. + Hex[a] + Hd[a] + Hext[a] for a in range(3)]
    px = my * H[2] - mz * H[1]
    py = mz * H[0] - mx * H[2]
    pz = mx * H[1] - my * H[0]
    qx = my * pz - mz * py
    qy = mz * px - mx * pz
    qz = mx * py - my * px
    out = [prec * px + alpha * prec * qx, prec * py + alpha * prec * qy, prec * pz + alpha * prec * qz]
    return np.stack([np.where(isfm, o, 0.) for o in out])


def run(mid, mats, dx, dy, dz, periodic, m0, dt, steps, magnetostatics=True, Hext_table=None,
        Hext_stat=(0., 0., 0.), Hext_altr=(0., 0., 0.), H_altr_freq=(0., 0., 0.)):
    """Advance m0 by `steps` RK4 steps (main.cpp:243-484 restricted to the
    magnetic system).  mats: list of dicts with keys fm, Ms, Aex, iDMI,
    aniso_type, K1, K2, alpha, gyro (1-based ids in mid).  Returns
    (trace of <m> per step including step 0, final m, final H_stat)."""
    m = np.array(m0, dtype=np.float64)
    isfm = np.array([False] + [bool(mt.get("fm", False)) for mt in mats])[mid]
    Msc = np.array([0.] + [float(mt.get("Ms", 0.)) for mt in mats])[mid]
    nfm = int(isfm.sum())
    Nk = demag_spectra(*mid.shape, dx, dy, dz) if magnetostatics else None

    def hstat(mm):
        if not magnetostatics:
            return np.zeros_like(mm)
        M = np.stack([np.where(isfm, Msc * mm[a], 0.) for a in range(3)])
        return h_static(Nk, M, dx, dy, dz)

    Hs = hstat(m)
    trace = [m.sum(axis=(1, 2, 3)) / nfm]
    t = 0.
    pidx = 0
    for _ in range(steps):
        t = t + dt
        if Hext_table is not None:
            tt = Hext_table[:, 0]
            if pidx < len(tt) and (t - dt) > tt[pidx]:
                pidx += 1
            Hp = Hext_table[pidx, 1:4] if pidx < len(tt) else np.zeros(3)
        lt = (t - dt, t - dt * 0.5, t - dt * 0.5, t)
        ks = []
        store = m
        for s in range(4):
            if Hext_table is not None:
                He = Hp
            else:
                He = [Hext_stat[a] + Hext_altr[a] * math.sin(2. * PI * H_altr_freq[a] * lt[s]) for a in range(3)]
            k = dm_fm(store, mid, mats, dx, dy, dz, periodic, Hs, He, dt)
            ks.append(k)
            if s < 2:
                store = m + k * 0.5
            elif s == 2:
                store = m + k
            else:
                m = m + (ks[0] / 6. + ks[1] / 3. + ks[2] / 3. + ks[3] / 6.)
                store = m
            Hs = hstat(store)
        trace.append(m.sum(axis=(1, 2, 3)) / nfm)
    return np.array(trace), m, Hs
