// Discrete adjoint of the ferromagnetic RK4 step (FP64).
//
// The adjoint differentiates the engine's own discretisation of
// magnetic_system::get_dm_RK{1..4} (magnetic_solver.cpp:3-229) and the RK4
// combination update_m_RK*/update_m (:1515-1636), restricted to the terms a
// sensitivity study of a ferromagnetic film needs: harmonic-mean exchange
// (interface slope 0, no DMI), cubic or uniaxial anisotropy without frame
// rotation, the periodic FFT magnetostatic field of every stage
// (magnetostatic_solver.cpp:114-219) and a uniform external field.  Two
// inputs the reference keeps per material become per cell / per step here:
// the damping alpha (an array over cells) and an x-directed excitation
// waveform added to the external field, piecewise constant over `nw`
// segments of the run.
//
// Forward stage s at state y (k = dt-scaled increment):
//   H = H_demag(y) + ex_c sum_f w_cf (y_f - y_c) + H_anis(y) + H_ext + w e_x
//   k = c1 (y x H) + c2 y x (y x H),  c1 = -gamma dt / (1 + alpha^2), c2 = alpha c1
// Vector-Jacobian product with cotangent u of k:
//   ybar = c1 (H x u) + c2 ((y x H) x u + H x (u x y)) + J_anis^T Hbar
//          + exchange^T Hbar + Ms K Hbar   (K: the demag convolution, symmetric)
//   Hbar = c1 (u x y) + c2 ((u x y) x y)
//   alphabar += u . (dc1 (y x H) + dc2 y x (y x H))
//   wbar[segment] += sum over cells of Hbar_x
// RK4 reverse sweep for lambda = d loss / d x_{n+1}:
//   u4 = lambda/6, u3 = lambda/3 + ybar4, u2 = lambda/3 + ybar3/2,
//   u1 = lambda/6 + ybar2/2, lambda_n = lambda + ybar4 + ybar3 + ybar2 + ybar1.
#pragma once

#include "gf_state.cuh"

namespace gf {

// per-material constants of the adjoint's dynamics
struct AdjMat {
    double gdt;        // gamma * dt (the material's gyro times the time step)
    double Ms, ex_coef, Aex, K1c, K2c;
    int aniso;
    uint32_t fm;
};

__device__ inline double3 cross3(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ inline double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline double3 ld3(const F3& f, int c) { return make_double3(f.c[0][c], f.c[1][c], f.c[2][c]); }
__device__ inline void st3(const F3& f, int c, double3 v) { f.c[0][c] = v.x; f.c[1][c] = v.y; f.c[2][c] = v.z; }

// neighbour cells with periodic wrap and the exchange weight A_cf / dx_f^2
// of each face (0 on ferromagnetic surfaces and non-periodic boundaries)
struct AdjNbr {
    int nb[6];
    double w[6];
};
__device__ inline void adj_neighbours(const Params& P, const uint8_t* mid, const AdjMat* am, const double* aij, int nmat,
                                      int i, int j, int k, uint8_t id, AdjNbr& n) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ib = (i == 0) ? nx - 1 : i - 1, iF = (i == nx - 1) ? 0 : i + 1;
    const int jb = (j == 0) ? ny - 1 : j - 1, jF = (j == ny - 1) ? 0 : j + 1;
    const int kb = (k == 0) ? nz - 1 : k - 1, kF = (k == nz - 1) ? 0 : k + 1;
    n.nb[0] = (ib * ny + j) * nz + k; n.nb[1] = (iF * ny + j) * nz + k;
    n.nb[2] = (i * ny + jb) * nz + k; n.nb[3] = (i * ny + jF) * nz + k;
    n.nb[4] = (i * ny + j) * nz + kb; n.nb[5] = (i * ny + j) * nz + kF;
    const bool edge[6] = {i == 0 && !P.per_x, i == nx - 1 && !P.per_x, j == 0 && !P.per_y,
                          j == ny - 1 && !P.per_y, k == 0 && !P.per_z, k == nz - 1 && !P.per_z};
    const double r2[3] = {P.rdx * P.rdx, P.rdy * P.rdy, P.rdz * P.rdz};
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const uint8_t q = mid[n.nb[f]];
        const bool fmq = q != 0 && am[q - 1].fm;
        n.w[f] = (edge[f] || !fmq) ? 0. : aij[id * (nmat + 1) + q] * r2[f / 2];
    }
}

// One RK stage of the adjoint's forward dynamics at state y with demag field
// hd: writes the effective field H (kept for the reverse sweep) and the RK4
// combination with step value x and increment sum acc (stage 3 updates x in
// place; stages 0-2 write the next stage state ynext).
template <int S>
__global__ void __launch_bounds__(256) k_adj_eval(Params P, const uint8_t* __restrict__ mid, const AdjMat* __restrict__ am,
                                                  const double* __restrict__ aij, int nmat, F3 y, F3 hd,
                                                  const double* __restrict__ alpha, double3 hext, F3 hs, F3 x, F3 acc,
                                                  F3 ynext) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const int nyz = P.ny * P.nz;
    const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const uint8_t id = mid[c];
    double3 kk = make_double3(0., 0., 0.);
    if (id != 0 && am[id - 1].fm) {
        const AdjMat& mt = am[id - 1];
        AdjNbr n;
        adj_neighbours(P, mid, am, aij, nmat, i, j, k, id, n);
        const double3 m = ld3(y, c);
        double3 hex = make_double3(0., 0., 0.);
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const double3 mf = ld3(y, n.nb[f]);
            hex.x += n.w[f] * (mf.x - m.x); hex.y += n.w[f] * (mf.y - m.y); hex.z += n.w[f] * (mf.z - m.z);
        }
        double3 H = ld3(hd, c);
        H.x += mt.ex_coef * hex.x + hext.x; H.y += mt.ex_coef * hex.y + hext.y; H.z += mt.ex_coef * hex.z + hext.z;
        if (mt.aniso == 1) {
            H.x += -2. * (mt.K1c * (m.y * m.y + m.z * m.z) + mt.K2c * m.y * m.y * m.z * m.z) * m.x;
            H.y += -2. * (mt.K1c * (m.x * m.x + m.z * m.z) + mt.K2c * m.x * m.x * m.z * m.z) * m.y;
            H.z += -2. * (mt.K1c * (m.x * m.x + m.y * m.y) + mt.K2c * m.x * m.x * m.y * m.y) * m.z;
        } else if (mt.aniso == 2) {
            H.z += 2. * mt.K1c * m.z;
        }
        st3(hs, c, H);
        const double a = alpha[c];
        const double c1 = -mt.gdt / (1. + a * a), c2 = a * c1;
        const double3 p = cross3(m, H), q = cross3(m, p);
        kk = make_double3(c1 * p.x + c2 * q.x, c1 * p.y + c2 * q.y, c1 * p.z + c2 * q.z);
    } else {
        st3(hs, c, make_double3(0., 0., 0.));
    }
    const double kv[3] = {kk.x, kk.y, kk.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double xv = x.c[a][c];
        if (S == 0) { acc.c[a][c] = kv[a] / 6.; ynext.c[a][c] = xv + kv[a] * 0.5; }
        else if (S == 1) { acc.c[a][c] = acc.c[a][c] + kv[a] / 3.; ynext.c[a][c] = xv + kv[a] * 0.5; }
        else if (S == 2) { acc.c[a][c] = acc.c[a][c] + kv[a] / 3.; ynext.c[a][c] = xv + kv[a]; }
        else { x.c[a][c] = xv + (acc.c[a][c] + kv[a] / 6.); }
    }
}

// Local part of the vector-Jacobian product of stage s: the cross products,
// the anisotropy Jacobian, the damping derivative; writes ybar (local part),
// Hbar and Hbar_x (for the waveform reduction); adds alphabar.
static __global__ void __launch_bounds__(256) k_adj_vjp(Params P, const uint8_t* __restrict__ mid, const AdjMat* __restrict__ am,
                                                 F3 y, F3 hs, F3 u, const double* __restrict__ alpha, F3 ybar, F3 hbar,
                                                 double* __restrict__ abar, double* __restrict__ hbx) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    if (!(id != 0 && am[id - 1].fm)) {
        st3(ybar, c, make_double3(0., 0., 0.));
        st3(hbar, c, make_double3(0., 0., 0.));
        hbx[c] = 0.;
        return;
    }
    const AdjMat& mt = am[id - 1];
    const double3 m = ld3(y, c), H = ld3(hs, c), w = ld3(u, c);
    const double a = alpha[c];
    const double c1 = -mt.gdt / (1. + a * a), c2 = a * c1;
    const double dc1 = c1 * (-2. * a / (1. + a * a)), dc2 = c1 + a * dc1;
    const double3 p = cross3(m, H), q = cross3(m, p);
    abar[c] += dot3(w, make_double3(dc1 * p.x + dc2 * q.x, dc1 * p.y + dc2 * q.y, dc1 * p.z + dc2 * q.z));
    const double3 um = cross3(w, m);
    const double3 umm = cross3(um, m);
    const double3 hb = make_double3(c1 * um.x + c2 * umm.x, c1 * um.y + c2 * umm.y, c1 * um.z + c2 * umm.z);
    const double3 t1 = cross3(H, w), t2 = cross3(p, w), t3 = cross3(H, um);
    double3 mb = make_double3(c1 * t1.x + c2 * (t2.x + t3.x), c1 * t1.y + c2 * (t2.y + t3.y), c1 * t1.z + c2 * (t2.z + t3.z));
    if (mt.aniso == 1) {
        const double K1 = mt.K1c, K2 = mt.K2c;
        const double x2 = m.x * m.x, y2 = m.y * m.y, z2 = m.z * m.z;
        const double jxx = -2. * (K1 * (y2 + z2) + K2 * y2 * z2);
        const double jyy = -2. * (K1 * (x2 + z2) + K2 * x2 * z2);
        const double jzz = -2. * (K1 * (x2 + y2) + K2 * x2 * y2);
        const double jxy = -4. * m.x * m.y * (K1 + K2 * z2);
        const double jxz = -4. * m.x * m.z * (K1 + K2 * y2);
        const double jyz = -4. * m.y * m.z * (K1 + K2 * x2);
        mb.x += jxx * hb.x + jxy * hb.y + jxz * hb.z;
        mb.y += jxy * hb.x + jyy * hb.y + jyz * hb.z;
        mb.z += jxz * hb.x + jyz * hb.y + jzz * hb.z;
    } else if (mt.aniso == 2) {
        mb.z += 2. * mt.K1c * hb.z;
    }
    st3(ybar, c, mb);
    st3(hbar, c, hb);
    hbx[c] = hb.x;
}

// ybar += transposed exchange of Hbar: sum_f w_cf (ex_f Hbar_f - ex_c Hbar_c);
// and ybar += Ms R where R is the demag convolution of Hbar (3 x n, the
// inverse-transform output), for ferromagnetic cells
static __global__ void __launch_bounds__(256) k_adj_field_T(Params P, const uint8_t* __restrict__ mid, const AdjMat* __restrict__ am,
                                                     const double* __restrict__ aij, int nmat, F3 hbar,
                                                     const double* __restrict__ R, F3 ybar) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    if (!(id != 0 && am[id - 1].fm)) return;
    const int nyz = P.ny * P.nz;
    const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    AdjNbr n;
    adj_neighbours(P, mid, am, aij, nmat, i, j, k, id, n);
    const double ec = am[id - 1].ex_coef, Ms = am[id - 1].Ms;
    const double3 hc = ld3(hbar, c);
    double3 s = make_double3(0., 0., 0.);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        if (n.w[f] == 0.) continue;
        const double ef = am[mid[n.nb[f]] - 1].ex_coef;
        const double3 hf = ld3(hbar, n.nb[f]);
        s.x += n.w[f] * (ef * hf.x - ec * hc.x);
        s.y += n.w[f] * (ef * hf.y - ec * hc.y);
        s.z += n.w[f] * (ef * hf.z - ec * hc.z);
    }
    double3 yb = ld3(ybar, c);
    yb.x += s.x; yb.y += s.y; yb.z += s.z;
    if (R) { yb.x += Ms * R[c]; yb.y += Ms * R[P.n + c]; yb.z += Ms * R[2 * P.n + c]; }
    st3(ybar, c, yb);
}

// Hbar (3 x n arrays) into the contiguous FFT input
static __global__ void k_adj_pack(Params P, F3 v, double* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    out[c] = v.c[0][c]; out[P.n + c] = v.c[1][c]; out[2 * P.n + c] = v.c[2][c];
}

// RK4 reverse sweep after the VJP of stage S (0-based): lamacc += ybar and the
// cotangent of the next (earlier) stage's increment
template <int S>
__global__ void k_adj_comb(Params P, F3 lam, F3 lamacc, F3 u, F3 ybar) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double yb = ybar.c[a][c], l = lam.c[a][c];
        lamacc.c[a][c] = lamacc.c[a][c] + yb;
        if (S == 3) u.c[a][c] = l / 3. + yb;
        else if (S == 2) u.c[a][c] = l / 3. + yb * 0.5;
        else if (S == 1) u.c[a][c] = l / 6. + yb * 0.5;
    }
}

// v *= f (3 x n)
static __global__ void k_scale_f3(Params P, F3 v, double f) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    v.c[0][c] *= f; v.c[1][c] *= f; v.c[2][c] *= f;
}

// lambda_x += g / NFM on ferromagnetic cells (d loss / d <m_x> of one step)
static __global__ void k_adj_inject(Params P, const uint8_t* __restrict__ mid, const AdjMat* __restrict__ am, F3 lam,
                             const double* __restrict__ g, long slot, double inv_nfm) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    if (id != 0 && am[id - 1].fm) lam.c[0][c] = lam.c[0][c] + g[slot] * inv_nfm;
}

// out[slot] += in[0] (single thread; waveform gradient of one stage)
static __global__ void k_adj_add_slot(double* out, long slot, const double* in) { out[slot] = out[slot] + in[0]; }

// out[slot] = in[0] * scale (single thread; one entry of the <m_x> trace)
static __global__ void k_adj_store_slot(double* out, long slot, const double* in, double scale) { out[slot] = in[0] * scale; }

}  // namespace gf
