// Discrete adjoint of the ferromagnetic RK4 step (FP64, and FP32 on a
// mixed-form engine).
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
#include "gf_elastic.cuh"

namespace gf {

// per-material constants of the adjoint's dynamics (R: the real type of the
// adjoint's fields, double on an FP64 engine, float on a mixed one)
template <class R>
struct AdjMatT {
    R gdt;             // gamma * dt (the material's gyro times the time step)
    R Ms, ex_coef, Aex, K1c, K2c;
    R B1c, B2c;        // magnetoelastic B1, B2 / (mu0 Ms)
    int aniso;
    uint32_t fm;
};
using AdjMat = AdjMatT<double>;

// six component arrays (strain, strain cotangent)
template <class R> struct C6T { R* c[6]; };
using C6 = C6T<double>;

// three-vector of the adjoint's real type
template <class R> struct V3 { R x, y, z; };
template <class R> __host__ __device__ inline V3<R> mk3(R a, R b, R c) { return V3<R>{a, b, c}; }
template <class R> __device__ inline V3<R> cross3(V3<R> a, V3<R> b) {
    return mk3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class R> __device__ inline R dot3(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> __device__ inline V3<R> ld3(const F3T<R>& f, int c) { return mk3<R>(f.c[0][c], f.c[1][c], f.c[2][c]); }
template <class R> __device__ inline void st3(const F3T<R>& f, int c, V3<R> v) { f.c[0][c] = v.x; f.c[1][c] = v.y; f.c[2][c] = v.z; }

// neighbour cells with periodic wrap and the exchange weight A_cf / dx_f^2
// of each face (0 on ferromagnetic surfaces and non-periodic boundaries)
template <class R>
struct AdjNbr {
    int nb[6];
    R w[6];
};
template <class R>
__device__ inline void adj_neighbours(const Params& P, const uint8_t* mid, const AdjMatT<R>* am, const R* aij, int nmat,
                                      int i, int j, int k, uint8_t id, AdjNbr<R>& n) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ib = (i == 0) ? nx - 1 : i - 1, iF = (i == nx - 1) ? 0 : i + 1;
    const int jb = (j == 0) ? ny - 1 : j - 1, jF = (j == ny - 1) ? 0 : j + 1;
    const int kb = (k == 0) ? nz - 1 : k - 1, kF = (k == nz - 1) ? 0 : k + 1;
    n.nb[0] = (ib * ny + j) * nz + k; n.nb[1] = (iF * ny + j) * nz + k;
    n.nb[2] = (i * ny + jb) * nz + k; n.nb[3] = (i * ny + jF) * nz + k;
    n.nb[4] = (i * ny + j) * nz + kb; n.nb[5] = (i * ny + j) * nz + kF;
    const bool edge[6] = {i == 0 && !P.per_x, i == nx - 1 && !P.per_x, j == 0 && !P.per_y,
                          j == ny - 1 && !P.per_y, k == 0 && !P.per_z, k == nz - 1 && !P.per_z};
    const R r2[3] = {R(P.rdx * P.rdx), R(P.rdy * P.rdy), R(P.rdz * P.rdz)};
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const uint8_t q = mid[n.nb[f]];
        const bool fmq = q != 0 && am[q - 1].fm;
        n.w[f] = (edge[f] || !fmq) ? R(0) : aij[id * (nmat + 1) + q] * r2[f / 2];
    }
}

// One RK stage of the adjoint's forward dynamics at state y with demag field
// hd: writes the effective field H (kept for the reverse sweep) and the RK4
// combination with step value x and increment sum acc (stage 3 updates x in
// place; stages 0-2 write the next stage state ynext).  In FP32 the step
// value carries a compensation word xc: stage 3 forms x + (acc + k/6) + xc
// by an error-free sum (the mixed engine's compensated RK update).
template <int S, class R>
__global__ void __launch_bounds__(256) k_adj_eval(Params P, const uint8_t* __restrict__ mid, const AdjMatT<R>* __restrict__ am,
                                                  const R* __restrict__ aij, int nmat, F3T<R> y, F3T<R> hd,
                                                  const R* __restrict__ alpha, V3<R> hext, F3T<R> hs, F3T<R> x, F3T<R> xc,
                                                  F3T<R> acc, F3T<R> ynext, C6T<R> str) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const int nyz = P.ny * P.nz;
    const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const uint8_t id = mid[c];
    V3<R> kk = mk3<R>(R(0), R(0), R(0));
    if (id != 0 && am[id - 1].fm) {
        const AdjMatT<R>& mt = am[id - 1];
        AdjNbr<R> n;
        adj_neighbours(P, mid, am, aij, nmat, i, j, k, id, n);
        const V3<R> m = ld3(y, c);
        V3<R> hex = mk3<R>(R(0), R(0), R(0));
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const V3<R> mf = ld3(y, n.nb[f]);
            hex.x += n.w[f] * (mf.x - m.x); hex.y += n.w[f] * (mf.y - m.y); hex.z += n.w[f] * (mf.z - m.z);
        }
        V3<R> H = ld3(hd, c);
        H.x += mt.ex_coef * hex.x + hext.x; H.y += mt.ex_coef * hex.y + hext.y; H.z += mt.ex_coef * hex.z + hext.z;
        if (mt.aniso == 1) {
            H.x += R(-2) * (mt.K1c * (m.y * m.y + m.z * m.z) + mt.K2c * m.y * m.y * m.z * m.z) * m.x;
            H.y += R(-2) * (mt.K1c * (m.x * m.x + m.z * m.z) + mt.K2c * m.x * m.x * m.z * m.z) * m.y;
            H.z += R(-2) * (mt.K1c * (m.x * m.x + m.y * m.y) + mt.K2c * m.x * m.x * m.y * m.y) * m.z;
        } else if (mt.aniso == 2) {
            H.z += R(2) * mt.K1c * m.z;
        }
        if (str.c[0]) {
            // magnetoelastic field of the stage strain (the engine's k_llg_fm)
            const R exx = str.c[0][c], eyy = str.c[1][c], ezz = str.c[2][c];
            const R eyz = str.c[3][c], exz = str.c[4][c], exy = str.c[5][c];
            H.x += R(-2) * (mt.B1c * exx * m.x + mt.B2c * (exy * m.y + exz * m.z));
            H.y += R(-2) * (mt.B1c * eyy * m.y + mt.B2c * (exy * m.x + eyz * m.z));
            H.z += R(-2) * (mt.B1c * ezz * m.z + mt.B2c * (exz * m.x + eyz * m.y));
        }
        st3(hs, c, H);
        const R a = alpha[c];
        const R c1 = -mt.gdt / (R(1) + a * a), c2 = a * c1;
        const V3<R> p = cross3(m, H), q = cross3(m, p);
        kk = mk3<R>(c1 * p.x + c2 * q.x, c1 * p.y + c2 * q.y, c1 * p.z + c2 * q.z);
    } else {
        st3(hs, c, mk3<R>(R(0), R(0), R(0)));
    }
    const R kv[3] = {kk.x, kk.y, kk.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R xv = x.c[a][c];
        if constexpr (is_mixed<R>::value) {
            if (S == 0) { acc.c[a][c] = kv[a] * (1.f / 6.f); ynext.c[a][c] = xv + kv[a] * 0.5f; }
            else if (S == 1) { acc.c[a][c] = acc.c[a][c] + kv[a] * (1.f / 3.f); ynext.c[a][c] = xv + kv[a] * 0.5f; }
            else if (S == 2) { acc.c[a][c] = acc.c[a][c] + kv[a] * (1.f / 3.f); ynext.c[a][c] = xv + kv[a]; }
            else {
                float sum, err;
                two_sum(xv, (acc.c[a][c] + kv[a] * (1.f / 6.f)) + xc.c[a][c], sum, err);
                x.c[a][c] = sum;
                xc.c[a][c] = err;
            }
        } else {
            if (S == 0) { acc.c[a][c] = kv[a] / 6.; ynext.c[a][c] = xv + kv[a] * 0.5; }
            else if (S == 1) { acc.c[a][c] = acc.c[a][c] + kv[a] / 3.; ynext.c[a][c] = xv + kv[a] * 0.5; }
            else if (S == 2) { acc.c[a][c] = acc.c[a][c] + kv[a] / 3.; ynext.c[a][c] = xv + kv[a]; }
            else { x.c[a][c] = xv + (acc.c[a][c] + kv[a] / 6.); }
        }
    }
}

// RK4 reverse-sweep combination of one component after the VJP of stage s
// (0-based), fused into the kernel that forms the final ybar of its group:
// lamacc := lacc0 + yb (lacc0 = lambda at stage 4, the running sum after),
// and the cotangent u of the next (earlier) stage's increment:
// u3 = lambda/3 + ybar4, u2 = lambda/3 + ybar3/2, u1 = lambda/6 + ybar2/2
template <class R>
__device__ __forceinline__ void adj_comb1(int s, R l, R lacc0, R yb, R* lamacc, R* u, int c) {
    lamacc[c] = lacc0 + yb;
    if (s == 3) u[c] = l / R(3) + yb;
    else if (s == 2) u[c] = l / R(3) + yb * R(0.5);
    else if (s == 1) u[c] = l / R(6) + yb * R(0.5);
}

// Local part of the vector-Jacobian product of stage s: the cross products,
// the anisotropy Jacobian, the damping derivative; writes ybar (local part)
// and Hbar; adds alphabar and Hbar_x (the waveform gradient's per-cell sum)
// in FP64 in both forms (they sum over many stages).  The increment's
// cotangent is us * u (u = lambda and us = 1/6 at stage 4).
template <class R>
__global__ void __launch_bounds__(256) k_adj_vjp(Params P, const uint8_t* __restrict__ mid, const AdjMatT<R>* __restrict__ am,
                                                 F3T<R> y, F3T<R> hs, F3T<R> u, R us, const R* __restrict__ alpha, F3T<R> ybar,
                                                 F3T<R> hbar, double* __restrict__ abar, double* __restrict__ hacc, C6T<R> str,
                                                 C6T<R> strbar) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    const R z = R(0);
    if (!(id != 0 && am[id - 1].fm)) {
        st3(ybar, c, mk3<R>(z, z, z));
        st3(hbar, c, mk3<R>(z, z, z));
        if (strbar.c[0])
            for (int q = 0; q < 6; q++) strbar.c[q][c] = z;
        return;
    }
    const AdjMatT<R>& mt = am[id - 1];
    const V3<R> m = ld3(y, c), H = ld3(hs, c);
    V3<R> w = ld3(u, c);
    w.x *= us; w.y *= us; w.z *= us;
    const R a = alpha[c];
    const R c1 = -mt.gdt / (R(1) + a * a), c2 = a * c1;
    const R dc1 = c1 * (R(-2) * a / (R(1) + a * a)), dc2 = c1 + a * dc1;
    const V3<R> p = cross3(m, H), q = cross3(m, p);
    abar[c] += (double)dot3(w, mk3<R>(dc1 * p.x + dc2 * q.x, dc1 * p.y + dc2 * q.y, dc1 * p.z + dc2 * q.z));
    const V3<R> um = cross3(w, m);
    const V3<R> umm = cross3(um, m);
    const V3<R> hb = mk3<R>(c1 * um.x + c2 * umm.x, c1 * um.y + c2 * umm.y, c1 * um.z + c2 * umm.z);
    const V3<R> t1 = cross3(H, w), t2 = cross3(p, w), t3 = cross3(H, um);
    V3<R> mb = mk3<R>(c1 * t1.x + c2 * (t2.x + t3.x), c1 * t1.y + c2 * (t2.y + t3.y), c1 * t1.z + c2 * (t2.z + t3.z));
    if (mt.aniso == 1) {
        const R K1 = mt.K1c, K2 = mt.K2c;
        const R x2 = m.x * m.x, y2 = m.y * m.y, z2 = m.z * m.z;
        const R jxx = R(-2) * (K1 * (y2 + z2) + K2 * y2 * z2);
        const R jyy = R(-2) * (K1 * (x2 + z2) + K2 * x2 * z2);
        const R jzz = R(-2) * (K1 * (x2 + y2) + K2 * x2 * y2);
        const R jxy = R(-4) * m.x * m.y * (K1 + K2 * z2);
        const R jxz = R(-4) * m.x * m.z * (K1 + K2 * y2);
        const R jyz = R(-4) * m.y * m.z * (K1 + K2 * x2);
        mb.x += jxx * hb.x + jxy * hb.y + jxz * hb.z;
        mb.y += jxy * hb.x + jyy * hb.y + jyz * hb.z;
        mb.z += jxz * hb.x + jyz * hb.y + jzz * hb.z;
    } else if (mt.aniso == 2) {
        mb.z += R(2) * mt.K1c * hb.z;
    }
    if (str.c[0]) {
        // magnetoelastic field H_me = -2 (B1 e_aa m_a + B2 sum_b e_ab m_b):
        // symmetric Jacobian in m, and the strain cotangent
        const R exx = str.c[0][c], eyy = str.c[1][c], ezz = str.c[2][c];
        const R eyz = str.c[3][c], exz = str.c[4][c], exy = str.c[5][c];
        const R B1 = mt.B1c, B2 = mt.B2c;
        mb.x += R(-2) * (B1 * exx * hb.x + B2 * exy * hb.y + B2 * exz * hb.z);
        mb.y += R(-2) * (B2 * exy * hb.x + B1 * eyy * hb.y + B2 * eyz * hb.z);
        mb.z += R(-2) * (B2 * exz * hb.x + B2 * eyz * hb.y + B1 * ezz * hb.z);
        strbar.c[0][c] = R(-2) * B1 * m.x * hb.x;
        strbar.c[1][c] = R(-2) * B1 * m.y * hb.y;
        strbar.c[2][c] = R(-2) * B1 * m.z * hb.z;
        strbar.c[3][c] = R(-2) * B2 * (m.z * hb.y + m.y * hb.z);
        strbar.c[4][c] = R(-2) * B2 * (m.z * hb.x + m.x * hb.z);
        strbar.c[5][c] = R(-2) * B2 * (m.y * hb.x + m.x * hb.y);
    }
    st3(ybar, c, mb);
    st3(hbar, c, hb);
    hacc[c] += (double)hb.x;
}

// ---------------------------------------------------------------------------
// Elastodynamic coupling (magnetoelastic decks).  Forward per stage s (the
// engine's own k_elastic_tile and k_elastic_rk on the adjoint's buffers):
//   f = div sigma(u_s, e0(m_s)),  e_s = cell strain of u_s (LLG field),
//   k_u = dt v_s,  k_v = dens_dt f + md v_x + sd w_s (f - fs),
// with v_x the step value, w = 1, 2, 2, 1 and fs the stage-1 force of the
// previous step at stage 1 and of this step afterwards (elastic_dynamic_
// solver.cpp:1295-1329); after stage 4 the Liao extrapolation replaces
// u(k = 0) (elastodynamics_AbsorbingBoundary.cpp:91-230).  The reverse sweep
// below transposes each of these maps.
// ---------------------------------------------------------------------------

// Cotangents of the elastic increments of stage S: us uku, us ukv = d loss /
// d k_u, d k_v (uk = lambda and us = 1/6 at stage 4).  v-stage cotangent
// ybar_v = dt uku; force cotangent fbar; lamacc_v gets md ukv (k_v reads the
// step value v_x); the stage-1 force collects -sd w ukv of the later stages
// (f0bar) and, at stage 1, the cotangent phi of the next step's fs;
// phi_new = -sd ukv (stage 1 reads fs).  ybar_v is final here, so the v
// group's RK combination (adj_comb1) follows in the same thread.
template <int S, class R>
__global__ void __launch_bounds__(256) k_adj_el_vjp(Params P, const uint8_t* __restrict__ mid, const DevMatT<R>* __restrict__ mats,
                                                   F3T<R> uku, F3T<R> ukv, R us, F3T<R> fbar, F3T<R> lam_v, F3T<R> lamacc_v,
                                                   F3T<R> u_v, F3T<R> f0bar, F3T<R> phi, F3T<R> phi_new) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    const R dt = is_mixed<R>::value ? R(P.f.dt) : R(P.dt);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R yb = dt * (uku.c[a][c] * us);
        const R g = ukv.c[a][c] * us;
        const R l = lam_v.c[a][c];
        R lacc = (S == 3) ? l : lamacc_v.c[a][c];
        R fb = R(0), pn = R(0);
        if (id != 0) {
            const DevMatT<R>& mt = mats[id - 1];
            const R w = (S == 1 || S == 2) ? R(2) : R(1);
            fb = (mt.dens_dt + mt.stiff_damp * w) * g;
            lacc += mt.mass_damp * g;
            if (S > 0) f0bar.c[a][c] += -mt.stiff_damp * w * g;
            else { fb += f0bar.c[a][c] + phi.c[a][c]; pn = -mt.stiff_damp * g; }
        }
        fbar.c[a][c] = fb;
        if (S == 0) phi_new.c[a][c] = pn;
        adj_comb1<R>(S, l, lacc, yb, lamacc_v.c[a], u_v.c[a], c);
    }
}

// Pass 1 of the transposed stress stencil, per cell x: for each of its six
// faces that is not stress-free, the face-stress cotangent
// sbar = (fbar_lower - fbar_upper) / h (the face adds +sigma/h to the force
// of the cell below it and -sigma/h to the one above), half of it to x's side
// (sigma = mean of the two sides), through the rows of C_x to x's side
// strain st (k_elastic_tile's side_rows: face normal and face shears from the
// face's own gradient, the other components from x's face-gradient means,
// engineering shears, minus e0).  Outputs per cell (27 x n, `to`):
//   T[d][a] (9): cotangent of x's gradient du_a/dx_d on both of its d-faces
//               (every mean (g_minus + g_plus)/2 or /4 enters both alike),
//               plus the LLG strain's cotangent (the cell strain is the same
//               means);
//   O[f][a] (18): cotangent of the gradient on face f (2d: -d, 2d+1: +d) from
//               x's own side of that face (normal and face shears).
// The eigenstrain cotangent -st (x2 for shears) goes through the
// magnetostriction e0_aa = 1.5 l100 (m_a^2 - 1/3), e0_ab = 1.5 l111 m_a m_b
// into ybar_m (back: the run feeds the eigenstrain back).
// With elastodynamics ybar_m is final here: the m group's RK combination
// (adj_comb1 at stage s: lam_m, lamacc_m, u_m) follows in the same thread.
template <class R>
__global__ void __launch_bounds__(256) k_adj_el_p1(Params P, const uint8_t* __restrict__ mid, const DevMatT<R>* __restrict__ mats,
                                                  F3T<R> fbar, C6T<R> strbar, F3T<R> m, F3T<R> ybar_m, int back, R* __restrict__ to,
                                                  int s, F3T<R> lam_m, F3T<R> lamacc_m, F3T<R> u_m) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long n = P.n;
    R T[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, O[6][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const uint8_t id = mid[c];
    if (id != 0) {
        const DevMatT<R>& mt = mats[id - 1];
        const int nyz = P.ny * P.nz;
        const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
        const int pos[3] = {i, j, k}, nn[3] = {P.nx, P.ny, P.nz}, per[3] = {P.per_x, P.per_y, P.per_z};
        const int stride[3] = {nyz, P.nz, 1};
        const R rh[3] = {R(P.rdx), R(P.rdy), R(P.rdz)};
        R d0b[6] = {0, 0, 0, 0, 0, 0};
        const R fx[3] = {fbar.c[0][c], fbar.c[1][c], fbar.c[2][c]};
        for (int D = 0; D < 3; D++) {
            for (int side = 0; side < 2; side++) {
                const bool edge = side == 0 ? pos[D] == 0 : pos[D] == nn[D] - 1;
                if (edge && !per[D]) continue;
                int q = pos[D] + (side == 0 ? -1 : 1);
                q = q < 0 ? q + nn[D] : (q >= nn[D] ? q - nn[D] : q);
                const int y = c + (q - pos[D]) * stride[D];
                if (mid[y] == 0) continue;
                const R fy_[3] = {fbar.c[0][y], fbar.c[1][y], fbar.c[2][y]};
                R S_[3];
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    const R lo = side == 0 ? fy_[r] : fx[r], up = side == 0 ? fx[r] : fy_[r];
                    S_[r] = R(0.5) * (lo - up) * rh[D];
                }
                R st[6];
#pragma unroll
                for (int qv = 0; qv < 6; qv++)
                    st[qv] = mt.cij[face_row(D, 0)][qv] * S_[0] + mt.cij[face_row(D, 1)][qv] * S_[1]
                             + mt.cij[face_row(D, 2)][qv] * S_[2];
                R* o = O[2 * D + side];
                if (D == 0) {
                    o[0] += st[0]; o[2] += st[4]; o[1] += st[5];
                    T[1][1] += R(0.5) * st[1]; T[2][2] += R(0.5) * st[2];
                    T[2][1] += R(0.5) * st[3]; T[1][2] += R(0.5) * st[3];
                    T[2][0] += R(0.5) * st[4]; T[1][0] += R(0.5) * st[5];
                } else if (D == 1) {
                    o[1] += st[1]; o[2] += st[3]; o[0] += st[5];
                    T[0][0] += R(0.5) * st[0]; T[2][2] += R(0.5) * st[2];
                    T[2][1] += R(0.5) * st[3];
                    T[2][0] += R(0.5) * st[4]; T[0][2] += R(0.5) * st[4];
                    T[0][1] += R(0.5) * st[5];
                } else {
                    o[2] += st[2]; o[1] += st[3]; o[0] += st[4];
                    T[0][0] += R(0.5) * st[0]; T[1][1] += R(0.5) * st[1];
                    T[1][2] += R(0.5) * st[3]; T[0][2] += R(0.5) * st[4];
                    T[1][0] += R(0.5) * st[5]; T[0][1] += R(0.5) * st[5];
                }
                d0b[0] -= st[0]; d0b[1] -= st[1]; d0b[2] -= st[2];
                d0b[3] -= R(2) * st[3]; d0b[4] -= R(2) * st[4]; d0b[5] -= R(2) * st[5];
            }
        }
        if (strbar.c[0]) {
            // cell strain of the LLG: e_aa = (gm + gp)(a, a) / 2, shears / 4
            const R e0_ = strbar.c[0][c], e1 = strbar.c[1][c], e2 = strbar.c[2][c];
            const R e3 = strbar.c[3][c], e4 = strbar.c[4][c], e5 = strbar.c[5][c];
            T[0][0] += R(0.5) * e0_; T[1][1] += R(0.5) * e1; T[2][2] += R(0.5) * e2;
            T[2][1] += R(0.25) * e3; T[1][2] += R(0.25) * e3;
            T[2][0] += R(0.25) * e4; T[0][2] += R(0.25) * e4;
            T[1][0] += R(0.25) * e5; T[0][1] += R(0.25) * e5;
        }
        if (back) {
            const R mx = m.c[0][c], my = m.c[1][c], mz = m.c[2][c];
            const R l1 = mt.l100_15, l2 = mt.l111_15;
            ybar_m.c[0][c] += R(2) * l1 * mx * d0b[0] + l2 * (mz * d0b[4] + my * d0b[5]);
            ybar_m.c[1][c] += R(2) * l1 * my * d0b[1] + l2 * (mz * d0b[3] + mx * d0b[5]);
            ybar_m.c[2][c] += R(2) * l1 * mz * d0b[2] + l2 * (my * d0b[3] + mx * d0b[4]);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R l = lam_m.c[a][c];
        adj_comb1<R>(s, l, s == 3 ? l : lamacc_m.c[a][c], ybar_m.c[a][c], lamacc_m.c[a], u_m.c[a], c);
    }
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int a = 0; a < 3; a++) to[(d * 3 + a) * n + c] = T[d][a];
#pragma unroll
    for (int f = 0; f < 6; f++)
#pragma unroll
        for (int a = 0; a < 3; a++) to[(9 + f * 3 + a) * n + c] = O[f][a];
}

// Pass 2, per cell c: cotangent of the gradient on each of its faces that is
// not stress-free (T of the two cells plus O of each side), then
// ubar_a(c) = sum_d (gbar_d(lower face) - gbar_d(upper face)) / h_d
// (g = (u(upper cell) - u(lower cell)) / h).  Written to ybar_u.
// ybar_u is final here: the u group's RK combination (adj_comb1 at stage s)
// follows in the same thread instead of a store of ybar_u.
template <class R>
__global__ void __launch_bounds__(256) k_adj_el_p2(Params P, const uint8_t* __restrict__ mid, const R* __restrict__ to,
                                                  int s, F3T<R> lam_u, F3T<R> lamacc_u, F3T<R> u_u) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long n = P.n;
    R ub[3] = {R(0), R(0), R(0)};
    const uint8_t id = mid[c];
    if (id != 0) {
        const int nyz = P.ny * P.nz;
        const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
        const int pos[3] = {i, j, k}, nn[3] = {P.nx, P.ny, P.nz}, per[3] = {P.per_x, P.per_y, P.per_z};
        const int stride[3] = {nyz, P.nz, 1};
        const R rh[3] = {R(P.rdx), R(P.rdy), R(P.rdz)};
        for (int d = 0; d < 3; d++) {
            const int qa = pos[d] == 0 ? nn[d] - 1 : pos[d] - 1, qb = pos[d] == nn[d] - 1 ? 0 : pos[d] + 1;
            const int a_ = c + (qa - pos[d]) * stride[d], b_ = c + (qb - pos[d]) * stride[d];
            const bool free_lo = (pos[d] == 0 && !per[d]) || mid[a_] == 0;
            const bool free_hi = (pos[d] == nn[d] - 1 && !per[d]) || mid[b_] == 0;
#pragma unroll
            for (int comp = 0; comp < 3; comp++) {
                const int tq = (d * 3 + comp);
                R gl = R(0), gu = R(0);
                if (!free_lo) gl = to[tq * n + a_] + to[tq * n + c] + to[(9 + (2 * d + 1) * 3 + comp) * n + a_]
                                   + to[(9 + (2 * d) * 3 + comp) * n + c];
                if (!free_hi) gu = to[tq * n + c] + to[tq * n + b_] + to[(9 + (2 * d + 1) * 3 + comp) * n + c]
                                   + to[(9 + (2 * d) * 3 + comp) * n + b_];
                ub[comp] += (gl - gu) * rh[d];
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R l = lam_u.c[a][c];
        adj_comb1<R>(s, l, s == 3 ? l : lamacc_u.c[a][c], ub[a], lamacc_u.c[a], u_u.c[a], c);
    }
}

// Liao extrapolation after the step (forward): the history slot of this
// step takes planes k = 1..4 of the step-start u, and u_new(k = 0) =
// c1 u(1) - c2 u_{-1}(2) + c3 u_{-2}(3) - w u_{-3}(4) (k_elastic_bc's form)
template <class R>
__global__ void k_adj_liao(Params P, F3T<R> ux, F3T<R> unew, F3T<R> ucmp, R* __restrict__ hist, R* __restrict__ last,
                           unsigned long long step) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long plane = (long)P.nx * P.ny;
    if (t >= plane) return;
    const long i = t / P.ny, j = t - i * P.ny;
    const double wd = P.liao_w;
    const R w = R(wd);
    const R c1 = R(4. * wd + 2. * (1. - wd)), c2 = R(6. * wd + (1. - wd)), c3 = R(4. * wd);
    R* slot = hist + (size_t)(step & 3ull) * 12 * plane;
    const R* h2 = hist + (size_t)((step + 3) & 3ull) * 12 * plane;
    const R* h3 = hist + (size_t)((step + 2) & 3ull) * 12 * plane;
    const R* h4 = hist + (size_t)((step + 1) & 3ull) * 12 * plane;
    for (int a = 0; a < 3; a++) {
        R uv[4];
        for (int p = 1; p <= 4; p++) uv[p - 1] = ux.c[a][cid(P, i, j, p)];
        const R t2 = h2[(a * 4 + 1) * plane + t], t3 = h3[(a * 4 + 2) * plane + t], t4 = h4[(a * 4 + 3) * plane + t];
        for (int p = 1; p <= 4; p++) slot[(a * 4 + (p - 1)) * plane + t] = uv[p - 1];
        const R v = c1 * uv[0] - c2 * t2 + c3 * t3 - w * t4;
        unew.c[a][cid(P, i, j, 0)] = v;
        if (ucmp.c[a]) ucmp.c[a][cid(P, i, j, 0)] = R(0);   // FP32: the value is replaced, not summed
        last[a * plane + t] = v;
    }
}

// Liao transpose at the start of a step's reverse sweep, before lambda is
// copied into the RK accumulators: the cotangent L of u_new(k = 0) is taken
// out of lambda (the RK's own value at k = 0 was overwritten) and parked for
// the step values it came from: c1 L for this step's plane 1, -c2 L, c3 L,
// -w L for planes 2, 3, 4 of the three earlier steps.  pend: 4 slots (target
// step mod 4) x 3 components x planes k = 1..4.
template <class R>
__global__ void k_adj_liao_T(Params P, F3T<R> lam, R* __restrict__ pend, unsigned long long step) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long plane = (long)P.nx * P.ny;
    if (t >= plane) return;
    const long i = t / P.ny, j = t - i * P.ny;
    const double wd = P.liao_w;
    const R w = R(wd);
    const R c1 = R(4. * wd + 2. * (1. - wd)), c2 = R(6. * wd + (1. - wd)), c3 = R(4. * wd);
    // every load before the first store (the parked values of the four
    // target steps do not alias, but the compiler cannot know it)
    auto off = [&](unsigned long long target, int a, int p) -> size_t {
        return ((size_t)((target & 3ull) * 3 + a) * 4 + (p - 1)) * plane + t;
    };
    const R coef[4] = {c1, -c2, c3, -w};
    R L[3], pv[3][4];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        L[a] = lam.c[a][cid(P, i, j, 0)];
#pragma unroll
        for (int p = 1; p <= 4; p++) pv[a][p - 1] = (step >= (unsigned long long)(p - 1)) ? pend[off(step - (p - 1), a, p)] : R(0);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        lam.c[a][cid(P, i, j, 0)] = R(0);
#pragma unroll
        for (int p = 1; p <= 4; p++)
            if (step >= (unsigned long long)(p - 1)) pend[off(step - (p - 1), a, p)] = pv[a][p - 1] + coef[p - 1] * L[a];
    }
}

// after a step's reverse sweep: the parked Liao cotangents of its step value
// (planes 1..4) join lambda, and the slot is cleared for reuse
template <class R>
__global__ void k_adj_liao_pend(Params P, F3T<R> lam, R* __restrict__ pend, unsigned long long step) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long plane = (long)P.nx * P.ny;
    if (t >= plane) return;
    const long i = t / P.ny, j = t - i * P.ny;
    R v[3][4], l[3][4];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int p = 1; p <= 4; p++) {
            v[a][p - 1] = pend[((size_t)((step & 3ull) * 3 + a) * 4 + (p - 1)) * plane + t];
            l[a][p - 1] = lam.c[a][cid(P, i, j, p)];
        }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int p = 1; p <= 4; p++) {
            lam.c[a][cid(P, i, j, p)] = l[a][p - 1] + v[a][p - 1];
            pend[((size_t)((step & 3ull) * 3 + a) * 4 + (p - 1)) * plane + t] = R(0);
        }
}

// ybar += transposed exchange of Hbar: sum_f w_cf (ex_f Hbar_f - ex_c Hbar_c);
// and ybar += Ms R where R is the demag convolution of Hbar (3 x n, the
// inverse-transform output), for ferromagnetic cells.  With comb != 0 (no
// elastodynamics) ybar is final here and the m group's RK combination
// (adj_comb1 at stage s) follows for every cell instead of a store of ybar.
template <class R>
__device__ __forceinline__ void adj_field_T_cell(const Params& P, const uint8_t* __restrict__ mid,
                                                 const AdjMatT<R>* __restrict__ am, const R* __restrict__ aij, int nmat,
                                                 F3T<R> hbar, const R* __restrict__ Rk, int c, V3<R>& yb) {
    const uint8_t id = mid[c];
    const int nyz = P.ny * P.nz;
    const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    AdjNbr<R> n;
    adj_neighbours(P, mid, am, aij, nmat, i, j, k, id, n);
    const R ec = am[id - 1].ex_coef, Ms = am[id - 1].Ms;
    const V3<R> hc = ld3(hbar, c);
    V3<R> s = mk3<R>(R(0), R(0), R(0));
#pragma unroll
    for (int f = 0; f < 6; f++) {
        if (n.w[f] == R(0)) continue;
        const R ef = am[mid[n.nb[f]] - 1].ex_coef;
        const V3<R> hf = ld3(hbar, n.nb[f]);
        s.x += n.w[f] * (ef * hf.x - ec * hc.x);
        s.y += n.w[f] * (ef * hf.y - ec * hc.y);
        s.z += n.w[f] * (ef * hf.z - ec * hc.z);
    }
    yb.x += s.x; yb.y += s.y; yb.z += s.z;
    if (Rk) { yb.x += Ms * Rk[c]; yb.y += Ms * Rk[P.n + c]; yb.z += Ms * Rk[2 * P.n + c]; }
}
template <class R>
__global__ void __launch_bounds__(256) k_adj_field_T(Params P, const uint8_t* __restrict__ mid, const AdjMatT<R>* __restrict__ am,
                                                     const R* __restrict__ aij, int nmat, F3T<R> hbar, const R* __restrict__ Rk,
                                                     F3T<R> ybar, int comb, int s, F3T<R> lam, F3T<R> lamacc, F3T<R> u) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    const bool fm = id != 0 && am[id - 1].fm;
    if (!fm && !comb) return;
    V3<R> yb = ld3(ybar, c);
    if (fm) adj_field_T_cell<R>(P, mid, am, aij, nmat, hbar, Rk, c, yb);
    if (!comb) {
        st3(ybar, c, yb);
        return;
    }
    const R ybv[3] = {yb.x, yb.y, yb.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const R l = lam.c[a][c];
        adj_comb1<R>(s, l, s == 3 ? l : lamacc.c[a][c], ybv[a], lamacc.c[a], u.c[a], c);
    }
}

// Hbar (3 x n arrays) into the contiguous FFT input
template <class R>
__global__ void k_adj_pack(Params P, F3T<R> v, R* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    out[c] = v.c[0][c]; out[P.n + c] = v.c[1][c]; out[2 * P.n + c] = v.c[2][c];
}

// lambda_x += g / NFM on ferromagnetic cells (d loss / d <m_x> of one step)
template <class R>
__global__ void k_adj_inject(Params P, const uint8_t* __restrict__ mid, const AdjMatT<R>* __restrict__ am, F3T<R> lam,
                             const double* __restrict__ g, long slot, double inv_nfm) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    if (id != 0 && am[id - 1].fm) lam.c[0][c] = lam.c[0][c] + R(g[slot] * inv_nfm);
}

// out[slot] += in[0] (single thread; waveform gradient of one stage)
static __global__ void k_adj_add_slot(double* out, long slot, const double* in) { out[slot] = out[slot] + in[0]; }

// out[slot] = in[0] * scale (single thread; one entry of the <m_x> trace)
static __global__ void k_adj_store_slot(double* out, long slot, const double* in, double scale) { out[slot] = in[0] * scale; }

}  // namespace gf
