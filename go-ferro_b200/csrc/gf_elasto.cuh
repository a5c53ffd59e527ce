// Elastostatic (static strain) solve, FP64, and the 1-D electrostatic model.
//
// Elastostatics.  The reference declares elastic_system::get_strain_static,
// get_eigenstrain_static and get_strain_static_glb (elastic_system.h:184-199)
// and calls them at set-up with elastodynamics and after every step without
// it (main.cpp:148-156, 213-215, 472-474), but its public sources do not
// define them.  What they do define fixes the method: the homogeneous
// reference stiffness C_h = (max c11, max c12, max c44) x scale_elasto
// (elastic_initialize.cpp:21-40), the cubic Green tensor G_ik(k) of C_h on
// the crystal-frame wave vector (elastic_initialize.cpp:340-389, the inverse
// of the acoustic tensor K_ik = C_h,ijkl k_j k_l), a D2Z/Z2D pair on the full
// grid, an iteration limit and a tolerance (read.cpp:64), and the outputs
// exxt0_crt (static strain) and exx0t0_crt (static eigenstrain) that the
// magnetic, ferroelectric and elastic solvers read.  This file restates that
// method from microelasticity (Khachaturyan's iteration for an elastically
// inhomogeneous body):
//
//   div C(r) (e - e0) = 0,  e = ebar + sym grad u,  periodic;
//   with C = C_h + dC:  div C_h e = div tau,  tau = C_h e0 - dC (e - e0),
//   so in k-space  u = -i G (tau k),  de_ij = (k_j n_i + k_i n_j) / 2,
//   n = G (tau k), de(k = 0) = 0, iterated from e = ebar.
//
// Everything is in the crystal frame (the materials' own cubic c11, c12,
// c44; the wave vector rotated by Tg2c), tensor (not engineering) shear
// strains.  ebar, the mean strain of the periodic box, is zero: the box is
// clamped, and vacuum layers in it let a film relax along their normal.
//
// 1-D electrostatics (if_elec_1Dmodel; get_E_static_1D, declared at
// ferroelectric_system.h:106 and called at set-up and after every p update
// without Maxwell fields, ferroelectric_solver.cpp:1897-1990, but not
// defined): the laterally uniform limit of the periodic electrostatic solve.
// Along each (i, j) column D_z is uniform and the column's mean E_z is zero
// (the k = 0 condition of the spectral solve), so
//   E_z = -(P'_z - D) / (e0 er),  D = sum_k (P'_z / er) / sum_k (1 / er),
// E_x = E_y = 0, with P'_z = P_z - P_z(t0) under if_elec_1D_compensate
// (pz_t0_glb, ferroelectric_initialize.cpp:25-27, 367-369), else P_z.
#pragma once

#include <cuComplex.h>

#include "gf_state.cuh"
#include "gf_elastic.cuh"

namespace gf {

// crystal-frame cubic constants of material id - 1 (row 0 = vacuum, zeros)
struct EsMats {
    double c[kMaxMat + 1][3];   // c11, c12, c44
};

// static eigenstrain of the current state, crystal frame (the dynamic
// eigenstrain of get_eigenstrain_dynamic without a static part and without
// flexoelectric terms), FP64 out, 6 x n contiguous
template <class R>
__global__ void __launch_bounds__(256) k_es_eigen(Params P, StageIOT<R> io, double* __restrict__ e0) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = io.mid[c];
    double out[6] = {0., 0., 0., 0., 0., 0.};
    if (id != 0) {
        Params Q = P;
        Q.flexo = 0;
        StageIOT<R> s = io;
        for (int a = 0; a < 6; a++) s.eig0_c[a] = nullptr;
        R e[6];
        eigen_crt(Q, s, c, e);
        for (int a = 0; a < 6; a++) out[a] = (double)e[a];
    }
    for (int a = 0; a < 6; a++) e0[(long)a * P.n + c] = out[a];
}

// tau = C_h e0 - dC (e - e0), 6 x n contiguous (xx, yy, zz, yz, xz, xy)
static __global__ void __launch_bounds__(256) k_es_tau(Params P, const uint8_t* __restrict__ mid, EsMats em,
                                                       double c11h, double c12h, double c44h,
                                                       const double* __restrict__ e, const double* __restrict__ e0,
                                                       double* __restrict__ tau) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = P.n;
    if (c >= n) return;
    const uint8_t id = mid[c];
    const double d11 = em.c[id][0] - c11h, d12 = em.c[id][1] - c12h, d44 = em.c[id][2] - c44h;
    double s[6], d[6];
#pragma unroll
    for (int a = 0; a < 6; a++) { s[a] = e0[a * n + c]; d[a] = e[a * n + c] - s[a]; }
    tau[0 * n + c] = (c11h * s[0] + c12h * (s[1] + s[2])) - (d11 * d[0] + d12 * (d[1] + d[2]));
    tau[1 * n + c] = (c11h * s[1] + c12h * (s[0] + s[2])) - (d11 * d[1] + d12 * (d[0] + d[2]));
    tau[2 * n + c] = (c11h * s[2] + c12h * (s[0] + s[1])) - (d11 * d[2] + d12 * (d[0] + d[1]));
#pragma unroll
    for (int a = 3; a < 6; a++) tau[a * n + c] = 2. * c44h * s[a] - 2. * d44 * d[a];
}

// de(k) = sym(k (x) G (tau k)) / n in place (the 1/n completes the
// unnormalised transform pair).  G: 6 x n21 real (11, 22, 33, 12, 13, 23),
// kq: crystal-frame wave vector, 3 x n21.  On the Nyquist planes (an even
// dimension at index n/2, where +k and -k are the same mode of a real field)
// the operator is the mean over both signs of each Nyquist component: a
// 6 x 6 matrix per point from nyq_op, indexed by nyq_idx (-1 elsewhere), so
// the result stays Hermitian and the inverse transform real
static __global__ void __launch_bounds__(256) k_es_green(long n21, double inv_n, const double* __restrict__ G,
                                                         const double* __restrict__ kq, const int* __restrict__ nyq_idx,
                                                         const double* __restrict__ nyq_op, cuDoubleComplex* __restrict__ T) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n21) return;
    const int ny = nyq_idx[q];
    if (ny >= 0) {
        const double* M = nyq_op + 36 * (long)ny;
        cuDoubleComplex t[6], o[6];
#pragma unroll
        for (int a = 0; a < 6; a++) t[a] = T[a * n21 + q];
#pragma unroll
        for (int a = 0; a < 6; a++) {
            double re = 0., im = 0.;
#pragma unroll
            for (int b = 0; b < 6; b++) { re += M[6 * a + b] * t[b].x; im += M[6 * a + b] * t[b].y; }
            o[a] = make_cuDoubleComplex(re * inv_n, im * inv_n);
        }
#pragma unroll
        for (int a = 0; a < 6; a++) T[a * n21 + q] = o[a];
        return;
    }
    const double k[3] = {kq[q], kq[n21 + q], kq[2 * n21 + q]};
    const double g11 = G[q], g22 = G[n21 + q], g33 = G[2 * n21 + q];
    const double g12 = G[3 * n21 + q], g13 = G[4 * n21 + q], g23 = G[5 * n21 + q];
    cuDoubleComplex t[6];
#pragma unroll
    for (int a = 0; a < 6; a++) t[a] = T[a * n21 + q];
    // tensor tau_ij from the Voigt-ordered components
    const int vi[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
    double fr[3], fi[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        fr[i] = 0.; fi[i] = 0.;
#pragma unroll
        for (int j = 0; j < 3; j++) { fr[i] += t[vi[i][j]].x * k[j]; fi[i] += t[vi[i][j]].y * k[j]; }
    }
    const double Gm[3][3] = {{g11, g12, g13}, {g12, g22, g23}, {g13, g23, g33}};
    double nr[3], ni[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        nr[i] = (Gm[i][0] * fr[0] + Gm[i][1] * fr[1] + Gm[i][2] * fr[2]) * inv_n;
        ni[i] = (Gm[i][0] * fi[0] + Gm[i][1] * fi[1] + Gm[i][2] * fi[2]) * inv_n;
    }
    const int pi_[6] = {0, 1, 2, 1, 0, 0}, pj[6] = {0, 1, 2, 2, 2, 1};
#pragma unroll
    for (int a = 0; a < 6; a++) {
        const int i = pi_[a], j = pj[a];
        T[a * n21 + q] = make_cuDoubleComplex(0.5 * (k[j] * nr[i] + k[i] * nr[j]), 0.5 * (k[j] * ni[i] + k[i] * ni[j]));
    }
}

// e := ebar + de (ebar = 0); per-block maxima of |e_new - e_old| and
// |e_new| for the convergence test (blockmax may be null)
static __global__ void __launch_bounds__(256) k_es_update(long n, const double* __restrict__ de, double* __restrict__ e,
                                                          double* __restrict__ blockmax) {
    double md = 0., me = 0.;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < 6; a++) {
            const double v = de[a * n + c];
            md = fmax(md, fabs(v - e[a * n + c]));
            me = fmax(me, fabs(v));
            e[a * n + c] = v;
        }
    }
    // block maxima: warp shuffles, then one value per warp through shared memory
    for (int o = 16; o > 0; o >>= 1) {
        md = fmax(md, __shfl_down_sync(0xffffffffu, md, o));
        me = fmax(me, __shfl_down_sync(0xffffffffu, me, o));
    }
    __shared__ double wd[8], we[8];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { wd[w] = md; we[w] = me; }
    __syncthreads();
    if (threadIdx.x == 0 && blockmax) {
        double a = 0., b = 0.;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) { a = fmax(a, wd[i]); b = fmax(b, we[i]); }
        blockmax[2 * blockIdx.x] = a;
        blockmax[2 * blockIdx.x + 1] = b;
    }
}

// the solver's FP64 strain and eigenstrain (6 x n) into the engine's static
// strain arrays (exxt0_crt, exx0t0_crt) of type R; vacuum cells get zeros
template <class R>
__global__ void __launch_bounds__(256) k_es_out(long n, const uint8_t* __restrict__ mid, const double* __restrict__ e,
                                                const double* __restrict__ e0, R* eps0, R* eps1, R* eps2, R* eps3,
                                                R* eps4, R* eps5, R* eig0, R* eig1, R* eig2, R* eig3, R* eig4, R* eig5) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    R* const o[6] = {eps0, eps1, eps2, eps3, eps4, eps5};
    R* const g[6] = {eig0, eig1, eig2, eig3, eig4, eig5};
    const bool solid = mid[c] != 0;
#pragma unroll
    for (int a = 0; a < 6; a++) {
        o[a][c] = solid ? (R)e[a * n + c] : R(0.);
        g[a][c] = solid ? (R)e0[a * n + c] : R(0.);
    }
}

// 1-D electrostatic field, one thread per (i, j) column (see the header)
template <class R>
__global__ void __launch_bounds__(256) k_elec_1d(Params P, const DevMatT<R>* __restrict__ mats, const uint8_t* __restrict__ mid,
                                                 const R* __restrict__ pz, const R* __restrict__ pz_t0, F3T<R> E) {
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= (long)P.nx * P.ny) return;
    const long base = col * P.nz;
    double sp = 0., sr = 0.;
    for (long k = 0; k < P.nz; k++) {
        const long c = base + k;
        const uint8_t id = mid[c];
        const bool fe = id != 0 && ((P.fe_mask >> (id - 1)) & 1u);
        const double er = id ? (double)mats[id - 1].er : 1.;
        const double p = fe ? (double)pz[c] - (pz_t0 ? (double)pz_t0[c] : 0.) : 0.;
        sp += p / er;
        sr += 1. / er;
    }
    const double D = sp / sr;
    for (long k = 0; k < P.nz; k++) {
        const long c = base + k;
        const uint8_t id = mid[c];
        const bool fe = id != 0 && ((P.fe_mask >> (id - 1)) & 1u);
        const double er = id ? (double)mats[id - 1].er : 1.;
        const double p = fe ? (double)pz[c] - (pz_t0 ? (double)pz_t0[c] : 0.) : 0.;
        E.c[0][c] = R(0.);
        E.c[1][c] = R(0.);
        E.c[2][c] = (R)(-(p - D) / (kE0 * er));
    }
}

}  // namespace gf
