// Electrostatic (depolarisation) field of the polarisation, FP64.
//
// The reference declares ferroelectric_system::get_E_static()
// (ferroelectric_system.h:103) and calls it at set-up and, without Maxwell
// fields, after every RK stage (main.cpp:122-131, 299-302), but its public
// sources do not define it.  What they do define fixes the method: a cuFFT
// D2Z/Z2D pair on the full grid (ferroelectric_initialize.cpp:351-352), the
// wave vectors kx, ky, kz and |k|^2 of global.cpp:276-316, a homogeneous
// reference permittivity er_homo = max_material(er) * scale_elec and the
// Green's function i * (-1 / (er_homo |k|^2)) (ferroelectric_initialize.cpp:
// 310-338), and an iteration limit and tolerance (read.cpp:56).  This file
// restates that method from electrostatics:
//
//   div(e0 er(r) E + P) = 0,  E = -grad(phi),  periodic in x, y, z.
//   With Q = P + e0 (er(r) - er_h) E:  e0 er_h div E = -div Q, so in k-space
//   E_k = -k (k . Q_k) / (e0 er_h |k|^2)  (E_0 = 0), iterated from E = 0.
//
// The fixed point is the exact solution for the discrete spectral operator;
// the map contracts when er(r) <= er_h.  Vacuum cells have er = 1, non-
// ferroelectric cells P = 0.
#pragma once

#include <cuComplex.h>

#include "gf_state.cuh"

namespace gf {

// Q = P + e0 (er - er_h) E into the contiguous FFT input (3 x n)
static __global__ void __launch_bounds__(256) k_elec_source(Params P, const DevMat* __restrict__ mats,
                                                            const uint8_t* __restrict__ mid, F3 p, F3 E, double er_h,
                                                            double* __restrict__ Q) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    const double er = id ? mats[id - 1].er : 1.;
    const bool fe = id && (mats[id - 1].flags & MF_FE);
    const double f = kE0 * (er - er_h);
#pragma unroll
    for (int a = 0; a < 3; a++) Q[a * P.n + c] = (fe ? p.c[a][c] : 0.) + f * E.c[a][c];
}

// E_k = -k (k . Q_k) / (e0 er_h |k|^2) / n  (the 1/n completes the
// unnormalised D2Z/Z2D round trip); k = 0 gives 0
static __global__ void __launch_bounds__(256) k_elec_mul(Params P, long n21, const double* __restrict__ kx,
                                                         const double* __restrict__ ky, const double* __restrict__ kz,
                                                         double inv_e0erh_n, cuDoubleComplex* __restrict__ Qk) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n21) return;
    const long nz2 = P.nz / 2 + 1;
    const long i = q / ((long)P.ny * nz2), j = (q / nz2) % P.ny, k = q % nz2;
    const double k0 = kx[i], k1 = ky[j], k2 = kz[k];
    const double kk = k0 * k0 + k1 * k1 + k2 * k2;
    const cuDoubleComplex qx = Qk[q], qy = Qk[n21 + q], qz = Qk[2 * n21 + q];
    cuDoubleComplex e0 = make_cuDoubleComplex(0., 0.), e1 = e0, e2 = e0;
    if (kk > 0.) {
        const double s = -inv_e0erh_n / kk;
        const double dr = k0 * qx.x + k1 * qy.x + k2 * qz.x, di = k0 * qx.y + k1 * qy.y + k2 * qz.y;
        e0 = make_cuDoubleComplex(s * k0 * dr, s * k0 * di);
        e1 = make_cuDoubleComplex(s * k1 * dr, s * k1 * di);
        e2 = make_cuDoubleComplex(s * k2 * dr, s * k2 * di);
    }
    Qk[q] = e0; Qk[n21 + q] = e1; Qk[2 * n21 + q] = e2;
}

// E := the inverse transform (3 x n contiguous); per-block maxima of
// |E_new - E_old| and |E_new| for the convergence test
static __global__ void __launch_bounds__(256) k_elec_update(Params P, const double* __restrict__ R, F3 E,
                                                            double* __restrict__ blockmax) {
    __shared__ double sd[256], se[256];
    double md = 0., me = 0.;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < P.n; c += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double v = R[a * P.n + c];
            md = fmax(md, fabs(v - E.c[a][c]));
            me = fmax(me, fabs(v));
            E.c[a][c] = v;
        }
    }
    sd[threadIdx.x] = md;
    se[threadIdx.x] = me;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sd[threadIdx.x] = fmax(sd[threadIdx.x], sd[threadIdx.x + s]);
            se[threadIdx.x] = fmax(se[threadIdx.x], se[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && blockmax) { blockmax[2 * blockIdx.x] = sd[0]; blockmax[2 * blockIdx.x + 1] = se[0]; }
}

}  // namespace gf
