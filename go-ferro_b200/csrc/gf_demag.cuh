// Magnetostatics: periodic FFT convolution of M with the demag
// tensor of a cuboid cell.
//
//   newell_cell   the nine real-space tensor tables' entries of one cell,
//                 evaluated on the host (the engine builds the tables with the
//                 host's libm, as the reference does, multithreaded): the
//                 far-field entries are small differences of large terms, so
//                 a last-bit difference in log or atan grows by orders of
//                 magnitude there.  The tables follow the reference's construction
//                 (initialize_intermediate_Hms, magnetic_initialize.cpp:
//                 1176-1402): the cell-averaged tensor of Newell, Williams and
//                 Dunlop (J. Geophys. Res. 98, 9551, 1993) written with the
//                 same auxiliary functions F2/F1/A and G2/G1/B (:1404-1557),
//                 evaluated on offsets |i| < nx/2 (the Nyquist offset is left
//                 zero), divided by 4*pi and by the cell count n.
//   k_demag_mul   k-space product H_k = -(N_k . M_k)/(dx dy dz) with the nine
//                 complex spectra (magnetostatic_solver.cpp:159-179); the
//                 mixed form's k_demag_mul_f32 uses the six real spectra of
//                 the symmetric tensor.
//   k_mag_source  M = Ms m for the forward transform, and the demag-factor
//                 and 1-D alternatives (magnetostatic_solver.cpp:114-249).
// The transforms themselves are cuFFT D2Z / Z2D (batched over the three
// components), unnormalised as in the reference.  The mixed form builds the
// tables and their spectra in FP64 (newell_cell, D2Z), stores the six real
// spectra in FP32 and runs R2C / C2R per stage.
#pragma once

#include <cuComplex.h>

#include "gf_state.cuh"

namespace gf {

// ---- Newell auxiliary functions (FP64) ----
__host__ __device__ inline double nw_f2(double x, double y, double z) {
    const double s = 1.0e-33;
    const double u = x * x, v = y * y, w = z * z;
    const double r = sqrt(u + v + w);
    const double ax = fabs(x), ay = fabs(y), az = fabs(z);
    double f = 0.;
    if (ax > s && ay > s && az > s)
        f = z * (u - v) * log(r - z) / 2. + y * (u - w) * log(r - y) / 2. - x * y * z * atan(y * z / (x * r)) + (2. * u - v - w) * r / 6.;
    else if (ax < s && ay > s && az > s)
        f = -(z * v / 2.) * log(r - z) - (y * w / 2.) * log(r - y) - r * r * r / 6.;
    else if (ax > s && ay < s && az > s)
        f = (z * u / 2.) * log(r - z) + (2. * u - w) * r / 6.;
    else if (ax > s && ay > s && az < s)
        f = (y * u / 2.) * log(r - y) + (2. * u - v) * r / 6.;
    else if (ax < s && ay < s && az > s)
        f = -az * az * az / 6.;
    else if (ax < s && ay > s && az < s)
        f = -ay * ay * ay / 6.;
    else if (ax > s && ay < s && az < s)
        f = ax * ax * ax / 3.;
    return f;
}

__host__ __device__ inline double nw_f1(double x, double y, double z, double dy) {
    const double ym = y - dy, yp = y + dy;
    return 2. * nw_f2(x, y, z) - nw_f2(x, ym, z) - nw_f2(x, yp, z);
}

__host__ __device__ inline double nw_a(double x, double y, double z, double dx, double dy, double dz) {
    const double xp = x + dx, xm = x - dx, zp = z + dz, zm = z - dz;
    return 4. * nw_f1(x, y, z, dy) - 2. * nw_f1(x, y, zp, dy) - 2. * nw_f1(x, y, zm, dy) - 2. * nw_f1(xp, y, z, dy)
           + nw_f1(xp, y, zp, dy) + nw_f1(xp, y, zm, dy) - 2. * nw_f1(xm, y, z, dy) + nw_f1(xm, y, zp, dy) + nw_f1(xm, y, zm, dy);
}

__host__ __device__ inline double nw_g2(double x, double y, double z) {
    const double s = 1.0e-33;
    const double u = x * x, v = y * y, w = z * z;
    const double r = sqrt(u + v + w);
    double g = 0.;
    if (fabs(x * y * z) > s)
        g = (y * y * y / 6. - y * w / 2.) * log(r + x) + (x / 6.) * (3. * w - u) * log(r - y) + x * y * r / 3.
            + x * y * z * log(r - z) + (v * z / 2.) * atan(x * z / (r * y)) + (z * z * z / 6.) * atan(x * y / (r * z))
            + (u * z / 2.) * atan(y * z / (r * x));
    else if (fabs(x) < s && fabs(y * z) > s)
        g = (y * y * y / 6. - y * w / 2.) * log(r);
    else if (fabs(x * z) > s && fabs(y) < s)
        g = (x * w / 2. - x * x * x / 6.) * log(r);
    else if (fabs(x * y) > s && fabs(z) < s)
        g = ((y * y * y) / 6.) * log(r + x) - (x * x * x / 6.) * log(r - y) + x * y * r / 3.;
    else if ((fabs(x) + fabs(y)) < s && fabs(z) > s)
        g = 0.;
    else if ((fabs(x) + fabs(z)) < s && fabs(y) > s)
        g = (y * y * y) / 12. * log(v);
    else if (fabs(x) > s && (fabs(y) + fabs(z)) < s)
        g = -((x * x * x) / 12.) * log(u);
    return g;
}

__host__ __device__ inline double nw_g1(double x, double y, double z, double dx, double dy, double dz) {
    const double xp = x + dx, xm = x - dx, yp = y + dy / 2., ym = y - dy / 2., zp = z + dz, zm = z - dz;
    return 4. * nw_g2(x, yp, z) - 4. * nw_g2(x, ym, z) - 2. * nw_g2(x, yp, zp) + 2. * nw_g2(x, ym, zp)
           - 2. * nw_g2(x, yp, zm) + 2. * nw_g2(x, ym, zm) - 2. * nw_g2(xm, yp, z) + 2. * nw_g2(xm, ym, z)
           + nw_g2(xm, yp, zp) - nw_g2(xm, ym, zp) + nw_g2(xm, yp, zm) - nw_g2(xm, ym, zm)
           - 2. * nw_g2(xp, yp, z) + 2. * nw_g2(xp, ym, z) + nw_g2(xp, yp, zp) - nw_g2(xp, ym, zp)
           + nw_g2(xp, yp, zm) - nw_g2(xp, ym, zm);
}

__host__ __device__ inline double nw_b(double x, double y, double z, double dx, double dy, double dz) {
    const double yp = y + dy / 2., ym = y - dy / 2.;
    return nw_g1(x, yp, z, dx, dy, dz) - nw_g1(x, ym, z, dx, dy, dz);
}

// signed offset of wrapped index a on a periodic axis of length n, or
// "none" for the entries the reference leaves zero
__host__ __device__ inline bool wrap_offset(long a, long n, long& off) {
    const long h = n / 2;
    if (a <= h - 1) { off = a; return true; }
    if (a >= n - h + 1) { off = a - n; return true; }
    return false;
}

// table t: 0 Axyz 1 Ayzx 2 Azxy 3 Bxyz 4 Byzx 5 Bzxy 6 Byxz 7 Bzyx 8 Bxzy
__host__ __device__ inline void newell_cell(const Params& P, long c, double v[9]) {
    const long nyz = (long)P.ny * P.nz;
    const long a = c / nyz, b = (c - a * nyz) / P.nz, g = c - a * nyz - b * P.nz;
    long oi, oj, ok;
    for (int t = 0; t < 9; t++) v[t] = 0.;
    const bool in = wrap_offset(a, P.nx, oi) && wrap_offset(b, P.ny, oj) && wrap_offset(g, P.nz, ok);
    if (!in) return;
    const double dx = P.dx, dy = P.dy, dz = P.dz;
    const double x = (double)oi * dx, y = (double)oj * dy, z = (double)ok * dz;
    const double fourpi = 2. * (2. * kPi);
    const double nn = (double)P.n;
    v[0] = nw_a(x, y, z, dx, dy, dz) / fourpi / nn;
    v[1] = nw_a(y, z, x, dy, dz, dx) / fourpi / nn;
    v[2] = nw_a(z, x, y, dz, dx, dy) / fourpi / nn;
    v[3] = nw_b(x, y, z, dx, dy, dz) / fourpi / nn;
    v[4] = nw_b(y, z, x, dy, dz, dx) / fourpi / nn;
    v[5] = nw_b(z, x, y, dz, dx, dy) / fourpi / nn;
    v[6] = nw_b(y, x, z, dy, dx, dz) / fourpi / nn;
    v[7] = nw_b(z, y, x, dz, dy, dx) / fourpi / nn;
    v[8] = nw_b(x, z, y, dx, dz, dy) / fourpi / nn;
}

__device__ inline cuDoubleComplex cmul(cuDoubleComplex a, cuDoubleComplex b) {
    return make_cuDoubleComplex(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ inline cuDoubleComplex cadd(cuDoubleComplex a, cuDoubleComplex b) {
    return make_cuDoubleComplex(a.x + b.x, a.y + b.y);
}

// M_k (3 x n21) and the nine complex spectra (9 x n21, the reference's
// Axyzk .. Bxzyk) -> H_k (3 x n21), in the reference's operation order
// (magnetostatic_solver.cpp:159-179).  The FP64 form keeps all nine: the
// tensor's spectra are real and N_ij = N_ji only up to the rounding of the
// tables, and the probed E of a 128x128x96 magnetoelastic run (driven by
// dm/dt of a nearly static m) moved by 3e-8 of its scale when the six real
// ones stood in for them.
static __global__ void __launch_bounds__(256) k_demag_mul(long n21, double vol_neg, const cuDoubleComplex* __restrict__ Mk,
                                                   const cuDoubleComplex* __restrict__ Nk, cuDoubleComplex* __restrict__ Hk) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n21) return;
    const cuDoubleComplex mx = Mk[q], my = Mk[n21 + q], mz = Mk[2 * n21 + q];
    const cuDoubleComplex* N = Nk;
    cuDoubleComplex hx = cadd(cadd(cmul(mx, N[0 * n21 + q]), cmul(my, N[3 * n21 + q])), cmul(mz, N[8 * n21 + q]));
    cuDoubleComplex hy = cadd(cadd(cmul(my, N[1 * n21 + q]), cmul(mz, N[4 * n21 + q])), cmul(mx, N[6 * n21 + q]));
    cuDoubleComplex hz = cadd(cadd(cmul(mz, N[2 * n21 + q]), cmul(mx, N[5 * n21 + q])), cmul(my, N[7 * n21 + q]));
    Hk[q] = make_cuDoubleComplex(hx.x / vol_neg, hx.y / vol_neg);
    Hk[n21 + q] = make_cuDoubleComplex(hy.x / vol_neg, hy.y / vol_neg);
    Hk[2 * n21 + q] = make_cuDoubleComplex(hz.x / vol_neg, hz.y / vol_neg);
}

// The mixed form's six real spectra (N_xx, N_yy, N_zz, N_xy, N_yz, N_zx)
// from the FP64 transforms of the nine tables (order Axyz Ayzx Azxy Bxyz
// Byzx Bzxy Byxz Bzyx Bxzy): the real parts of the first six.  The tensor's
// tables are real and even under r -> -r, so their spectra are real, and
// N_ij = N_ji: the other three spectra and all imaginary parts differ from
// these by the tables' rounding, far below FP32 resolution.
template <class T>
static __global__ void k_spectra_real(const cuDoubleComplex* __restrict__ in9, long n21, T* __restrict__ out6) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n21) return;
#pragma unroll
    for (int t = 0; t < 6; t++) out6[t * n21 + q] = (T)in9[t * n21 + q].x;
}

// mode 0: M into the FFT input, Ms m for ferromagnetic cells and
//         Ms1 m1 + Ms2 m2 for antiferromagnetic cells, 0 elsewhere (the
//         buffer holds the previous inverse transform, so every cell is set);
// mode 1: demag factors H = M N_i; mode 2: 1-D model Hz = -Mz
// (magnetostatic_solver.cpp:114-249)
static __global__ void k_mag_source(Params P, const DevMat* mats, const uint8_t* mid, F3 m, F3 a1, F3 a2, int mode, double* M3,
                             F3 Hs, double f0, double f1, double f2) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    const uint32_t fl = id ? mats[id - 1].flags : 0u;
    if (fl & MF_FM) {
        const double Ms = mats[id - 1].Ms;
        if (mode == 0) {
            M3[c] = Ms * m.c[0][c]; M3[P.n + c] = Ms * m.c[1][c]; M3[2 * P.n + c] = Ms * m.c[2][c];
        } else if (mode == 1) {
            Hs.c[0][c] = Ms * m.c[0][c] * f0; Hs.c[1][c] = Ms * m.c[1][c] * f1; Hs.c[2][c] = Ms * m.c[2][c] * f2;
        } else {
            Hs.c[0][c] = 0.; Hs.c[1][c] = 0.; Hs.c[2][c] = -Ms * m.c[2][c];
        }
    } else if (fl & MF_AFM) {
        const double Ms1 = mats[id - 1].Ms1, Ms2 = mats[id - 1].Ms2;
        if (mode == 0) {
            for (int a = 0; a < 3; a++) M3[a * P.n + c] = Ms1 * a1.c[a][c] + Ms2 * a2.c[a][c];
        } else if (mode == 1) {
            const double f[3] = {f0, f1, f2};
            for (int a = 0; a < 3; a++) Hs.c[a][c] = (Ms1 * a1.c[a][c] + Ms2 * a2.c[a][c]) * f[a];
        } else {
            Hs.c[0][c] = 0.; Hs.c[1][c] = 0.; Hs.c[2][c] = -Ms1 * a1.c[2][c] - Ms2 * a2.c[2][c];
        }
    } else if (mode == 0) {
        M3[c] = 0.; M3[P.n + c] = 0.; M3[2 * P.n + c] = 0.;
    }
}

// ---- mixed form: FP32 transforms; the spectra are built in FP64 ----

// k_demag_mul on the six real FP32 spectra (a third of the nine complex
// ones' bytes); inv_vol_neg = -1/(dx dy dz)
static __global__ void __launch_bounds__(256) k_demag_mul_f32(long n21, float inv_vol_neg, const cuComplex* __restrict__ Mk,
                                                       const float* __restrict__ Nr, cuComplex* __restrict__ Hk) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n21) return;
    const cuComplex mx = Mk[q], my = Mk[n21 + q], mz = Mk[2 * n21 + q];
    const float nxx = Nr[q], nyy = Nr[n21 + q], nzz = Nr[2 * n21 + q];
    const float nxy = Nr[3 * n21 + q], nyz = Nr[4 * n21 + q], nzx = Nr[5 * n21 + q];
    const float hxr = (mx.x * nxx + my.x * nxy) + mz.x * nzx, hxi = (mx.y * nxx + my.y * nxy) + mz.y * nzx;
    const float hyr = (my.x * nyy + mz.x * nyz) + mx.x * nxy, hyi = (my.y * nyy + mz.y * nyz) + mx.y * nxy;
    const float hzr = (mz.x * nzz + mx.x * nzx) + my.x * nyz, hzi = (mz.y * nzz + mx.y * nzx) + my.y * nyz;
    Hk[q] = make_cuComplex(hxr * inv_vol_neg, hxi * inv_vol_neg);
    Hk[n21 + q] = make_cuComplex(hyr * inv_vol_neg, hyi * inv_vol_neg);
    Hk[2 * n21 + q] = make_cuComplex(hzr * inv_vol_neg, hzi * inv_vol_neg);
}

// k_mag_source for the mixed form
static __global__ void k_mag_source_f32(Params P, const DevMatT<float>* mats, const uint8_t* mid, F3T<float> m,
                                        F3T<float> a1, F3T<float> a2, int mode, float* M3, F3T<float> Hs, float f0,
                                        float f1, float f2) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = mid[c];
    const uint32_t fl = id ? mats[id - 1].flags : 0u;
    if (fl & MF_FM) {
        const float Ms = mats[id - 1].Ms;
        if (mode == 0) {
            M3[c] = Ms * m.c[0][c]; M3[P.n + c] = Ms * m.c[1][c]; M3[2 * P.n + c] = Ms * m.c[2][c];
        } else if (mode == 1) {
            Hs.c[0][c] = Ms * m.c[0][c] * f0; Hs.c[1][c] = Ms * m.c[1][c] * f1; Hs.c[2][c] = Ms * m.c[2][c] * f2;
        } else {
            Hs.c[0][c] = 0.f; Hs.c[1][c] = 0.f; Hs.c[2][c] = -Ms * m.c[2][c];
        }
    } else if (fl & MF_AFM) {
        const float Ms1 = mats[id - 1].Ms1, Ms2 = mats[id - 1].Ms2;
        if (mode == 0) {
            for (int a = 0; a < 3; a++) M3[a * P.n + c] = Ms1 * a1.c[a][c] + Ms2 * a2.c[a][c];
        } else if (mode == 1) {
            const float f[3] = {f0, f1, f2};
            for (int a = 0; a < 3; a++) Hs.c[a][c] = (Ms1 * a1.c[a][c] + Ms2 * a2.c[a][c]) * f[a];
        } else {
            Hs.c[0][c] = 0.f; Hs.c[1][c] = 0.f; Hs.c[2][c] = -Ms1 * a1.c[2][c] - Ms2 * a2.c[2][c];
        }
    } else if (mode == 0) {
        M3[c] = 0.f; M3[P.n + c] = 0.f; M3[2 * P.n + c] = 0.f;
    }
}

}  // namespace gf
