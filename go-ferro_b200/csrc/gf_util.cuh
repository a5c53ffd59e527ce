// Small utility kernels: step counter, deterministic FP64 sums, health
// check, cell-centred E/H for output.
#pragma once

#include "gf_state.cuh"

namespace gf {

static __global__ void k_step_inc(unsigned long long* step) { *step = *step + 1ull; }

// Deterministic sum: thread t of T adds elements t, t+T, t+2T, ... of
// `in` (length n) in index order and writes partial[t].  Applied three times
// (n -> 8192 -> 64 -> 1) the result depends only on n, never on scheduling.
static __global__ void k_sum_stride(const double* __restrict__ in, long n, double* __restrict__ partial, long T) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    double acc = 0.;
    long i = t;
    // in order, with the loads of eight terms issued before their additions
    for (; i + 7 * T < n; i += 8 * T) {
        double v[8];
#pragma unroll
        for (int b = 0; b < 8; b++) v[b] = in[i + b * T];
#pragma unroll
        for (int b = 0; b < 8; b++) acc = acc + v[b];
    }
    for (; i < n; i += T) acc = acc + in[i];
    partial[t] = acc;
}

// The same first pass over an FP32 array, each term widened to FP64 (the
// later passes are k_sum_stride over the FP64 partials).
static __global__ void k_sum_stride_f(const float* __restrict__ in, long n, double* __restrict__ partial, long T) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    double acc = 0.;
    long i = t;
    for (; i + 7 * T < n; i += 8 * T) {
        float v[8];
#pragma unroll
        for (int b = 0; b < 8; b++) v[b] = in[i + b * T];
#pragma unroll
        for (int b = 0; b < 8; b++) acc = acc + (double)v[b];
    }
    for (; i < n; i += T) acc = acc + (double)in[i];
    partial[t] = acc;
}

// Three arrays (component y = blockIdx.y), each term the FP64 value of an
// element: a double, or in the mixed form (f32) the FP64 value x + c of an
// FP32 pair (c may be null).
struct Sum3In {
    const void* x[3];
    const float* cm[3];
    int f32;          // x holds floats (mixed form) rather than doubles
};

// Sum of a warp's 32 values by a fixed shuffle tree (lane 0 gets the total):
// the order of the additions depends on nothing but the lane numbers.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// One pass over the data: block b of component y sums the contiguous chunk
// [b*L, min((b+1)*L, n)) of array y — each thread the elements t, t+256, ...
// of the chunk in order, then the 8 warps by a fixed shuffle tree and the 8
// warp totals in warp order — into partial[y * gridDim.x + b].  With the
// grid fixed by the caller the sum depends only on n.  The loads of
// GF_SUM_BATCH terms are issued before their additions.
#ifndef GF_SUM_BATCH
#define GF_SUM_BATCH 8
#endif
constexpr int kSumThreads = 256;
static __global__ void __launch_bounds__(kSumThreads) k_sum3_block(Sum3In in, long n, double* __restrict__ partial) {
    const int y = blockIdx.y;
    const long L = (n + gridDim.x - 1) / gridDim.x;
    const long i0 = (long)blockIdx.x * L;
    const long i1 = min(i0 + L, n);
    constexpr int B = GF_SUM_BATCH;
    double acc = 0.;
    long i = i0 + threadIdx.x;
    if (in.f32) {
        const float* x = static_cast<const float*>(in.x[y]);
        const float* cm = in.cm[y];
        for (; i + (B - 1) * kSumThreads < i1; i += B * kSumThreads) {
            double v[B];
#pragma unroll
            for (int b = 0; b < B; b++) v[b] = (double)x[i + b * kSumThreads] + (cm ? (double)cm[i + b * kSumThreads] : 0.);
#pragma unroll
            for (int b = 0; b < B; b++) acc = acc + v[b];
        }
        for (; i < i1; i += kSumThreads) acc = acc + ((double)x[i] + (cm ? (double)cm[i] : 0.));
    } else {
        const double* x = static_cast<const double*>(in.x[y]);
        for (; i + (B - 1) * kSumThreads < i1; i += B * kSumThreads) {
            double v[B];
#pragma unroll
            for (int b = 0; b < B; b++) v[b] = x[i + b * kSumThreads];
#pragma unroll
            for (int b = 0; b < B; b++) acc = acc + v[b];
        }
        for (; i < i1; i += kSumThreads) acc = acc + x[i];
    }
    __shared__ double ws[kSumThreads / 32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kSumThreads / 32 ? ws[threadIdx.x] : 0.;
        v = warp_sum(v);
        if (threadIdx.x == 0) partial[y * gridDim.x + blockIdx.x] = v;
    }
}

// out[y] = sum of the nb partials of component y (blockIdx.x = y), each
// thread its partials t, t+256, ... in order, then the same fixed tree.
static __global__ void __launch_bounds__(kSumThreads) k_sum3_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    const int y = blockIdx.x;
    double acc = 0.;
    for (int i = threadIdx.x; i < nb; i += kSumThreads) acc = acc + partial[y * nb + i];
    __shared__ double ws[kSumThreads / 32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kSumThreads / 32 ? ws[threadIdx.x] : 0.;
        v = warp_sum(v);
        if (threadIdx.x == 0) out[y] = v;
    }
}

// numerators for gf_check_quotients: odd i draws a random double with
// exponent in about 2^-100..2^100; even i a value whose quotient by d lies
// within rounding noise of a midpoint between two doubles.  Counts the
// quotients where qdiv and IEEE division differ in any bit.
__device__ inline unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static __global__ void k_check_quotients(double d, double rd, unsigned long long n, unsigned long long seed,
                                  unsigned long long* bad) {
    const unsigned long long T = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long local = 0;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += T) {
        const unsigned long long z = mix64(seed ^ mix64(i));
        const int e = (int)((z >> 52) % 201ull) - 100;
        const double mant = 1. + (double)(z & ((1ull << 52) - 1)) * 0x1p-52;
        double x = ldexp(mant, e);
        if (i & 1ull) {
            if (z >> 63) x = -x;
        } else {
            // t = mant + half an ulp of mant, scaled: x = RN(d * t)
            const double t = ldexp(mant, e), half_ulp = ldexp(0x1p-53, e);
            x = __fma_rn(d, t, __dmul_rn(d, half_ulp));
        }
        const double a = qdiv(x, d, rd), b = x / d;
        if (__double_as_longlong(a) != __double_as_longlong(b)) local++;
    }
    if (local) atomicAdd(bad, local);
}

// x[0] := x[0] / d  (single thread; the mean of gf_field_mean_noalloc)
static __global__ void k_scale(double* x, double d) { x[0] = x[0] / d; }

// flag := 1 if any element of in[0..n) is not finite
static __global__ void k_check_finite(const double* __restrict__ in, long n, int* flag) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long T = (long)gridDim.x * blockDim.x;
    for (long i = t; i < n; i += T) {
        const double v = in[i];
        if (!(v - v == 0.)) { *flag = 1; return; }
    }
}

// cell-centred E (4-edge means) and H (2-face means) of the current step
// value, as update_DE_cell / update_DH_cell compute them
// (EMdynamic_solver.cpp:3780-3826)
// over the cells c0 .. c0 + count - 1
template <class R = double>
__global__ void k_em_cell(Params P, F3T<R> E, F3T<R> H, F3 Ec, F3 Hc, long c0, long count) {
    const long c = c0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c0 + count) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const long ny1 = P.ny + 1, nz1 = P.nz + 1;
    const long ex = (i * ny1 + j) * nz1 + k;
    const long ey = (i * P.ny + j) * nz1 + k;
    const long ez = (i * ny1 + j) * P.nz + k;
    Ec.c[0][c] = (E.c[0][ex] + E.c[0][ex + nz1] + E.c[0][ex + 1] + E.c[0][ex + nz1 + 1]) / R(4.);
    Ec.c[1][c] = (E.c[1][ey] + E.c[1][ey + P.ny * nz1] + E.c[1][ey + 1] + E.c[1][ey + P.ny * nz1 + 1]) / R(4.);
    Ec.c[2][c] = (E.c[2][ez] + E.c[2][ez + ny1 * P.nz] + E.c[2][ez + P.nz] + E.c[2][ez + ny1 * P.nz + P.nz]) / R(4.);
    const long hx0 = (i * P.ny + j) * P.nz + k, hx1 = ((i + 1) * P.ny + j) * P.nz + k;
    const long hy0 = (i * ny1 + j) * P.nz + k, hy1 = (i * ny1 + j + 1) * P.nz + k;
    const long hz0 = (i * P.ny + j) * nz1 + k;
    Hc.c[0][c] = (H.c[0][hx0] + H.c[0][hx1]) / R(2.);
    Hc.c[1][c] = (H.c[1][hy0] + H.c[1][hy1]) / R(2.);
    Hc.c[2][c] = (H.c[2][hz0] + H.c[2][hz0 + 1]) / R(2.);
}

// ---------------------------------------------------------------------------
// Mixed form (FP32 state with a compensation word): FP64 reductions and the
// conversions at the C ABI, which stays FP64.
// ---------------------------------------------------------------------------

// out = x + c in FP64 (c may be null)
static __global__ void k_widen(const float* __restrict__ x, const float* __restrict__ cm, long n, double* __restrict__ out) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (double)x[i] + (cm ? (double)cm[i] : 0.);
}

// x = RN_f32(in), c = RN_f32(in - x) (c may be null)
static __global__ void k_split(const double* __restrict__ in, long n, float* __restrict__ x, float* __restrict__ cm) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = in[i];
    const float h = (float)v;
    x[i] = h;
    if (cm) cm[i] = (float)(v - (double)h);
}

static __global__ void k_check_finite_f32(const float* __restrict__ in, long n, int* flag) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long T = (long)gridDim.x * blockDim.x;
    for (long i = t; i < n; i += T) {
        const float v = in[i];
        if (!(v - v == 0.f)) { *flag = 1; return; }
    }
}

}  // namespace gf
