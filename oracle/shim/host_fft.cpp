/*
 * Host mixed-radix FFT implementing the cuFFT subset declared in cufft.h.
 *
 * TEST INFRASTRUCTURE for the CPU oracle only (see cufft.h).
 *
 * Algorithm: recursive decimation-in-time Cooley-Tukey over the prime
 * factors of each length (2, 3, 5, ... with a direct DFT for any larger
 * prime factor), twiddles from a per-length table of exp(sign*2*pi*i*k/n).
 * A 3-D transform is three passes of 1-D transforms (z, then y, then x),
 * each line gathered into a contiguous buffer.  Real-to-complex runs the
 * full complex transform of the real input and keeps k_z = 0..nz/2;
 * complex-to-real rebuilds the full spectrum by Hermitian symmetry and keeps
 * the real part of the inverse transform.  Both are unnormalised, as cuFFT.
 */
#include "cufft.h"

#include <cmath>
#include <complex>
#include <map>
#include <memory>
#include <vector>

namespace {

using cd = std::complex<double>;

struct Line1D {
    int n = 0;
    std::vector<int> factors;
    std::vector<cd> tw_fwd, tw_inv;  // exp(-/+ 2 pi i k / n), k < n
    explicit Line1D(int n_) : n(n_) {
        int m = n, p = 2;
        while (m > 1) {
            if ((long)p * p > m) { factors.push_back(m); break; }
            if (m % p == 0) { factors.push_back(p); m /= p; }
            else p = (p == 2) ? 3 : p + 2;
        }
        tw_fwd.resize(n); tw_inv.resize(n);
        const double two_pi = 6.283185307179586476925286766559;
        for (int k = 0; k < n; ++k) {
            double a = two_pi * (double)k / (double)n;
            tw_fwd[k] = cd(std::cos(a), -std::sin(a));
            tw_inv[k] = cd(std::cos(a), std::sin(a));
        }
    }
    // out[0..len) = DFT of in[0], in[stride], ... ; len divides n.
    void rec(const cd* in, cd* out, int len, long stride, size_t fi,
             const std::vector<cd>& tw, std::vector<cd>& tmp) const {
        if (len == 1) { out[0] = in[0]; return; }
        int p = factors[fi];
        int m = len / p;
        for (int r = 0; r < p; ++r)
            rec(in + r * stride, out + (long)r * m, m, stride * p, fi + 1, tw, tmp);
        // combine: X[k + q m] = sum_r W_len^{r (k + q m)} Y_r[k]
        long step = n / len;  // W_len^e = tw[e * step mod n]
        cd buf[64];
        std::vector<cd> big;
        cd* y = buf;
        if (p > 64) { big.resize(p); y = big.data(); }
        for (int k = 0; k < m; ++k) {
            for (int r = 0; r < p; ++r) {
                long e = ((long)r * k * step) % n;
                y[r] = out[(long)r * m + k] * tw[e];
            }
            for (int q = 0; q < p; ++q) {
                cd acc = 0.0;
                for (int r = 0; r < p; ++r) {
                    long e = ((long)r * q * m * step) % n;
                    acc += y[r] * tw[e];
                }
                tmp[q] = acc;
            }
            for (int q = 0; q < p; ++q) out[k + (long)q * m] = tmp[q];
        }
    }
    void run(cd* data, int sign, std::vector<cd>& scratch) const {
        scratch.resize(2 * (size_t)n + 64);
        cd* out = scratch.data();
        std::vector<cd> tmp(64 > n ? 64 : n);
        rec(data, out, n, 1, 0, sign < 0 ? tw_fwd : tw_inv, tmp);
        for (int k = 0; k < n; ++k) data[k] = out[k];
    }
};

struct Plan3D {
    int nx, ny, nz;
    cufftType type;
    std::shared_ptr<Line1D> lx, ly, lz;
};

std::map<int, Plan3D> g_plans;
std::map<int, std::shared_ptr<Line1D>> g_lines;
int g_next = 1;

std::shared_ptr<Line1D> line(int n) {
    auto it = g_lines.find(n);
    if (it != g_lines.end()) return it->second;
    auto l = std::make_shared<Line1D>(n);
    g_lines[n] = l;
    return l;
}

// in-place complex 3-D transform of a nx*ny*nz array (z fastest)
void fft3(std::vector<cd>& a, const Plan3D& p, int sign) {
    const long nx = p.nx, ny = p.ny, nz = p.nz;
    std::vector<cd> buf, scratch;
    buf.resize(std::max(nx, std::max(ny, nz)));
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j) {
            cd* row = &a[(i * ny + j) * nz];
            p.lz->run(row, sign, scratch);
        }
    for (long i = 0; i < nx; ++i)
        for (long k = 0; k < nz; ++k) {
            for (long j = 0; j < ny; ++j) buf[j] = a[(i * ny + j) * nz + k];
            p.ly->run(buf.data(), sign, scratch);
            for (long j = 0; j < ny; ++j) a[(i * ny + j) * nz + k] = buf[j];
        }
    for (long j = 0; j < ny; ++j)
        for (long k = 0; k < nz; ++k) {
            for (long i = 0; i < nx; ++i) buf[i] = a[(i * ny + j) * nz + k];
            p.lx->run(buf.data(), sign, scratch);
            for (long i = 0; i < nx; ++i) a[(i * ny + j) * nz + k] = buf[i];
        }
}

}  // namespace

cufftResult cufftPlan3d(cufftHandle* plan, int nx, int ny, int nz, cufftType type) {
    if (!plan || nx < 1 || ny < 1 || nz < 1) return CUFFT_INVALID_VALUE;
    Plan3D p{nx, ny, nz, type, line(nx), line(ny), line(nz)};
    int h = g_next++;
    g_plans[h] = p;
    *plan = h;
    return CUFFT_SUCCESS;
}

cufftResult cufftDestroy(cufftHandle plan) {
    g_plans.erase(plan);
    return CUFFT_SUCCESS;
}

cufftResult cufftExecD2Z(cufftHandle plan, cufftDoubleReal* idata, cufftDoubleComplex* odata) {
    auto it = g_plans.find(plan);
    if (it == g_plans.end()) return CUFFT_INVALID_PLAN;
    const Plan3D& p = it->second;
    const long nx = p.nx, ny = p.ny, nz = p.nz, nzh = nz / 2 + 1;
    std::vector<cd> a((size_t)(nx * ny * nz));
    for (long i = 0; i < nx * ny * nz; ++i) a[i] = cd(idata[i], 0.0);
    fft3(a, p, -1);
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j)
            for (long k = 0; k < nzh; ++k) {
                const cd v = a[(i * ny + j) * nz + k];
                odata[(i * ny + j) * nzh + k].x = v.real();
                odata[(i * ny + j) * nzh + k].y = v.imag();
            }
    return CUFFT_SUCCESS;
}

cufftResult cufftExecZ2D(cufftHandle plan, cufftDoubleComplex* idata, cufftDoubleReal* odata) {
    auto it = g_plans.find(plan);
    if (it == g_plans.end()) return CUFFT_INVALID_PLAN;
    const Plan3D& p = it->second;
    const long nx = p.nx, ny = p.ny, nz = p.nz, nzh = nz / 2 + 1;
    std::vector<cd> a((size_t)(nx * ny * nz));
    for (long i = 0; i < nx; ++i)
        for (long j = 0; j < ny; ++j)
            for (long k = 0; k < nz; ++k) {
                cd v;
                if (k < nzh) {
                    const cufftDoubleComplex& c = idata[(i * ny + j) * nzh + k];
                    v = cd(c.x, c.y);
                } else {
                    long ii = (nx - i) % nx, jj = (ny - j) % ny, kk = nz - k;
                    const cufftDoubleComplex& c = idata[(ii * ny + jj) * nzh + kk];
                    v = cd(c.x, -c.y);
                }
                a[(i * ny + j) * nz + k] = v;
            }
    fft3(a, p, +1);
    for (long i = 0; i < nx * ny * nz; ++i) odata[i] = a[i].real();
    return CUFFT_SUCCESS;
}
