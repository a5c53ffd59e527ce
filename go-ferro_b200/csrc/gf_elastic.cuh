// Elastodynamics stage kernels (FP64).
//
//   k_strain      per cell: dynamic strain of the stage displacement from
//                 face-normal gradients (get_dudxyz_glb + get_Dstrain,
//                 elastic_dynamic_solver.cpp:106-227) and the dynamic
//                 eigenstrain of m and p (get_eigenstrain_dynamic, :3-104).
//   k_elastic     per cell: face stresses, stress divergence, velocity and
//                 displacement increments and their RK4 combination
//                 (get_dv_RK{1..4} :841-2800, get_du_RK* :2801-2847,
//                 update_v*/update_u* :2849-3057).
//   k_elastic_bc  per (i,j) column: z absorbing boundary (Liao 4th order or
//                 first-order Mur, elastodynamics_AbsorbingBoundary.cpp:91-230)
//                 and the displacement source plane (update_Du_Gaussian*,
//                 elastic_dynamic_solver.cpp:3059-3284), in that order.
//
// The reference materialises nine face-gradient arrays per stage; here they
// are recomputed where used from the stage displacement and the material
// ids, so only the cell strains are written.
#pragma once

#include "gf_state.cuh"

namespace gf {

struct UGrad {
    const Params& P;
    const StageIO& io;
    __device__ UGrad(const Params& p, const StageIO& s) : P(p), io(s) {}
    __device__ bool solid(long i, long j, long k) const { return io.mid[cid(P, i, j, k)] != 0; }
    // stress-free masks (elastic_initialize.cpp:245-335)
    __device__ bool free_x(long f, long j, long k) const {
        if (f == 0 || f == P.nx) return P.per_x ? !(solid(0, j, k) && solid(P.nx - 1, j, k)) : true;
        return !(solid(f - 1, j, k) && solid(f, j, k));
    }
    __device__ bool free_y(long i, long f, long k) const {
        if (f == 0 || f == P.ny) return P.per_y ? !(solid(i, 0, k) && solid(i, P.ny - 1, k)) : true;
        return !(solid(i, f - 1, k) && solid(i, f, k));
    }
    __device__ bool free_z(long i, long j, long f) const {
        if (f == 0 || f == P.nz) return P.per_z ? !(solid(i, j, 0) && solid(i, j, P.nz - 1)) : true;
        return !(solid(i, j, f - 1) && solid(i, j, f));
    }
    __device__ double u(int a, long i, long j, long k) const { return io.u_in.c[a][cid(P, i, j, k)]; }
    // face-normal gradients of component a (get_dudxyz_glb)
    __device__ double gx(int a, long f, long j, long k) const {
        if (free_x(f, j, k)) return 0.;
        if (f == 0 || f == P.nx) return (u(a, 0, j, k) - u(a, P.nx - 1, j, k)) / P.dx;
        return (u(a, f, j, k) - u(a, f - 1, j, k)) / P.dx;
    }
    __device__ double gy(int a, long i, long f, long k) const {
        if (free_y(i, f, k)) return 0.;
        if (f == 0 || f == P.ny) return (u(a, i, 0, k) - u(a, i, P.ny - 1, k)) / P.dy;
        return (u(a, i, f, k) - u(a, i, f - 1, k)) / P.dy;
    }
    __device__ double gz(int a, long i, long j, long f) const {
        if (free_z(i, j, f)) return 0.;
        if (f == 0 || f == P.nz) return (u(a, i, j, 0) - u(a, i, j, P.nz - 1)) / P.dz;
        return (u(a, i, j, f) - u(a, i, j, f - 1)) / P.dz;
    }
};

__global__ void __launch_bounds__(256) k_strain(Params P, StageIO io) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    UGrad g(P, io);

    // ---- dynamic strain (get_Dstrain) ----
    double s[3][3];
    s[0][0] = (g.gx(0, i, j, k) + g.gx(0, i + 1, j, k)) / 2.;
    s[1][1] = (g.gy(1, i, j, k) + g.gy(1, i, j + 1, k)) / 2.;
    s[2][2] = (g.gz(2, i, j, k) + g.gz(2, i, j, k + 1)) / 2.;
    s[1][2] = (g.gz(1, i, j, k) + g.gz(1, i, j, k + 1) + g.gy(2, i, j, k) + g.gy(2, i, j + 1, k)) / 4.;
    s[0][2] = (g.gz(0, i, j, k) + g.gz(0, i, j, k + 1) + g.gx(2, i, j, k) + g.gx(2, i + 1, j, k)) / 4.;
    s[0][1] = (g.gy(0, i, j, k) + g.gy(0, i, j + 1, k) + g.gx(1, i, j, k) + g.gx(1, i + 1, j, k)) / 4.;
    s[2][1] = s[1][2]; s[2][0] = s[0][2]; s[1][0] = s[0][1];
    io.eps_g[0][c] = s[0][0]; io.eps_g[1][c] = s[1][1]; io.eps_g[2][c] = s[2][2];
    io.eps_g[3][c] = s[1][2]; io.eps_g[4][c] = s[0][2]; io.eps_g[5][c] = s[0][1];
    if (P.rot) {
        double o[3][3];
        rot_tensor(P.Tg2c, s, o);
        io.eps_c[0][c] = o[0][0]; io.eps_c[1][c] = o[1][1]; io.eps_c[2][c] = o[2][2];
        io.eps_c[3][c] = o[1][2]; io.eps_c[4][c] = o[0][2]; io.eps_c[5][c] = o[0][1];
    }

    // ---- dynamic eigenstrain (get_eigenstrain_dynamic) ----
    if (!P.elasto_back) return;
    const uint8_t id = io.mid[c];
    double e[3][3] = {{0., 0., 0.}, {0., 0., 0.}, {0., 0., 0.}};
    if (id != 0) {
        const DevMat& mt = io.mats[id - 1];
        double px = 0., py = 0., pz = 0., mx = 0., my = 0., mz = 0.;
        if (P.fe) glb2crt(P, io.p_in.c[0][c], io.p_in.c[1][c], io.p_in.c[2][c], px, py, pz);
        if (P.fm) glb2crt(P, io.m_in.c[0][c], io.m_in.c[1][c], io.m_in.c[2][c], mx, my, mz);
        const double third = 1. / 3.;
        double e0[6] = {0., 0., 0., 0., 0., 0.};
        if (io.eig0_c[0]) for (int a = 0; a < 6; a++) e0[a] = io.eig0_c[a][c];
        // (the reference's two-sublattice terms are exact zeros for decks
        // without antiferromagnets, which this build rejects)
        e[0][0] = mt.l100_15 * (mx * mx - third) + mt.Q11 * (px * px) + mt.Q12 * ((py * py) + (pz * pz)) - e0[0];
        e[1][1] = mt.l100_15 * (my * my - third) + mt.Q11 * (py * py) + mt.Q12 * ((px * px) + (pz * pz)) - e0[1];
        e[2][2] = mt.l100_15 * (mz * mz - third) + mt.Q11 * (pz * pz) + mt.Q12 * ((py * py) + (px * px)) - e0[2];
        e[1][2] = mt.l111_15 * my * mz + mt.Q44 * py * pz - e0[3];
        e[0][2] = mt.l111_15 * mx * mz + mt.Q44 * px * pz - e0[4];
        e[0][1] = mt.l111_15 * my * mx + mt.Q44 * py * px - e0[5];
        e[2][1] = e[1][2]; e[2][0] = e[0][2]; e[1][0] = e[0][1];
    }
    io.eig_c[0][c] = e[0][0]; io.eig_c[1][c] = e[1][1]; io.eig_c[2][c] = e[2][2];
    io.eig_c[3][c] = e[1][2]; io.eig_c[4][c] = e[0][2]; io.eig_c[5][c] = e[0][1];
    if (P.rot) {
        double o[3][3];
        rot_tensor(P.Tc2g, e, o);
        io.eig_g[0][c] = o[0][0]; io.eig_g[1][c] = o[1][1]; io.eig_g[2][c] = o[2][2];
        io.eig_g[3][c] = o[1][2]; io.eig_g[4][c] = o[0][2]; io.eig_g[5][c] = o[0][1];
    }
}

// Stress on one face, averaged over the two cells sharing it (each with its
// own stiffness, strain and eigenstrain), in the reference's order.
__device__ inline void face_avg(const double sa[6], const double sb[6], double out[6]) {
    for (int a = 0; a < 6; a++) out[a] = (sa[a] + sb[a]) / 2.;
}

template <int S>
__global__ void __launch_bounds__(256) k_elastic(Params P, StageIO io) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    UGrad g(P, io);
    const StageDrive& dr = stage_drive(io, S);
    const uint8_t id = io.mid[c];

    auto E = [&](int a, long cc) { return io.eps_g[a][cc]; };
    auto D0 = [&](int a, long cc) { return P.elasto_back ? io.eig_g[a][cc] : 0.; };
    auto stress_of = [&](long cc, const double st[6], double out[6]) {
        strain2stress(io.mats[io.mid[cc] - 1], st, out);
    };

    double dv[3] = {0., 0., 0.};
    if (id != 0) {
        double s1x[6], s2x[6], s1y[6], s2y[6], s1z[6], s2z[6];
        double st[6], sa[6], sb[6];
        // ---------------- x faces ----------------
        for (int side = 0; side < 2; side++) {
            const long f = i + side;                 // face index
            double* out = side ? s2x : s1x;
            if (g.free_x(f, j, k)) { for (int a = 0; a < 6; a++) out[a] = 0.; continue; }
            const long io2 = side ? ((i == P.nx - 1) ? 0 : i + 1) : ((i == 0) ? P.nx - 1 : i - 1);
            const double gxx = g.gx(0, f, j, k), gxz = g.gx(2, f, j, k), gxy = g.gx(1, f, j, k);
            for (int which = 0; which < 2; which++) {
                const long ii = which ? io2 : i;
                const long cc = cid(P, ii, j, k);
                st[0] = gxx - D0(0, cc);
                st[1] = E(1, cc) - D0(1, cc);
                st[2] = E(2, cc) - D0(2, cc);
                st[3] = (E(3, cc) - D0(3, cc)) * 2.;
                st[4] = ((g.gz(0, ii, j, k) + g.gz(0, ii, j, k + 1) + gxz * 2.) / 4. - D0(4, cc)) * 2.;
                st[5] = ((g.gy(0, ii, j, k) + g.gy(0, ii, j + 1, k) + gxy * 2.) / 4. - D0(5, cc)) * 2.;
                stress_of(cc, st, which ? sb : sa);
            }
            face_avg(sa, sb, out);
        }
        // ---------------- y faces ----------------
        for (int side = 0; side < 2; side++) {
            const long f = j + side;
            double* out = side ? s2y : s1y;
            if (g.free_y(i, f, k)) { for (int a = 0; a < 6; a++) out[a] = 0.; continue; }
            const long jo = side ? ((j == P.ny - 1) ? 0 : j + 1) : ((j == 0) ? P.ny - 1 : j - 1);
            const double gyy = g.gy(1, i, f, k), gyz = g.gy(2, i, f, k), gyx = g.gy(0, i, f, k);
            for (int which = 0; which < 2; which++) {
                const long jj = which ? jo : j;
                const long cc = cid(P, i, jj, k);
                st[0] = E(0, cc) - D0(0, cc);
                st[1] = gyy - D0(1, cc);
                st[2] = E(2, cc) - D0(2, cc);
                st[3] = ((g.gz(1, i, jj, k) + g.gz(1, i, jj, k + 1) + gyz * 2.) / 4. - D0(3, cc)) * 2.;
                st[4] = (E(4, cc) - D0(4, cc)) * 2.;
                st[5] = ((gyx * 2. + g.gx(1, i, jj, k) + g.gx(1, i + 1, jj, k)) / 4. - D0(5, cc)) * 2.;
                stress_of(cc, st, which ? sb : sa);
            }
            face_avg(sa, sb, out);
        }
        // ---------------- z faces ----------------
        for (int side = 0; side < 2; side++) {
            const long f = k + side;
            double* out = side ? s2z : s1z;
            if (g.free_z(i, j, f)) {
                for (int a = 0; a < 6; a++) out[a] = 0.;
                if (side == 1 && P.strain_pulse && P.strain_type == 3 && k == (long)P.source_z)
                    out[4 - P.strain_comp] = dr.traction;   // x -> [4], y -> [3], z -> [2]
                continue;
            }
            // +z neighbour: the reference wraps when k == ny-1 (sic), see
            // elastic_dynamic_solver.cpp:1247
            // (k == nz-1 != ny-1 with a non-free top face reads out of the
            // column in the reference; such decks are rejected at creation)
            long ko = side ? ((k == P.ny - 1) ? 0 : k + 1) : ((k == 0) ? P.nz - 1 : k - 1);
            if (ko >= P.nz) ko = 0;
            const double gzz = g.gz(2, i, j, f), gzy = g.gz(1, i, j, f), gzx = g.gz(0, i, j, f);
            for (int which = 0; which < 2; which++) {
                const long kk = which ? ko : k;
                const long cc = cid(P, i, j, kk);
                st[0] = E(0, cc) - D0(0, cc);
                st[1] = E(1, cc) - D0(1, cc);
                st[2] = gzz - D0(2, cc);
                st[3] = ((gzy * 2. + g.gy(2, i, j, kk) + g.gy(2, i, j + 1, kk)) / 4. - D0(3, cc)) * 2.;
                st[4] = ((gzx * 2. + g.gx(2, i, j, kk) + g.gx(2, i + 1, j, kk)) / 4. - D0(4, cc)) * 2.;
                st[5] = (E(5, cc) - D0(5, cc)) * 2.;
                stress_of(cc, st, which ? sb : sa);
            }
            face_avg(sa, sb, out);
        }

        const DevMat& mt = io.mats[id - 1];
        double f3[3];
        f3[0] = (s2x[0] - s1x[0]) / P.dx + (s2y[5] - s1y[5]) / P.dy + (s2z[4] - s1z[4]) / P.dz;
        f3[1] = (s2x[5] - s1x[5]) / P.dx + (s2y[1] - s1y[1]) / P.dy + (s2z[3] - s1z[3]) / P.dz;
        f3[2] = (s2x[4] - s1x[4]) / P.dx + (s2y[3] - s1y[3]) / P.dy + (s2z[2] - s1z[2]) / P.dz;
        for (int a = 0; a < 3; a++) {
            const double fs = io.force_store.c[a][c];
            if (S == 1 || S == 2)
                dv[a] = f3[a] * mt.dens_dt + mt.mass_damp * io.v_x.c[a][c] + mt.stiff_damp * (f3[a] - fs) * 2.;
            else
                dv[a] = f3[a] * mt.dens_dt + mt.mass_damp * io.v_x.c[a][c] + mt.stiff_damp * (f3[a] - fs);
            io.force.c[a][c] = f3[a];
            if (S == 0) io.force_store.c[a][c] = f3[a];
        }
    }

    // ---- RK4 combination for v and u (du = v_stage * dt) ----
    for (int a = 0; a < 3; a++) {
        const double du = io.v_in.c[a][c] * P.dt;
        const double vx = io.v_x.c[a][c], ux = io.u_x.c[a][c];
        if (S == 0) {
            io.v_out.c[a][c] = vx + dv[a] * 0.5; io.v_acc.c[a][c] = vx + dv[a] / 6.;
            io.u_out.c[a][c] = ux + du * 0.5;    io.u_acc.c[a][c] = ux + du / 6.;
        } else if (S == 1) {
            io.v_out.c[a][c] = vx + dv[a] * 0.5; io.v_acc.c[a][c] = io.v_acc.c[a][c] + dv[a] / 3.;
            io.u_out.c[a][c] = ux + du * 0.5;    io.u_acc.c[a][c] = io.u_acc.c[a][c] + du / 3.;
        } else if (S == 2) {
            io.v_out.c[a][c] = vx + dv[a];       io.v_acc.c[a][c] = io.v_acc.c[a][c] + dv[a] / 3.;
            io.u_out.c[a][c] = ux + du;          io.u_acc.c[a][c] = io.u_acc.c[a][c] + du / 3.;
        } else {
            io.v_acc.c[a][c] = io.v_acc.c[a][c] + dv[a] / 6.;
            io.u_acc.c[a][c] = io.u_acc.c[a][c] + du / 6.;
        }
    }
}

// Boundary planes of u after the stage update, one thread per (i,j).
// For stages 0..2 `tgt` is the stage output (F_glb_store); for the last
// stage it is the new step value and `old` the step-start value (the
// reference's history copy Du?_glb_t1).
template <int S>
__global__ void k_elastic_bc(Params P, StageIO io) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)P.nx * P.ny) return;
    const long i = t / P.ny, j = t - i * P.ny;
    const long nz = P.nz;
    const long plane = (long)P.nx * P.ny;
    const StageDrive& dr = stage_drive(io, S);
    const unsigned long long step = *io.step;      // 0-based step being finished

    if (!P.abc_1D) {
        // Liao 4th-order extrapolation on k = 0.  History slot h holds planes
        // k=1..4 of u at the start of step h (mod 4).
        const double w = P.liao_w;
        const double c1 = 4. * w + 2. * (1. - w), c2 = 6. * w + (1. - w), c3 = 4. * w;
        if (S < 3) {
            // stages 1-3 rewrite u(k=0) with the value of the last full update
            for (int a = 0; a < 3; a++)
                io.u_x.c[a][cid(P, i, j, 0)] = io.liao_last[a * plane + t];
        } else {
            // shift history: slot (step mod 4) <- planes 1..4 of the step-start u
            double* slot = io.liao_hist + (size_t)(step & 3ull) * 12 * plane;
            for (int a = 0; a < 3; a++)
                for (int p = 1; p <= 4; p++) slot[(a * 4 + (p - 1)) * plane + t] = io.u_x.c[a][cid(P, i, j, p)];
            const double* h1 = io.liao_hist + (size_t)((step + 0) & 3ull) * 12 * plane;   // t1 = u(step)
            const double* h2 = io.liao_hist + (size_t)((step + 3) & 3ull) * 12 * plane;   // t2 = u(step-1)
            const double* h3 = io.liao_hist + (size_t)((step + 2) & 3ull) * 12 * plane;   // t3 = u(step-2)
            const double* h4 = io.liao_hist + (size_t)((step + 1) & 3ull) * 12 * plane;   // t4 = u(step-3)
            for (int a = 0; a < 3; a++) {
                const double v = c1 * h1[(a * 4 + 0) * plane + t] - c2 * h2[(a * 4 + 1) * plane + t]
                                 + c3 * h3[(a * 4 + 2) * plane + t] - w * h4[(a * 4 + 3) * plane + t];
                io.u_acc.c[a][cid(P, i, j, 0)] = v;
                io.liao_last[a * plane + t] = v;
            }
        }
    } else {
        // first-order Mur on k = 0 (unless only the top is absorbing) and k = nz-1
        const double* cf = (S == 0 || S == 1) ? P.mur_el_half : P.mur_el_full;
        const double cl1 = cf[0], ct1 = cf[1], cll = cf[2], ctl = cf[3];
        const long b0 = cid(P, i, j, 0), b1 = cid(P, i, j, 1), t0 = cid(P, i, j, nz - 1), t1 = cid(P, i, j, nz - 2);
        for (int a = 0; a < 3; a++) {
            const double c1st = (a == 2) ? cl1 : ct1, clast = (a == 2) ? cll : ctl;
            if (S < 3) {
                double* so = io.u_out.c[a];
                const double* x = io.u_x.c[a];
                if (!P.abc_elast_onlytop) so[b0] = x[b1] + c1st * (x[b0] - so[b1]);
                so[t0] = x[t1] + clast * (x[t0] - so[t1]);
            } else {
                double* nw = io.u_acc.c[a];
                const double* old = io.u_x.c[a];
                if (!P.abc_elast_onlytop) nw[b0] = old[b1] + c1st * (old[b0] - nw[b1]);
                nw[t0] = old[t1] + clast * (old[t0] - nw[t1]);
            }
        }
    }

    // displacement source on plane source_z (types 1 and 2)
    if (P.strain_pulse && dr.usrc_on && io.mid[cid(P, i, j, P.source_z)] != 0) {
        double* tgt = (S < 3) ? io.u_out.c[P.strain_comp] : io.u_acc.c[P.strain_comp];
        tgt[cid(P, i, j, P.source_z)] = dr.usrc;
    }
}

}  // namespace gf
