// Elastodynamics stage kernels (FP64).
//
//   k_face_grad   per cell: the face-normal displacement gradients on the
//                 cell's -x, -y and -z faces, 3 components each, 0 on
//                 stress-free faces (get_dudxyz_glb, elastic_dynamic_solver.cpp:
//                 106-187).  Each gradient is computed once per stage.
//   k_elastic     per cell: cell strains (get_Dstrain, :189-227) and dynamic
//                 eigenstrains of m and p (get_eigenstrain_dynamic, :3-104) of
//                 the cell and its six face neighbours, the six face stresses,
//                 stress divergence, velocity and displacement increments and
//                 their RK4 combination (get_dv_RK{1..4} :841-2800,
//                 get_du_RK* :2801-2847, update_v*/update_u* :2849-3057).
//   k_elastic_bc  per (i,j) column: z absorbing boundary (Liao 4th order or
//                 first-order Mur, elastodynamics_AbsorbingBoundary.cpp:91-230)
//                 and the displacement source plane (update_Du_Gaussian*,
//                 elastic_dynamic_solver.cpp:3059-3284), in that order.
//
// Face f of an axis with n cells is stored at cell index f for f < n; face n
// is read from index 0, which holds the same value (periodic axis) or the
// same zero (non-periodic axis: both end faces are stress-free).  Strains and
// eigenstrains are recomputed where used instead of being stored.
#pragma once

#include "gf_state.cuh"

namespace gf {

__device__ inline bool solid_at(const Params& P, const uint8_t* mid, long i, long j, long k) {
    return mid[cid(P, i, j, k)] != 0;
}
// stress-free masks (elastic_initialize.cpp:245-335)
__device__ inline bool free_x(const Params& P, const uint8_t* mid, long f, long j, long k) {
    if (f == 0 || f == P.nx) return P.per_x ? !(solid_at(P, mid, 0, j, k) && solid_at(P, mid, P.nx - 1, j, k)) : true;
    return !(solid_at(P, mid, f - 1, j, k) && solid_at(P, mid, f, j, k));
}
__device__ inline bool free_y(const Params& P, const uint8_t* mid, long i, long f, long k) {
    if (f == 0 || f == P.ny) return P.per_y ? !(solid_at(P, mid, i, 0, k) && solid_at(P, mid, i, P.ny - 1, k)) : true;
    return !(solid_at(P, mid, i, f - 1, k) && solid_at(P, mid, i, f, k));
}
__device__ inline bool free_z(const Params& P, const uint8_t* mid, long i, long j, long f) {
    if (f == 0 || f == P.nz) return P.per_z ? !(solid_at(P, mid, i, j, 0) && solid_at(P, mid, i, j, P.nz - 1)) : true;
    return !(solid_at(P, mid, i, j, f - 1) && solid_at(P, mid, i, j, f));
}

__global__ void __launch_bounds__(256) k_face_grad(Params P, StageIO io) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const bool fx = free_x(P, io.mid, i, j, k), fy = free_y(P, io.mid, i, j, k), fz = free_z(P, io.mid, i, j, k);
    const long cx = cid(P, i == 0 ? P.nx - 1 : i - 1, j, k);
    const long cy = cid(P, i, j == 0 ? P.ny - 1 : j - 1, k);
    const long cz = cid(P, i, j, k == 0 ? P.nz - 1 : k - 1);
    for (int a = 0; a < 3; a++) {
        const double* u = io.u_in.c[a];
        const double uc = u[c];
        io.fg[a][c] = fx ? 0. : (uc - u[cx]) / P.dx;
        io.fg[3 + a][c] = fy ? 0. : (uc - u[cy]) / P.dy;
        io.fg[6 + a][c] = fz ? 0. : (uc - u[cz]) / P.dz;
    }
}

// read access to the stored face gradients; f may equal n
struct GradView {
    const Params& P;
    const StageIO& io;
    __device__ GradView(const Params& p, const StageIO& s) : P(p), io(s) {}
    __device__ double gx(int a, long f, long j, long k) const { return io.fg[a][cid(P, f == P.nx ? 0 : f, j, k)]; }
    __device__ double gy(int a, long i, long f, long k) const { return io.fg[3 + a][cid(P, i, f == P.ny ? 0 : f, k)]; }
    __device__ double gz(int a, long i, long j, long f) const { return io.fg[6 + a][cid(P, i, j, f == P.nz ? 0 : f)]; }
    // cell strain components in the global frame (get_Dstrain)
    __device__ double exx(long i, long j, long k) const { return (gx(0, i, j, k) + gx(0, i + 1, j, k)) / 2.; }
    __device__ double eyy(long i, long j, long k) const { return (gy(1, i, j, k) + gy(1, i, j + 1, k)) / 2.; }
    __device__ double ezz(long i, long j, long k) const { return (gz(2, i, j, k) + gz(2, i, j, k + 1)) / 2.; }
    __device__ double eyz(long i, long j, long k) const {
        return (gz(1, i, j, k) + gz(1, i, j, k + 1) + gy(2, i, j, k) + gy(2, i, j + 1, k)) / 4.;
    }
    __device__ double exz(long i, long j, long k) const {
        return (gz(0, i, j, k) + gz(0, i, j, k + 1) + gx(2, i, j, k) + gx(2, i + 1, j, k)) / 4.;
    }
    __device__ double exy(long i, long j, long k) const {
        return (gy(0, i, j, k) + gy(0, i, j + 1, k) + gx(1, i, j, k) + gx(1, i + 1, j, k)) / 4.;
    }
    __device__ void strain_glb(long i, long j, long k, double e[6]) const {
        e[0] = exx(i, j, k); e[1] = eyy(i, j, k); e[2] = ezz(i, j, k);
        e[3] = eyz(i, j, k); e[4] = exz(i, j, k); e[5] = exy(i, j, k);
    }
};

// cell strain in the crystal frame (Dexx_crt ..., get_Dstrain)
__device__ inline void strain_crt(const Params& P, const GradView& g, long i, long j, long k, double e[6]) {
    g.strain_glb(i, j, k, e);
    if (P.rot) {
        double s[3][3] = {{e[0], e[5], e[4]}, {e[5], e[1], e[3]}, {e[4], e[3], e[2]}}, o[3][3];
        rot_tensor(P.Tg2c, s, o);
        e[0] = o[0][0]; e[1] = o[1][1]; e[2] = o[2][2]; e[3] = o[1][2]; e[4] = o[0][2]; e[5] = o[0][1];
    }
}

// dynamic eigenstrain of cell c in the crystal frame (Dexx0_crt ...,
// get_eigenstrain_dynamic); the reference's two-sublattice terms are exact
// zeros for decks without antiferromagnets, which this build rejects
__device__ inline void eigen_crt(const Params& P, const StageIO& io, long c, double e[6]) {
    const uint8_t id = io.mid[c];
    for (int a = 0; a < 6; a++) e[a] = 0.;
    if (id == 0) return;
    const DevMat& mt = io.mats[id - 1];
    double px = 0., py = 0., pz = 0., mx = 0., my = 0., mz = 0.;
    if (P.fe) glb2crt(P, io.p_in.c[0][c], io.p_in.c[1][c], io.p_in.c[2][c], px, py, pz);
    if (P.fm) glb2crt(P, io.m_in.c[0][c], io.m_in.c[1][c], io.m_in.c[2][c], mx, my, mz);
    const double third = 1. / 3.;
    double e0[6] = {0., 0., 0., 0., 0., 0.};
    if (io.eig0_c[0]) for (int a = 0; a < 6; a++) e0[a] = io.eig0_c[a][c];
    e[0] = mt.l100_15 * (mx * mx - third) + mt.Q11 * (px * px) + mt.Q12 * ((py * py) + (pz * pz)) - e0[0];
    e[1] = mt.l100_15 * (my * my - third) + mt.Q11 * (py * py) + mt.Q12 * ((px * px) + (pz * pz)) - e0[1];
    e[2] = mt.l100_15 * (mz * mz - third) + mt.Q11 * (pz * pz) + mt.Q12 * ((py * py) + (px * px)) - e0[2];
    e[3] = mt.l111_15 * my * mz + mt.Q44 * py * pz - e0[3];
    e[4] = mt.l111_15 * mx * mz + mt.Q44 * px * pz - e0[4];
    e[5] = mt.l111_15 * my * mx + mt.Q44 * py * px - e0[5];
}

// eigenstrain in the global frame (Dexx0_glb ...)
__device__ inline void eigen_glb(const Params& P, const StageIO& io, long c, double e[6]) {
    eigen_crt(P, io, c, e);
    if (P.rot) {
        double s[3][3] = {{e[0], e[5], e[4]}, {e[5], e[1], e[3]}, {e[4], e[3], e[2]}}, o[3][3];
        rot_tensor(P.Tc2g, s, o);
        e[0] = o[0][0]; e[1] = o[1][1]; e[2] = o[2][2]; e[3] = o[1][2]; e[4] = o[0][2]; e[5] = o[0][1];
    }
}

// Rows of the Voigt stress that the divergence uses from a face normal to
// direction d: x-face -> xx, xy, xz; y-face -> xy, yy, yz; z-face -> xz, yz, zz
__constant__ const int kFaceRows[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};

// rows r[0..2] of C * e with the accumulation order of strain2stress_glb
// (mathlib.cpp:127-135); zero entries of the cubic pattern are skipped,
// which leaves every partial sum unchanged
__device__ inline double stress_row(const DevMat& m, const double e[6], int r) {
    if (m.cubic_c) {
        if (r < 3) return m.cij[r][0] * e[0] + m.cij[r][1] * e[1] + m.cij[r][2] * e[2];
        return m.cij[r][r] * e[r];
    }
    double acc = 0.;
    for (int q = 0; q < 6; q++) acc = acc + m.cij[r][q] * e[q];
    return acc;
}

// Face-normal component d, side 0 (-face) or 1 (+face) of cell (i,j,k):
// the three stress rows averaged over the two cells sharing the face
// (get_dv_RK*, elastic_dynamic_solver.cpp:876-1289), 0 on stress-free faces
// except the surface traction source.
template <int S, int D>
__device__ inline void face_stress(const Params& P, const StageIO& io, const GradView& g, long i, long j, long k,
                                   int side, const double d0c[6], double out[3]) {
    const bool back = P.elasto_back;
    long f, ii = i, jj = j, kk = k;
    bool fr;
    if (D == 0) { f = i + side; fr = free_x(P, io.mid, f, j, k); }
    else if (D == 1) { f = j + side; fr = free_y(P, io.mid, i, f, k); }
    else { f = k + side; fr = free_z(P, io.mid, i, j, f); }
    if (fr) {
        out[0] = out[1] = out[2] = 0.;
        if (D == 2 && side == 1 && P.strain_pulse && P.strain_type == 3 && k == (long)P.source_z) {
            const double tr = stage_drive(io, S).traction;   // x -> xz, y -> yz, z -> zz
            if (P.strain_comp == 0) out[0] = tr; else if (P.strain_comp == 1) out[1] = tr; else out[2] = tr;
        }
        return;
    }
    // neighbour across the face (the +z neighbour wraps when k == ny-1, sic:
    // elastic_dynamic_solver.cpp:1247; k == nz-1 != ny-1 with a non-free top
    // face reads out of the column in the reference and is rejected at creation)
    if (D == 0) ii = side ? ((i == P.nx - 1) ? 0 : i + 1) : ((i == 0) ? P.nx - 1 : i - 1);
    else if (D == 1) jj = side ? ((j == P.ny - 1) ? 0 : j + 1) : ((j == 0) ? P.ny - 1 : j - 1);
    else { kk = side ? ((k == P.ny - 1) ? 0 : k + 1) : ((k == 0) ? P.nz - 1 : k - 1); if (kk >= P.nz) kk = 0; }
    double ga, gb, gc;   // face gradients: normal comp, and the two shear comps used below
    if (D == 0) { ga = g.gx(0, f, j, k); gb = g.gx(2, f, j, k); gc = g.gx(1, f, j, k); }
    else if (D == 1) { ga = g.gy(1, i, f, k); gb = g.gy(2, i, f, k); gc = g.gy(0, i, f, k); }
    else { ga = g.gz(2, i, j, f); gb = g.gz(1, i, j, f); gc = g.gz(0, i, j, f); }
    double sa[3], sb[3];
    for (int which = 0; which < 2; which++) {
        const long ci = which ? ii : i, cj = which ? jj : j, ck = which ? kk : k;
        const long cc = cid(P, ci, cj, ck);
        double d0[6];
        if (which == 0) { for (int a = 0; a < 6; a++) d0[a] = d0c[a]; }
        else if (back) eigen_glb(P, io, cc, d0);
        else { for (int a = 0; a < 6; a++) d0[a] = 0.; }
        double st[6];
        if (D == 0) {
            st[0] = ga - d0[0];
            st[1] = g.eyy(ci, cj, ck) - d0[1];
            st[2] = g.ezz(ci, cj, ck) - d0[2];
            st[3] = (g.eyz(ci, cj, ck) - d0[3]) * 2.;
            st[4] = ((g.gz(0, ci, cj, ck) + g.gz(0, ci, cj, ck + 1) + gb * 2.) / 4. - d0[4]) * 2.;
            st[5] = ((g.gy(0, ci, cj, ck) + g.gy(0, ci, cj + 1, ck) + gc * 2.) / 4. - d0[5]) * 2.;
        } else if (D == 1) {
            st[0] = g.exx(ci, cj, ck) - d0[0];
            st[1] = ga - d0[1];
            st[2] = g.ezz(ci, cj, ck) - d0[2];
            st[3] = ((g.gz(1, ci, cj, ck) + g.gz(1, ci, cj, ck + 1) + gb * 2.) / 4. - d0[3]) * 2.;
            st[4] = (g.exz(ci, cj, ck) - d0[4]) * 2.;
            st[5] = ((gc * 2. + g.gx(1, ci, cj, ck) + g.gx(1, ci + 1, cj, ck)) / 4. - d0[5]) * 2.;
        } else {
            st[0] = g.exx(ci, cj, ck) - d0[0];
            st[1] = g.eyy(ci, cj, ck) - d0[1];
            st[2] = ga - d0[2];
            st[3] = ((gb * 2. + g.gy(2, ci, cj, ck) + g.gy(2, ci, cj + 1, ck)) / 4. - d0[3]) * 2.;
            st[4] = ((gc * 2. + g.gx(2, ci, cj, ck) + g.gx(2, ci + 1, cj, ck)) / 4. - d0[4]) * 2.;
            st[5] = (g.exy(ci, cj, ck) - d0[5]) * 2.;
        }
        const DevMat& m = io.mats[io.mid[cc] - 1];
        if (which == 0) { for (int r = 0; r < 3; r++) sa[r] = stress_row(m, st, kFaceRows[D][r]); }
        else { for (int r = 0; r < 3; r++) sb[r] = stress_row(m, st, kFaceRows[D][r]); }
    }
    for (int r = 0; r < 3; r++) out[r] = (sa[r] + sb[r]) / 2.;
}

// divergence term of direction D: (sigma(+face) - sigma(-face)) / h for the
// three rows of kFaceRows[D], ordered as force x, y, z components
template <int S, int D>
__device__ inline void div_term(const Params& P, const StageIO& io, const GradView& g, long i, long j, long k,
                                const double d0c[6], double t[3]) {
    double s1[3], s2[3];
    face_stress<S, D>(P, io, g, i, j, k, 0, d0c, s1);
    face_stress<S, D>(P, io, g, i, j, k, 1, d0c, s2);
    const double h = (D == 0) ? P.dx : (D == 1 ? P.dy : P.dz);
    // kFaceRows[D][r] is the row feeding force component r
    for (int r = 0; r < 3; r++) t[r] = (s2[r] - s1[r]) / h;
}

template <int S>
__global__ void __launch_bounds__(256, 2) k_elastic(Params P, StageIO io) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const GradView g(P, io);
    const uint8_t id = io.mid[c];

    double dv[3] = {0., 0., 0.};
    if (id != 0) {
        double d0c[6];
        if (P.elasto_back) eigen_glb(P, io, c, d0c); else for (int a = 0; a < 6; a++) d0c[a] = 0.;
        double tx[3], ty[3], tz[3];
        div_term<S, 0>(P, io, g, i, j, k, d0c, tx);
        div_term<S, 1>(P, io, g, i, j, k, d0c, ty);
        div_term<S, 2>(P, io, g, i, j, k, d0c, tz);
        const DevMat& mt = io.mats[id - 1];
        for (int a = 0; a < 3; a++) {
            const double f = tx[a] + ty[a] + tz[a];
            const double fs = io.force_store.c[a][c];
            if (S == 1 || S == 2)
                dv[a] = f * mt.dens_dt + mt.mass_damp * io.v_x.c[a][c] + mt.stiff_damp * (f - fs) * 2.;
            else
                dv[a] = f * mt.dens_dt + mt.mass_damp * io.v_x.c[a][c] + mt.stiff_damp * (f - fs);
            if (S == 0) io.force_store.c[a][c] = f;
        }
    }

    // ---- RK4 combination for v and u (du = v_stage * dt) ----
    for (int a = 0; a < 3; a++) {
        const double du = io.v_in.c[a][c] * P.dt;
        if (S == 0) {
            const double vx = io.v_x.c[a][c], ux = io.u_x.c[a][c];
            io.v_out.c[a][c] = vx + dv[a] * 0.5; io.v_acc.c[a][c] = vx + dv[a] / 6.;
            io.u_out.c[a][c] = ux + du * 0.5;    io.u_acc.c[a][c] = ux + du / 6.;
        } else if (S == 1) {
            const double vx = io.v_x.c[a][c], ux = io.u_x.c[a][c];
            io.v_out.c[a][c] = vx + dv[a] * 0.5; io.v_acc.c[a][c] = io.v_acc.c[a][c] + dv[a] / 3.;
            io.u_out.c[a][c] = ux + du * 0.5;    io.u_acc.c[a][c] = io.u_acc.c[a][c] + du / 3.;
        } else if (S == 2) {
            const double vx = io.v_x.c[a][c], ux = io.u_x.c[a][c];
            io.v_out.c[a][c] = vx + dv[a];       io.v_acc.c[a][c] = io.v_acc.c[a][c] + dv[a] / 3.;
            io.u_out.c[a][c] = ux + du;          io.u_acc.c[a][c] = io.u_acc.c[a][c] + du / 3.;
        } else {
            io.v_acc.c[a][c] = io.v_acc.c[a][c] + dv[a] / 6.;
            io.u_acc.c[a][c] = io.u_acc.c[a][c] + du / 6.;
        }
    }
}

// cell strain (global frame) of the current step for output (Dexx_glb ...)
__global__ void k_cell_strain(Params P, StageIO io, double* out6) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const GradView g(P, io);
    double e[6];
    g.strain_glb(i, j, k, e);
    for (int a = 0; a < 6; a++) out6[(long)a * P.n + c] = e[a];
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
