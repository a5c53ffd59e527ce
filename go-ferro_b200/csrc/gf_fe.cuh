// Ferroelectric second-order TDGL stage kernel (FP64 parity form and FP32
// mixed form).
//
// One thread per cell: q-increment of ferroelectric_system::get_dq_RK{1..4}
// (ferroelectric_solver.cpp:534-842: 8th-order Landau polynomial,
// electrostriction, gradient energy with the mirror interface condition of
// get_laplacian_p_local :3-131, static, external and Maxwell fields, damping),
// p-increment of get_dp_RK* (:1786-1832) and the RK4 combination of
// update_q*/update_p* (:1835-1999), fused in one pass.  Integer powers are
// evaluated by multiplication instead of pow().
#pragma once

#include "gf_elastic.cuh"

namespace gf {

template <class R>
__device__ inline bool is_fe(const DevMatT<R>* mats, uint8_t id) {
    return id != 0 && (mats[id - 1].flags & MF_FE);
}

// Global-frame cell strain of the stage displacement of cell (i,j,k)
// (Dexx_glb ..., get_dudxyz_glb + get_Dstrain, elastic_dynamic_solver.cpp:
// 106-227), formed from u_in directly: the face-normal gradient on each of
// the six faces (0 on stress-free faces: a non-periodic end face, or vacuum
// on either side), averaged per component exactly as the stored face
// gradients are in k_elastic_tile.  u = the cell's displacement, un = the
// six neighbours' (-x, +x, -y, +y, -z, +z, wrapped), solid_nb = whether each
// neighbour is a material cell.  gn, when given, receives the normal
// gradients gn[d][0 / 1] = d u_d / d x_d on the -d / +d face.
// cell_strain_glb loads u and un of cell c and neighbour indices nb.
template <class R>
__device__ inline void cell_strain_vals(const Params& P, int i, int j, int k, const R u[3], const R (&un)[3][6],
                                        const bool solid_nb[6], bool solid, R e[6], R (*gn)[2] = nullptr) {
    R g[3][2][3];   // g[d][0 / 1][a]: d u_a / d x_d on the -d / +d face
    const int pos[3] = {i, j, k}, n[3] = {P.nx, P.ny, P.nz}, per[3] = {P.per_x, P.per_y, P.per_z};
    const double h[3] = {P.dx, P.dy, P.dz}, rh[3] = {P.rdx, P.rdy, P.rdz};
    const float rhf[3] = {P.f.rdx, P.f.rdy, P.f.rdz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const bool fm = (pos[d] == 0 && !per[d]) || !(solid && solid_nb[2 * d]);
        const bool fp = (pos[d] == n[d] - 1 && !per[d]) || !(solid && solid_nb[2 * d + 1]);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            g[d][0][a] = fm ? R(0.) : qdivR((u[a] - un[a][2 * d]), h[d], rh[d], rhf[d]);
            g[d][1][a] = fp ? R(0.) : qdivR((un[a][2 * d + 1] - u[a]), h[d], rh[d], rhf[d]);
        }
    }
    e[0] = (g[0][0][0] + g[0][1][0]) / R(2.);
    e[1] = (g[1][0][1] + g[1][1][1]) / R(2.);
    e[2] = (g[2][0][2] + g[2][1][2]) / R(2.);
    e[3] = (g[2][0][1] + g[2][1][1] + g[1][0][2] + g[1][1][2]) / R(4.);
    e[4] = (g[2][0][0] + g[2][1][0] + g[0][0][2] + g[0][1][2]) / R(4.);
    e[5] = (g[1][0][0] + g[1][1][0] + g[0][0][1] + g[0][1][1]) / R(4.);
    if (gn) {
#pragma unroll
        for (int d = 0; d < 3; d++) { gn[d][0] = g[d][0][d]; gn[d][1] = g[d][1][d]; }
    }
}
template <class R>
__device__ inline void cell_strain_glb(const Params& P, const StageIOT<R>& io, int i, int j, int k, int c,
                                       const int nb[6], const bool solid_nb[6], bool solid, R e[6], R (*gn)[2] = nullptr) {
    R u[3], un[3][6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        u[a] = io.u_in.c[a][c];
#pragma unroll
        for (int f = 0; f < 6; f++) un[a][f] = io.u_in.c[a][nb[f]];
    }
    cell_strain_vals(P, i, j, k, u, un, solid_nb, solid, e, gn);
}

// crystal frame of a global-frame strain (Voigt order), in place
template <class R>
__device__ inline void strain_to_crt(const Params& P, R e[6]) {
    if (P.rot) {
        R t3[3][3] = {{e[0], e[5], e[4]}, {e[5], e[1], e[3]}, {e[4], e[3], e[2]}}, o3[3][3];
        rot_tensor(Tg2c<R>(P), t3, o3);
        e[0] = o3[0][0]; e[1] = o3[1][1]; e[2] = o3[2][2]; e[3] = o3[1][2]; e[4] = o3[0][2]; e[5] = o3[0][1];
    }
}

// Crystal-frame cell strain (Dexx_crt ...): cell_strain_glb rotated with Tg2c.
template <class R>
__device__ inline void fe_cell_strain(const Params& P, const StageIOT<R>& io, int i, int j, int k, int c,
                                      const int nb[6], const bool solid_nb[6], bool solid, R e[6]) {
    cell_strain_glb(P, io, i, j, k, c, nb, solid_nb, solid, e);
    strain_to_crt(P, e);
}

// Neighbour indices of cell (i,j,k), wrapped: -x, +x, -y, +y, -z, +z.
__device__ inline void cell_neighbours(const Params& P, int i, int j, int k, int nb[6]) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ib = (i == 0) ? nx - 1 : i - 1, iF = (i == nx - 1) ? 0 : i + 1;
    const int jb = (j == 0) ? ny - 1 : j - 1, jF = (j == ny - 1) ? 0 : j + 1;
    const int kb = (k == 0) ? nz - 1 : k - 1, kF = (k == nz - 1) ? 0 : k + 1;
    nb[0] = (ib * ny + j) * nz + k; nb[1] = (iF * ny + j) * nz + k;
    nb[2] = (i * ny + jb) * nz + k; nb[3] = (i * ny + jF) * nz + k;
    nb[4] = (i * ny + j) * nz + kb; nb[5] = (i * ny + j) * nz + kF;
}

// Flexoelectric inputs of one RK stage, from the stage state, one thread per
// cell (run before the stage's elastic and TDGL kernels):
//  * sg: the global-frame cell strain of every cell (get_Dstrain,
//    elastic_dynamic_solver.cpp:189-227, which update_u_RK* recomputes after
//    each displacement update), read by k_fe for the strain gradients;
//  * pge: the polarisation-gradient combinations of the dynamic eigenstrain
//    (elastic_dynamic_solver.cpp:63-70) from get_p_gradient
//    (ferroelectric_solver.cpp:133-280: central differences of p_store with
//    the mirror condition at ferroelectric surfaces), zero outside
//    ferroelectric cells.
template <class R>
__global__ void __launch_bounds__(256) k_flexo_prep(Params P, StageIOT<R> io) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.ny * P.nz) return;
    const int i = blockIdx.y, j = t / P.nz, k = t - (t / P.nz) * P.nz;
    const int c = (i * P.ny + j) * P.nz + k;
    const uint8_t id = io.mid[c];
    int nb[6];
    cell_neighbours(P, i, j, k, nb);
    if (P.elastic) {
        const bool solid_nb[6] = {io.mid[nb[0]] != 0, io.mid[nb[1]] != 0, io.mid[nb[2]] != 0,
                                  io.mid[nb[3]] != 0, io.mid[nb[4]] != 0, io.mid[nb[5]] != 0};
        R e[6];
        cell_strain_glb(P, io, i, j, k, c, nb, solid_nb, id != 0, e);
#pragma unroll
        for (int a = 0; a < 6; a++) io.sg[a][c] = e[a];
    }
    if (io.pge[0]) {
        R g[6] = {R(0.), R(0.), R(0.), R(0.), R(0.), R(0.)};
        if (id != 0 && ((P.fe_mask >> (id - 1)) & 1u)) {
            const int pos[3] = {i, j, k}, n[3] = {P.nx, P.ny, P.nz}, per[3] = {P.per_x, P.per_y, P.per_z};
            const double h[3] = {P.dx, P.dy, P.dz}, rh[3] = {P.rdx, P.rdy, P.rdz};
            const float rhf[3] = {P.f.rdx, P.f.rdy, P.f.rdz};
            R dp[3][3];   // dp[a][d] = d p_a / d x_d
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const uint8_t ib = io.mid[nb[2 * d]], iF = io.mid[nb[2 * d + 1]];
                const bool sb = (pos[d] == 0 && !per[d]) || !(ib != 0 && ((P.fe_mask >> (ib - 1)) & 1u));
                const bool sf = (pos[d] == n[d] - 1 && !per[d]) || !(iF != 0 && ((P.fe_mask >> (iF - 1)) & 1u));
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const R pc = io.p_in.c[a][c];
                    const R pb = sb ? pc : io.p_in.c[a][nb[2 * d]];
                    const R pf = sf ? pc : io.p_in.c[a][nb[2 * d + 1]];
                    dp[a][d] = qdivR(pf - pb, h[d], rh[d], rhf[d]) / R(2.);
                }
            }
            g[0] = dp[0][0]; g[1] = dp[1][1]; g[2] = dp[2][2];
            g[3] = dp[1][2] + dp[2][1];
            g[4] = dp[0][2] + dp[2][0];
            g[5] = dp[1][0] + dp[0][1];
        }
#pragma unroll
        for (int a = 0; a < 6; a++) io.pge[a][c] = g[a];
    }
}

// Grid: (blocks over the (j,k) plane) x (nx planes), 32-bit indices.
#ifndef GF_FE_MINB_F32
#define GF_FE_MINB_F32 5
#endif
#ifndef GF_FE_MINB_F64
#define GF_FE_MINB_F64 3
#endif
// The TDGL increment dq of a ferroelectric cell (get_dq_RK*,
// ferroelectric_solver.cpp:534-842) from its stencil results: the global-
// frame p of the cell, the Laplacian lap of p with the mirror condition, the
// dynamic crystal-frame strain edyn of the stage displacement (read with
// elastodynamics and if_elasto_on), and, for flexoelectric runs, the second
// and first p derivatives d2s, dp with the neighbour indices nb and ids idn.
template <int S, class R, bool FX>
__device__ __forceinline__ void fe_dq(const Params& P, const StageIOT<R>& io, int i, int j, int k, int c,
                                      const DevMatT<R>& mt, R pxg, R pyg, R pzg, const R lap[3], const R edyn[6],
                                      const R (&d2s)[3][3], const R (&dp)[3][3], const int nb[6], const uint8_t idn[6],
                                      R dq[3]) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const double h[3] = {P.dx, P.dy, P.dz}, rh[3] = {P.rdx, P.rdy, P.rdz};
    const float rhf[3] = {P.f.rdx, P.f.rdy, P.f.rdz};
    (void)nx; (void)h; (void)rh; (void)rhf; (void)nb; (void)idn; (void)d2s; (void)dp;
    R px, py, pz;
    glb2crt(P, pxg, pyg, pzg, px, py, pz);

    R exx = R(0), eyy = R(0), ezz = R(0), eyz = R(0), exz = R(0), exy = R(0);
    R exx0 = R(0), eyy0 = R(0), ezz0 = R(0), eyz0 = R(0), exz0 = R(0), exy0 = R(0);
    if (P.elasto_on) {
        // dynamic strain and eigenstrain of the stage state, crystal frame
        // (Dexx_crt, Dexx0_crt: ferroelectric_solver.cpp:624-652)
        if (P.elastic) {
            exx = edyn[0]; eyy = edyn[1]; ezz = edyn[2]; eyz = edyn[3]; exz = edyn[4]; exy = edyn[5];
        }
        if (P.elasto_back) {
            R e0[6];
            eigen_crt(P, io, c, e0);
            exx0 = e0[0]; eyy0 = e0[1]; ezz0 = e0[2]; eyz0 = e0[3]; exz0 = e0[4]; exy0 = e0[5];
        }
        if (P.elastostatic) {
            // plus the static strain and static eigenstrain
            // (ferroelectric_solver.cpp:638-651; zeros when absent)
            auto st = [&](const R* const* f, int q) { return f[q] ? f[q][c] : R(0.); };
            exx = exx + st(io.eps0_c, 0); eyy = eyy + st(io.eps0_c, 1); ezz = ezz + st(io.eps0_c, 2);
            eyz = eyz + st(io.eps0_c, 3); exz = exz + st(io.eps0_c, 4); exy = exy + st(io.eps0_c, 5);
            exx0 = exx0 + st(io.eig0_c, 0); eyy0 = eyy0 + st(io.eig0_c, 1); ezz0 = ezz0 + st(io.eig0_c, 2);
            eyz0 = eyz0 + st(io.eig0_c, 3); exz0 = exz0 + st(io.eig0_c, 4); exy0 = exy0 + st(io.eig0_c, 5);
        }
    }

    const R fm = mt.fe_coef;
    R qxc, qyc, qzc;
    if constexpr (is_mixed<R>::value) {
        // mixed form: the same Landau field with p_a factored out and the
        // powers and pair sums shared by the three components (FMA
        // contraction; FP32 rounding, not the reference's order):
        // dF/dp_a = p_a [2a1 + o2 (4a11 + o2 (6a111 + 8a1111 o2))
        //   + s (2a12 + 4a112 o2 + 6a1112 o4) + q (2a112 + 4a1122 o2)
        //   + 2a1112 c + r (2a123 + 2a1123 (2 o2 + s))]
        // with o2, o4 = p_a^2, p_a^4 and s, q, c, r = the sum of squares,
        // fourth and sixth powers, and the product of squares of the
        // other two components
        const R x2 = px * px, y2 = py * py, z2 = pz * pz;
        const R x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;
        const R x6 = x4 * x2, y6 = y4 * y2, z6 = z4 * z2;
        const R c1 = R(2.) * mt.a1, c11 = R(4.) * mt.a11, c111 = R(6.) * mt.a111, c1111 = R(8.) * mt.a1111;
        const R c12 = R(2.) * mt.a12, c112a = R(4.) * mt.a112, c1112a = R(6.) * mt.a1112, c112b = R(2.) * mt.a112;
        const R c1122 = R(4.) * mt.a1122, c1112b = R(2.) * mt.a1112, c123 = R(2.) * mt.a123, c1123 = R(2.) * mt.a1123;
        auto br = [&](R o2, R o4, R s_, R q_, R cc, R r_) {
            R b = c1 + o2 * (c11 + o2 * (c111 + c1111 * o2));
            b = b + s_ * (c12 + c112a * o2 + c1112a * o4);
            b = b + q_ * (c112b + c1122 * o2);
            b = b + c1112b * cc;
            b = b + r_ * (c123 + c1123 * (R(2.) * o2 + s_));
            return b;
        };
        qxc = fm * (px * br(x2, x4, y2 + z2, y4 + z4, y6 + z6, y2 * z2)
                    + (mt.tv1 * (exx0 - exx) + mt.tv2 * (eyy0 - eyy + ezz0 - ezz)) * px
                    + mt.tv3 * ((exy0 - exy) * py + (exz0 - exz) * pz));
        qyc = fm * (py * br(y2, y4, x2 + z2, x4 + z4, x6 + z6, x2 * z2)
                    + (mt.tv1 * (eyy0 - eyy) + mt.tv2 * (exx0 - exx + ezz0 - ezz)) * py
                    + mt.tv3 * ((exy0 - exy) * px + (eyz0 - eyz) * pz));
        qzc = fm * (pz * br(z2, z4, x2 + y2, x4 + y4, x6 + y6, x2 * y2)
                    + (mt.tv1 * (ezz0 - ezz) + mt.tv2 * (exx0 - exx + eyy0 - eyy)) * pz
                    + mt.tv3 * ((exz0 - exz) * px + (eyz0 - eyz) * py));
    } else {
        const R px2 = px * px, py2 = py * py, pz2 = pz * pz;
        const R px3 = px2 * px, py3 = py2 * py, pz3 = pz2 * pz;
        const R px4 = px2 * px2, py4 = py2 * py2, pz4 = pz2 * pz2;
        const R px5 = px4 * px, py5 = py4 * py, pz5 = pz4 * pz;
        const R px6 = px4 * px2, py6 = py4 * py2, pz6 = pz4 * pz2;
        const R px7 = px6 * px, py7 = py6 * py, pz7 = pz6 * pz;
        qxc = fm * (R(2.) * mt.a1 * px + R(4.) * mt.a11 * px3
            + R(2.) * mt.a12 * (py2 + pz2) * px
            + R(6.) * mt.a111 * px5
            + R(4.) * mt.a112 * px3 * (py2 + pz2)
            + R(2.) * mt.a112 * (py4 + pz4) * px
            + R(2.) * mt.a123 * px * py2 * pz2
            + R(8.) * mt.a1111 * px7
            + R(2.) * mt.a1112 * px * (py6 + pz6 + R(3.) * px4 * (py2 + pz2))
            + R(4.) * mt.a1122 * px3 * (py4 + pz4)
            + R(2.) * mt.a1123 * px * py2 * pz2 * (R(2.) * px2 + py2 + pz2)
            + (mt.tv1 * (exx0 - exx) + mt.tv2 * (eyy0 - eyy + ezz0 - ezz)) * px
            + mt.tv3 * ((exy0 - exy) * py + (exz0 - exz) * pz));
        qyc = fm * (R(2.) * mt.a1 * py + R(4.) * mt.a11 * py3
            + R(2.) * mt.a12 * (pz2 + px2) * py
            + R(6.) * mt.a111 * py5
            + R(4.) * mt.a112 * py3 * (px2 + pz2)
            + R(2.) * mt.a112 * (px4 + pz4) * py
            + R(2.) * mt.a123 * py * px2 * pz2
            + R(8.) * mt.a1111 * py7
            + R(2.) * mt.a1112 * py * (px6 + pz6 + R(3.) * py4 * (px2 + pz2))
            + R(4.) * mt.a1122 * py3 * (px4 + pz4)
            + R(2.) * mt.a1123 * py * px2 * pz2 * (px2 + R(2.) * py2 + pz2)
            + (mt.tv1 * (eyy0 - eyy) + mt.tv2 * (exx0 - exx + ezz0 - ezz)) * py
            + mt.tv3 * ((exy0 - exy) * px + (eyz0 - eyz) * pz));
        qzc = fm * (R(2.) * mt.a1 * pz + R(4.) * mt.a11 * pz3
            + R(2.) * mt.a12 * (py2 + px2) * pz
            + R(6.) * mt.a111 * pz5
            + R(4.) * mt.a112 * pz3 * (py2 + px2)
            + R(2.) * mt.a112 * (py4 + px4) * pz
            + R(2.) * mt.a123 * pz * py2 * px2
            + R(8.) * mt.a1111 * pz7
            + R(2.) * mt.a1112 * pz * (py6 + px6 + R(3.) * pz4 * (py2 + px2))
            + R(4.) * mt.a1122 * pz3 * (py4 + px4)
            + R(2.) * mt.a1123 * pz * px2 * py2 * (px2 + py2 + R(2.) * pz2)
            + (mt.tv1 * (ezz0 - ezz) + mt.tv2 * (exx0 - exx + eyy0 - eyy)) * pz
            + mt.tv3 * ((exz0 - exz) * px + (eyz0 - eyz) * py));
    }
    R gx, gy, gz;
    crt2glb(P, qxc, qyc, qzc, gx, gy, gz);

    const StageDrive& dr = stage_drive(io, S);
    const R g[3] = {gx, gy, gz};
    // E_stat is read only where it may be nonzero: x - (+0) is x in
    // every bit, so leaving out an all-zero field changes nothing
    for (int a = 0; a < 3; a++) {
        R inner = -R(1.) * mt.G11 * lap[a];
        if (P.estat) inner = inner - io.Estat.c[a][c];
        dq[a] = g[a] + fm * (inner - R(dr.Eext[a])) + mt.fe_damp * io.q_in.c[a][c];
    }

    if (P.em_back_P) {
        // cell-centred Maxwell E of the stage state (EMdynamic_solver.cpp:3813-3826)
        const int ny1 = ny + 1, nz1 = nz + 1;
        const int ex = (i * ny1 + j) * nz1 + k;
        const int ey = (i * ny + j) * nz1 + k;
        const int ez = (i * ny1 + j) * nz + k;
        const R Ecx = (io.E_in.c[0][ex] + io.E_in.c[0][ex + nz1] + io.E_in.c[0][ex + 1] + io.E_in.c[0][ex + nz1 + 1]) / R(4.);
        const R Ecy = (io.E_in.c[1][ey] + io.E_in.c[1][ey + ny * nz1] + io.E_in.c[1][ey + 1] + io.E_in.c[1][ey + ny * nz1 + 1]) / R(4.);
        const R Ecz = (io.E_in.c[2][ez] + io.E_in.c[2][ez + ny1 * nz] + io.E_in.c[2][ez + nz] + io.E_in.c[2][ez + ny1 * nz + nz]) / R(4.);
        dq[0] = dq[0] - fm * Ecx;
        dq[1] = dq[1] - fm * Ecy;
        dq[2] = dq[2] - fm * Ecz;
    }

    if constexpr (FX) {
        // strain gradients of the stage displacement (get_Dstrain_gradient,
        // elastic_dynamic_solver.cpp:229-399): eg[q][d] = d e_q / d x_d of
        // the global-frame cell strain (q = xx, yy, zz, yz, xz, xy).  The
        // normal component differentiates the face gradients of the two
        // d-faces; the others take central differences of the
        // neighbours' strains, one-sided next to a stress-free face and
        // zero between two.  Zero without elastodynamics.
        R eg[6][3];
#pragma unroll
        for (int q = 0; q < 6; q++)
#pragma unroll
            for (int d = 0; d < 3; d++) eg[q][d] = R(0.);
        if (P.elastic) {
            const int pos[3] = {i, j, k}, n[3] = {nx, ny, nz}, per[3] = {P.per_x, P.per_y, P.per_z};
            // the components each direction needs besides its normal one
            constexpr int need[3][4] = {{1, 2, 5, 4}, {0, 2, 5, 3}, {0, 1, 3, 4}};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const bool fb = (pos[d] == 0 && !per[d]) || idn[2 * d] == 0;
                const bool ff = (pos[d] == n[d] - 1 && !per[d]) || idn[2 * d + 1] == 0;
                const R* ud = io.u_in.c[d];
                const R uc = ud[c];
                const R gb = fb ? R(0.) : qdivR((uc - ud[nb[2 * d]]), h[d], rh[d], rhf[d]);
                const R gf = ff ? R(0.) : qdivR((ud[nb[2 * d + 1]] - uc), h[d], rh[d], rhf[d]);
                eg[d][d] = qdivR(gf - gb, h[d], rh[d], rhf[d]);
                // the cell itself stands in for the neighbour across a
                // stress-free face; the step is two cells only when
                // neither face is free
                const int cb = fb ? c : nb[2 * d];
                const int cf = ff ? c : nb[2 * d + 1];
                const bool two = !fb && !ff;
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int q = need[d][r];
                    const R v = qdivR(io.sg[q][cf] - io.sg[q][cb], h[d], rh[d], rhf[d]);
                    eg[q][d] = two ? v / R(2.) : v;
                }
            }
        }
        // the flexoelectric effective field of each component, in the
        // reference's term order
        const R ax = mt.tv4 * pxg * dp[0][0]
            + mt.tv5 * (pyg * dp[1][0] + pzg * dp[2][0])
            + mt.tv6 * (pxg * dp[1][1] + pxg * dp[2][2] + pyg * dp[0][1] + pzg * dp[0][2])
            - mt.tv7 * d2s[0][0]
            - mt.tv8 * (d2s[0][2] + d2s[0][1])
            - mt.f11 * eg[0][0] - mt.f12 * (eg[1][0] + eg[2][0])
            - mt.f44x2 * (eg[5][1] + eg[4][2]);
        const R ay = mt.tv4 * pyg * dp[1][1]
            + mt.tv5 * (pxg * dp[0][1] + pzg * dp[2][1])
            + mt.tv6 * (pyg * dp[0][0] + pyg * dp[2][2] + pxg * dp[1][0] + pzg * dp[1][2])
            - mt.tv7 * d2s[1][1]
            - mt.tv8 * (d2s[1][0] + d2s[1][2])
            - mt.f11 * eg[1][1] - mt.f12 * (eg[0][1] + eg[2][1])
            - mt.f44x2 * (eg[5][0] + eg[3][2]);
        const R az = mt.tv4 * pzg * dp[2][2]
            + mt.tv5 * (pxg * dp[0][2] + pyg * dp[1][2])
            + mt.tv6 * (pzg * dp[0][0] + pzg * dp[1][1] + pxg * dp[2][0] + pyg * dp[2][1])
            - mt.tv7 * d2s[2][2]
            - mt.tv8 * (d2s[2][0] + d2s[2][1])
            - mt.f11 * eg[2][2] - mt.f12 * (eg[0][2] + eg[1][2])
            - mt.f44x2 * (eg[3][1] + eg[4][0]);
        dq[0] = dq[0] + fm * ax;
        dq[1] = dq[1] + fm * ay;
        dq[2] = dq[2] + fm * az;
    }
}

// RK4 combination of q and p of one cell (update_q*/update_p*,
// ferroelectric_solver.cpp:1835-1999) with the TDGL increment dq (zero
// outside ferroelectric cells; dp = q_stage * dt): the operands of all three
// components are loaded before the first store, so the six scalars' loads
// are in flight together
template <int S, class R>
__device__ __forceinline__ void fe_rk(const Params& P, const StageIOT<R>& io, int c, const R dq[3]) {
    R qin[3], qx[3], px0[3], qa[3], pa[3], qc[3], pcm[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        qin[a] = io.q_in.c[a][c]; qx[a] = io.q_x.c[a][c]; px0[a] = io.p_x.c[a][c];
        qa[a] = pa[a] = qc[a] = pcm[a] = R(0.);
        if (S > 0) { qa[a] = io.q_acc.c[a][c]; pa[a] = io.p_acc.c[a][c]; }
        if constexpr (is_mixed<R>::value) { if (S == 3) { qc[a] = io.q_cmp.c[a][c]; pcm[a] = io.p_cmp.c[a][c]; } }
    }
    if constexpr (is_mixed<R>::value) {
        // mixed form: compensated RK4
        const float dt = P.f.dt;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float dp = qin[a] * dt;
            rk_mixed_v<S>(qx[a], qa[a], qc[a], dq[a], io.q_out.c[a], io.q_acc.c[a], io.q_cmp.c[a], c);
            rk_mixed_v<S>(px0[a], pa[a], pcm[a], dp, io.p_out.c[a], io.p_acc.c[a], io.p_cmp.c[a], c);
        }
    } else {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double dp = qin[a] * P.dt;
            if (S == 0) {
                io.q_out.c[a][c] = qx[a] + dq[a] * 0.5; io.q_acc.c[a][c] = qx[a] + qdiv(dq[a], 6., kInv6);
                io.p_out.c[a][c] = px0[a] + dp * 0.5;   io.p_acc.c[a][c] = px0[a] + qdiv(dp, 6., kInv6);
            } else if (S == 1) {
                io.q_out.c[a][c] = qx[a] + dq[a] * 0.5; io.q_acc.c[a][c] = qa[a] + qdiv(dq[a], 3., kInv3);
                io.p_out.c[a][c] = px0[a] + dp * 0.5;   io.p_acc.c[a][c] = pa[a] + qdiv(dp, 3., kInv3);
            } else if (S == 2) {
                io.q_out.c[a][c] = qx[a] + dq[a];       io.q_acc.c[a][c] = qa[a] + qdiv(dq[a], 3., kInv3);
                io.p_out.c[a][c] = px0[a] + dp;         io.p_acc.c[a][c] = pa[a] + qdiv(dp, 3., kInv3);
            } else {
                io.q_acc.c[a][c] = qa[a] + qdiv(dq[a], 6., kInv6);
                io.p_acc.c[a][c] = pa[a] + qdiv(dp, 6., kInv6);
            }
        }
    }
}

template <int S, class R, bool FX>
// FX: the run has flexoelectricity (the polarisation- and strain-gradient
// terms of get_dq_RK*, ferroelectric_solver.cpp:800-833).
// FP64 (256, 3): 80 registers, 24 resident warps per SM (measured best of 2-4
// blocks); FP32 (256, 5): 48 registers, 40 warps, no spills.  With the RK
// operands of all three components gathered before the first store: 0.61 ms
// (FP64) per step on the 128^3 ferroelectric workload, against 0.79 at
// (256, 2); FP32 0.363 ms per step at (256, 5), against 0.381 at 4 (64
// registers), 0.368 at 6 (spills) and 0.49 at 3
__device__ __forceinline__ void fe_body(const Params& P, const StageIOT<R>& io, int bx, int by) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int t = bx * blockDim.x + threadIdx.x;
    if (t >= ny * nz) return;
    const int i = by, j = t / nz, k = t - (t / nz) * nz;
    const int c = (i * ny + j) * nz + k;
    const uint8_t id = io.mid[c];
    R dq[3] = {R(0.), R(0.), R(0.)};

    // material classes from the run's bitmask: no table load on the path to
    // the neighbour loads
    auto fe_id = [&](uint8_t q) { return q != 0 && ((P.fe_mask >> (q - 1)) & 1u); };
    if (fe_id(id)) {
        const DevMatT<R>& mt = io.mats[id - 1];
        const R pxg = io.p_in.c[0][c], pyg = io.p_in.c[1][c], pzg = io.p_in.c[2][c];

        // ---- Laplacian with mirror condition at FE interfaces ----
        const int ib = (i == 0) ? nx - 1 : i - 1, iF = (i == nx - 1) ? 0 : i + 1;
        const int jb = (j == 0) ? ny - 1 : j - 1, jF = (j == ny - 1) ? 0 : j + 1;
        const int kb = (k == 0) ? nz - 1 : k - 1, kF = (k == nz - 1) ? 0 : k + 1;
        const int nb[6] = {(ib * ny + j) * nz + k, (iF * ny + j) * nz + k, (i * ny + jb) * nz + k,
                           (i * ny + jF) * nz + k, (i * ny + j) * nz + kb, (i * ny + j) * nz + kF};
        // the six neighbours' p is loaded whether or not it is used (the
        // wrapped indices are always inside the array), so these loads do not
        // wait for the neighbour ids
        R pn[3][6];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int f = 0; f < 6; f++) pn[a][f] = io.p_in.c[a][nb[f]];
        uint8_t idn[6];
#pragma unroll
        for (int f = 0; f < 6; f++) idn[f] = io.mid[nb[f]];
        const bool surf[6] = {(i == 0 && !P.per_x) || !fe_id(idn[0]),
                              (i == nx - 1 && !P.per_x) || !fe_id(idn[1]),
                              (j == 0 && !P.per_y) || !fe_id(idn[2]),
                              (j == ny - 1 && !P.per_y) || !fe_id(idn[3]),
                              (k == 0 && !P.per_z) || !fe_id(idn[4]),
                              (k == nz - 1 && !P.per_z) || !fe_id(idn[5])};
        const double h[3] = {P.dx, P.dy, P.dz}, rh[3] = {P.rdx, P.rdy, P.rdz};
        const float rhf[3] = {P.f.rdx, P.f.rdy, P.f.rdz};
        R lap[3];   // sum of the three second derivatives per component
        // flexoelectric runs keep each second derivative and the first
        // derivatives of get_p_gradient (same mirrored neighbours)
        R d2s[3][3], dp[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const R pc = io.p_in.c[a][c];
            R d2[3];
#pragma unroll
            for (int dir = 0; dir < 3; dir++) {
                const R pb = surf[2 * dir] ? pc : pn[a][2 * dir];
                const R pf = surf[2 * dir + 1] ? pc : pn[a][2 * dir + 1];
                d2[dir] = qdivR(qdivR(pf - R(2.) * pc + pb, h[dir], rh[dir], rhf[dir]), h[dir], rh[dir], rhf[dir]);
                if constexpr (FX) {
                    d2s[a][dir] = d2[dir];
                    dp[a][dir] = qdivR(pf - pb, h[dir], rh[dir], rhf[dir]) / R(2.);
                }
            }
            lap[a] = d2[0] + d2[1] + d2[2];
        }

        R edyn[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
        if (P.elasto_on && P.elastic) {
            if constexpr (is_mixed<R>::value) {
                // mixed form: from the stage displacement (the values
                // k_elastic_tile forms), 12 bytes of u instead of 24 of strain
                const bool solid_nb[6] = {idn[0] != 0, idn[1] != 0, idn[2] != 0, idn[3] != 0, idn[4] != 0, idn[5] != 0};
                fe_cell_strain(P, io, i, j, k, c, nb, solid_nb, true, edyn);
            } else {
                // FP64: written by k_elastic_tile earlier in the same stage
                // (forming it here costs the FP64 kernel more in registers
                // and latency than the 48 bytes it saves)
#pragma unroll
                for (int q = 0; q < 6; q++) edyn[q] = io.strain_c[q][c];
            }
        }
        fe_dq<S, R, FX>(P, io, i, j, k, c, mt, pxg, pyg, pzg, lap, edyn, d2s, dp, nb, idn, dq);
    }
    fe_rk<S, R>(P, io, c, dq);
}


// block (bx, by): 256 cells of the (j, k) plane bx of x-plane by
template <int S, class R = double, bool FX = false>
__global__ void __launch_bounds__(256, is_mixed<R>::value ? GF_FE_MINB_F32 : GF_FE_MINB_F64) k_fe(Params P, StageIOT<R> io) {
    fe_body<S, R, FX>(P, io, blockIdx.x, blockIdx.y);
}

}  // namespace gf
