// Elastodynamics stage kernels (FP64 parity form and FP32 mixed form).
//
//   k_elastic_tile  per cell, tiled over (j,k) and marching along x: the
//                 face-normal displacement gradients (get_dudxyz_glb,
//                 elastic_dynamic_solver.cpp:106-187), cell strains (get_Dstrain,
//                 :189-227) and dynamic eigenstrains of m and p
//                 (get_eigenstrain_dynamic, :3-104), the six face stresses and
//                 the stress divergence (the stress part of get_dv_RK{1..4}
//                 :841-2800); it also stores the crystal-frame cell strain of
//                 magnetic cells for the LLG kernels and, in the FP64 form, of
//                 ferroelectric cells for the TDGL kernel.
//   k_elastic_rk  per cell: damping terms, f_store, the velocity and
//                 displacement increments and their RK4 combination
//                 (get_dv_RK* :1295-1329, get_du_RK* :2801-2847,
//                 update_v*/update_u* :2849-3057).
//   k_elastic_bc  per (i,j) column: z absorbing boundary (Liao 4th order or
//                 first-order Mur, elastodynamics_AbsorbingBoundary.cpp:91-230)
//                 and the displacement source plane (update_Du_Gaussian*,
//                 elastic_dynamic_solver.cpp:3059-3284), in that order.
//   k_face_grad, k_cell_strain  the cell strain of the current state, for
//                 output only.
//
// Face f of an axis with n cells is stored at cell index f for f < n; face n
// is read from index 0, which holds the same value (periodic axis) or the
// same zero (non-periodic axis: both end faces are stress-free).
#pragma once

#include <cuda.h>

#include "gf_launch.cuh"
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

template <class R = double>
__global__ void __launch_bounds__(256) k_face_grad(Params P, StageIOT<R> io) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const bool fx = free_x(P, io.mid, i, j, k), fy = free_y(P, io.mid, i, j, k), fz = free_z(P, io.mid, i, j, k);
    const long cx = cid(P, i == 0 ? P.nx - 1 : i - 1, j, k);
    const long cy = cid(P, i, j == 0 ? P.ny - 1 : j - 1, k);
    const long cz = cid(P, i, j, k == 0 ? P.nz - 1 : k - 1);
    for (int a = 0; a < 3; a++) {
        const R* u = io.u_in.c[a];
        const R uc = u[c];
        io.fg[a][c] = fx ? R(0.) : qdivR((uc - u[cx]), P.dx, P.rdx, P.f.rdx);
        io.fg[3 + a][c] = fy ? R(0.) : qdivR((uc - u[cy]), P.dy, P.rdy, P.f.rdy);
        io.fg[6 + a][c] = fz ? R(0.) : qdivR((uc - u[cz]), P.dz, P.rdz, P.f.rdz);
    }
}

// read access to the stored face gradients; f may equal n
template <class R>
struct GradView {
    const Params& P;
    const StageIOT<R>& io;
    __device__ GradView(const Params& p, const StageIOT<R>& s) : P(p), io(s) {}
    __device__ R gx(int a, long f, long j, long k) const { return io.fg[a][cid(P, f == P.nx ? 0 : f, j, k)]; }
    __device__ R gy(int a, long i, long f, long k) const { return io.fg[3 + a][cid(P, i, f == P.ny ? 0 : f, k)]; }
    __device__ R gz(int a, long i, long j, long f) const { return io.fg[6 + a][cid(P, i, j, f == P.nz ? 0 : f)]; }
    // cell strain components in the global frame (get_Dstrain)
    __device__ R exx(long i, long j, long k) const { return (gx(0, i, j, k) + gx(0, i + 1, j, k)) / R(2.); }
    __device__ R eyy(long i, long j, long k) const { return (gy(1, i, j, k) + gy(1, i, j + 1, k)) / R(2.); }
    __device__ R ezz(long i, long j, long k) const { return (gz(2, i, j, k) + gz(2, i, j, k + 1)) / R(2.); }
    __device__ R eyz(long i, long j, long k) const {
        return (gz(1, i, j, k) + gz(1, i, j, k + 1) + gy(2, i, j, k) + gy(2, i, j + 1, k)) / R(4.);
    }
    __device__ R exz(long i, long j, long k) const {
        return (gz(0, i, j, k) + gz(0, i, j, k + 1) + gx(2, i, j, k) + gx(2, i + 1, j, k)) / R(4.);
    }
    __device__ R exy(long i, long j, long k) const {
        return (gy(0, i, j, k) + gy(0, i, j + 1, k) + gx(1, i, j, k) + gx(1, i + 1, j, k)) / R(4.);
    }
    __device__ void strain_glb(long i, long j, long k, R e[6]) const {
        e[0] = exx(i, j, k); e[1] = eyy(i, j, k); e[2] = ezz(i, j, k);
        e[3] = eyz(i, j, k); e[4] = exz(i, j, k); e[5] = exy(i, j, k);
    }
};

// ε0 of the cell from the crystal-frame m and p (get_eigenstrain_dynamic,
// elastic_dynamic_solver.cpp:38-61): magnetostriction of m, electrostriction
// of p, then the two AFM sublattices with half weight, minus the static
// eigenstrain e0.  The sublattice terms are added only when the run has
// antiferromagnets; without them they are exact zeros in the reference.
template <class R, class M>
__device__ inline void eigen_terms(const Params& P, const StageIOT<R>& io, long c, const M& mt, R mx, R my,
                                   R mz, R px, R py, R pz, const R e0[6], R e[6]) {
    const R third = R(1.) / R(3.);
    R t[6];
    t[0] = mt.l100_15 * (mx * mx - third);
    t[1] = mt.l100_15 * (my * my - third);
    t[2] = mt.l100_15 * (mz * mz - third);
    t[3] = mt.l111_15 * my * mz;
    t[4] = mt.l111_15 * mx * mz;
    t[5] = mt.l111_15 * my * mx;
    // electrostriction, added in the same order.  Evaluated also without
    // ferroelectrics (p = 0): the terms are then zeros, but adding +0 turns a
    // -0 magnetostriction term (e.g. l111 my mz with mz = 0, my < 0) into +0,
    // as the reference's unconditional sum does, so the sign of every zero
    // matches too
    t[0] = t[0] + mt.Q11 * (px * px) + mt.Q12 * ((py * py) + (pz * pz));
    t[1] = t[1] + mt.Q11 * (py * py) + mt.Q12 * ((px * px) + (pz * pz));
    t[2] = t[2] + mt.Q11 * (pz * pz) + mt.Q12 * ((py * py) + (px * px));
    t[3] = t[3] + mt.Q44 * py * pz;
    t[4] = t[4] + mt.Q44 * px * pz;
    t[5] = t[5] + mt.Q44 * py * px;
    if (P.afm) {
        R a1x, a1y, a1z, a2x, a2y, a2z;
        glb2crt(P, io.a1_in.c[0][c], io.a1_in.c[1][c], io.a1_in.c[2][c], a1x, a1y, a1z);
        glb2crt(P, io.a2_in.c[0][c], io.a2_in.c[1][c], io.a2_in.c[2][c], a2x, a2y, a2z);
        t[0] = t[0] + mt.l100a1_075 * (a1x * a1x - third) + mt.l100a2_075 * (a2x * a2x - third);
        t[1] = t[1] + mt.l100a1_075 * (a1y * a1y - third) + mt.l100a2_075 * (a2y * a2y - third);
        t[2] = t[2] + mt.l100a1_075 * (a1z * a1z - third) + mt.l100a2_075 * (a2z * a2z - third);
        t[3] = t[3] + mt.l111a1_075 * a1y * a1z + mt.l111a2_075 * a2y * a2z;
        t[4] = t[4] + mt.l111a1_075 * a1x * a1z + mt.l111a2_075 * a2x * a2z;
        t[5] = t[5] + mt.l111a1_075 * a1y * a1x + mt.l111a2_075 * a2y * a2x;
    }
    for (int a = 0; a < 6; a++) e[a] = t[a] - e0[a];
    if (P.flexo) {
        // flexoelectric eigenstrain of the polarisation gradient
        // (elastic_dynamic_solver.cpp:63-70), subtracted after e0 in the
        // reference's order; applied in every material cell (the gradients
        // are zero outside ferroelectrics), as the reference does
        const R g0 = io.pge[0][c], g1 = io.pge[1][c], g2 = io.pge[2][c];
        e[0] = e[0] - mt.F11 * g0 - mt.F12 * (g2 + g1);
        e[1] = e[1] - mt.F11 * g1 - mt.F12 * (g2 + g0);
        e[2] = e[2] - mt.F11 * g2 - mt.F12 * (g0 + g1);
        e[3] = e[3] - mt.F44h * io.pge[3][c];
        e[4] = e[4] - mt.F44h * io.pge[4][c];
        e[5] = e[5] - mt.F44h * io.pge[5][c];
    }
}

// dynamic eigenstrain of cell c in the crystal frame (Dexx0_crt ...,
// get_eigenstrain_dynamic)
template <class R>
__device__ inline void eigen_crt(const Params& P, const StageIOT<R>& io, long c, R e[6]) {
    const uint8_t id = io.mid[c];
    for (int a = 0; a < 6; a++) e[a] = R(0.);
    if (id == 0) return;
    const DevMatT<R>& mt = io.mats[id - 1];
    R px = R(0.), py = R(0.), pz = R(0.), mx = R(0.), my = R(0.), mz = R(0.);
    if (P.fe) glb2crt(P, io.p_in.c[0][c], io.p_in.c[1][c], io.p_in.c[2][c], px, py, pz);
    if (P.fm) glb2crt(P, io.m_in.c[0][c], io.m_in.c[1][c], io.m_in.c[2][c], mx, my, mz);
    R e0[6] = {R(0.), R(0.), R(0.), R(0.), R(0.), R(0.)};
    if (io.eig0_c[0]) for (int a = 0; a < 6; a++) e0[a] = io.eig0_c[a][c];
    eigen_terms(P, io, c, mt, mx, my, mz, px, py, pz, e0, e);
}

// eigenstrain in the global frame (Dexx0_glb ...)
template <class R>
__device__ inline void eigen_glb(const Params& P, const StageIOT<R>& io, long c, R e[6]) {
    eigen_crt(P, io, c, e);
    if (P.rot) {
        R s[3][3] = {{e[0], e[5], e[4]}, {e[5], e[1], e[3]}, {e[4], e[3], e[2]}}, o[3][3];
        rot_tensor(Tc2g<R>(P), s, o);
        e[0] = o[0][0]; e[1] = o[1][1]; e[2] = o[2][2]; e[3] = o[1][2]; e[4] = o[0][2]; e[5] = o[0][1];
    }
}

// ---------------------------------------------------------------------------
// Tiled stage kernel.  A block owns a TJ x TK tile of (j,k) columns and
// marches along x over `chunk` planes.  Per plane p it
//   A. computes from a two-plane ring of staged u and material ids the
//      face-normal gradients of the tile's cells and a one-cell halo (x-faces
//      on two planes, y- and z-faces) and the cells' eigenstrains,
//   B1. computes every y- and z-face stress of the tile once (one thread per
//      face) while the next plane's u and ids are staged,
//   B2. per column: the x-face stress (the cell below a face contributes its
//      half one plane earlier), the divergence of the previous plane's cell,
//      its RK4 update, and the strain output of this plane's cell.
// A face stress (get_dv_RK*, elastic_dynamic_solver.cpp:876-1289) is the
// mean over the two cells sharing the face of three rows of C (strain -
// eigenstrain), where each cell's strain takes the face's own gradient for
// the normal component and for the shear components that involve it; it is
// 0 on stress-free faces, except for the surface traction source.  Every
// expression keeps the reference's operation order (rounding included).
// ---------------------------------------------------------------------------

// elastic constants of one material, staged in shared memory
template <class R>
struct ElMat {
    R cij[6][6];
    R dens_dt, mass_damp, stiff_damp;
    R l100_15, l111_15, Q11, Q12, Q44;
    R l100a1_075, l100a2_075, l111a1_075, l111a2_075;
    R F11, F12, F44h;
    uint32_t flags;
    int cubic_c;
};

namespace etile {
constexpr int TJ = 8, TK = 32, NT = TJ * TK;
constexpr int UR = TJ + 4, UC = TK + 4;      // staged u and ids: rows j0-2..j0+TJ+1, columns k0-2..k0+TK+1
constexpr int HJ = TJ + 2, HK = TK + 2;      // cells with gradients: rows j0-1..j0+TJ, columns k0-1..k0+TK
constexpr int GYR = TJ + 3, GZC = TK + 3;    // -y face gradients of rows j0-1..j0+TJ+1; -z of columns k0-1..k0+TK+1
constexpr int FYR = TJ + 1, FZC = TK + 1;    // face stresses: y-faces j0..j0+TJ, z-faces k0..k0+TK
constexpr int kGX = 3 * HJ * HK, kGY = 3 * GYR * HK, kGZ = 3 * HJ * GZC, kD0 = 6 * HJ * HK;
constexpr int kFY = 3 * FYR * TK, kFZ = 3 * TJ * FZC;
constexpr int kRest = 2 * kGX + kGY + kGZ + kD0 + kFY + kFZ;   // reals after the staged planes
// A staged plane is one TMA box per array: rows j0-2..j0+TJ+1 and a column
// range whose first element sits on a 16-byte boundary (k0 is a multiple of
// 32): from k0-2 for FP64 u (36 columns, 288 B), from k0-4 for FP32 u (40
// columns, 160 B), from k0-16 for the one-byte material ids (64 columns).
// UP/IP = row pitch, UO/IO = column of k0-2 in a row.
template <class R> constexpr int UP = is_mixed<R>::value ? TK + 8 : TK + 4;
template <class R> constexpr int UO = is_mixed<R>::value ? 2 : 0;
constexpr int IP = 64, IO = 14;
template <class R> constexpr int kUP = UR * UP<R>;             // one component of one staged plane
template <class R> constexpr int kU = 3 * kUP<R>;
constexpr int kIDS = UR * IP;                                    // bytes of one staged id plane
// byte offsets in the dynamic shared memory (TMA destinations 128-byte aligned)
template <class R> constexpr size_t OFF_ID = (size_t)2 * kU<R> * sizeof(R);
template <class R> constexpr size_t OFF_R = OFF_ID<R> + 2 * (size_t)kIDS;
template <class R> constexpr size_t OFF_I = OFF_R<R> + (size_t)kRest * sizeof(R);
template <class R> constexpr size_t OFF_IDC = OFF_I<R> + (size_t)(2 * UR + UC) * sizeof(int);
template <class R> constexpr size_t OFF_BAR = (OFF_IDC<R> + HJ * HK + 7) / 8 * 8;
template <class R> constexpr size_t kFixedBytes = OFF_BAR<R> + 2 * sizeof(unsigned long long);
template <class R>
constexpr size_t kMatOffset = (kFixedBytes<R> + 15) / 16 * 16;
template <class R>
inline size_t smem_bytes(int nmat) { return kMatOffset<R> + (size_t)nmat * sizeof(ElMat<R>); }
static_assert(OFF_ID<double> % 128 == 0 && OFF_ID<float> % 128 == 0, "id planes 128-byte aligned");
static_assert((kUP<double> * sizeof(double)) % 128 == 0 && (kUP<float> * sizeof(float)) % 128 == 0, "u planes 128-byte aligned");
static_assert(kIDS % 128 == 0, "id planes 128-byte aligned");
}  // namespace etile

// Tensor maps of the TMA staging of k_elastic_tile (one 3-D map per u
// component of the stage input and one of the material ids, box = one
// staged plane), the flag a timed-out wait sets, and whether they are usable
// for this run (otherwise every block stages with cp.async).
struct ETileMaps {
    CUtensorMap u[3];
    CUtensorMap id;
    unsigned* err;
    int on;
};

// index x in [-n, 2n) wrapped into [0, n)
__device__ inline int wrapm(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// Rows of the Voigt stress that the divergence uses from a face normal to
// direction d: x-face -> xx, xy, xz; y-face -> xy, yy, yz; z-face -> xz, yz, zz
__host__ __device__ constexpr int face_row(int d, int r) {
    return d == 0 ? (r == 0 ? 0 : (r == 1 ? 5 : 4)) : (d == 1 ? (r == 0 ? 5 : (r == 1 ? 1 : 3)) : (r == 0 ? 4 : (r == 1 ? 3 : 2)));
}

// row r of C * e with the accumulation order of strain2stress_glb
// (mathlib.cpp:127-135); zero entries of the cubic pattern are skipped,
// which leaves every partial sum unchanged.  CUB: every material of the
// run has the cubic pattern.
template <bool CUB, class M, class R>
__device__ inline R stress_row(const M& m, const R e[6], int r) {
    if (CUB || m.cubic_c) {
        if (r < 3) return m.cij[r][0] * e[0] + m.cij[r][1] * e[1] + m.cij[r][2] * e[2];
        return m.cij[r][r] * e[r];
    }
    R acc = R(0.);
#pragma unroll
    for (int q = 0; q < 6; q++) acc = acc + m.cij[r][q] * e[q];
    return acc;
}

// global-frame dynamic eigenstrain of cell c with material constants mt
// (get_eigenstrain_dynamic; eigen_glb with the constants taken from mt)
template <class R, class M>
__device__ inline void eigen_glb_m(const Params& P, const StageIOT<R>& io, long c, const M& mt, R e[6]) {
    R px = R(0.), py = R(0.), pz = R(0.), mx = R(0.), my = R(0.), mz = R(0.);
    if (P.fe) glb2crt(P, io.p_in.c[0][c], io.p_in.c[1][c], io.p_in.c[2][c], px, py, pz);
    if (P.fm) glb2crt(P, io.m_in.c[0][c], io.m_in.c[1][c], io.m_in.c[2][c], mx, my, mz);
    R e0[6] = {R(0.), R(0.), R(0.), R(0.), R(0.), R(0.)};
    if (io.eig0_c[0]) for (int a = 0; a < 6; a++) e0[a] = io.eig0_c[a][c];
    eigen_terms(P, io, c, mt, mx, my, mz, px, py, pz, e0, e);
    if (P.rot) {
        R s[3][3] = {{e[0], e[5], e[4]}, {e[5], e[1], e[3]}, {e[4], e[3], e[2]}}, o[3][3];
        rot_tensor(Tc2g<R>(P), s, o);
        e[0] = o[0][0]; e[1] = o[1][1]; e[2] = o[2][2]; e[3] = o[1][2]; e[4] = o[0][2]; e[5] = o[0][1];
    }
}

// gradients of a cell held in the shared tile: gm(d,a) on the -d face,
// gp(d,a) on the +d face, d0(a) the global-frame eigenstrain
template <class R>
struct TileCell {
    const R *gxm, *gxp, *gy, *gz, *d0s;
    int r, s;
    __device__ R gm(int d, int a) const {
        using namespace etile;
        return d == 0 ? gxm[(a * HJ + r) * HK + s] : (d == 1 ? gy[(a * GYR + r) * HK + s] : gz[(a * HJ + r) * GZC + s]);
    }
    __device__ R gp(int d, int a) const {
        using namespace etile;
        return d == 0 ? gxp[(a * HJ + r) * HK + s] : (d == 1 ? gy[(a * GYR + r + 1) * HK + s] : gz[(a * HJ + r) * GZC + s + 1]);
    }
    __device__ R d0(int a) const { return d0s[(a * etile::HJ + r) * etile::HK + s]; }
};

// the same quantities read from global memory (face gradients recomputed as
// k_face_grad does); used for the k == ny-1 neighbour of the z-face quirk
template <class R>
struct GlobalCell {
    const Params& P;
    const StageIOT<R>& io;
    long i, j, k;
    R d0v[6];
    __device__ GlobalCell(const Params& p, const StageIOT<R>& s, long i_, long j_, long k_) : P(p), io(s), i(i_), j(j_), k(k_) {
        if (P.elasto_back) eigen_glb(P, io, cid(P, i, j, k), d0v); else for (int a = 0; a < 6; a++) d0v[a] = R(0.);
    }
    __device__ R grad(int d, int a, long ci, long cj, long ck) const {
        const R* u = io.u_in.c[a];
        const long c = cid(P, ci, cj, ck);
        if (d == 0) return free_x(P, io.mid, ci, cj, ck) ? R(0.) : qdivR((u[c] - u[cid(P, ci == 0 ? P.nx - 1 : ci - 1, cj, ck)]), P.dx, P.rdx, P.f.rdx);
        if (d == 1) return free_y(P, io.mid, ci, cj, ck) ? R(0.) : qdivR((u[c] - u[cid(P, ci, cj == 0 ? P.ny - 1 : cj - 1, ck)]), P.dy, P.rdy, P.f.rdy);
        return free_z(P, io.mid, ci, cj, ck) ? R(0.) : qdivR((u[c] - u[cid(P, ci, cj, ck == 0 ? P.nz - 1 : ck - 1)]), P.dz, P.rdz, P.f.rdz);
    }
    __device__ R gm(int d, int a) const { return grad(d, a, i, j, k); }
    __device__ R gp(int d, int a) const {
        if (d == 0) return grad(0, a, i == P.nx - 1 ? 0 : i + 1, j, k);
        if (d == 1) return grad(1, a, i, j == P.ny - 1 ? 0 : j + 1, k);
        return grad(2, a, i, j, k == P.nz - 1 ? 0 : k + 1);
    }
    __device__ R d0(int a) const { return d0v[a]; }
};

// One cell's contribution to the stress rows of a face normal to D; ga is
// the face's gradient of the normal displacement component, gb and gc those
// of the two tangential components (x-face: u_z, u_y; y-face: u_z, u_x;
// z-face: u_y, u_x).
template <int D, bool CUB, class V, class M, class R>
__device__ inline void side_rows(const V& v, const M& m, R ga, R gb, R gc, R out[3]) {
    R st[6];
    if (D == 0) {
        st[0] = ga - v.d0(0);
        st[1] = (v.gm(1, 1) + v.gp(1, 1)) / R(2.) - v.d0(1);
        st[2] = (v.gm(2, 2) + v.gp(2, 2)) / R(2.) - v.d0(2);
        st[3] = ((v.gm(2, 1) + v.gp(2, 1) + v.gm(1, 2) + v.gp(1, 2)) / R(4.) - v.d0(3)) * R(2.);
        st[4] = ((v.gm(2, 0) + v.gp(2, 0) + gb * R(2.)) / R(4.) - v.d0(4)) * R(2.);
        st[5] = ((v.gm(1, 0) + v.gp(1, 0) + gc * R(2.)) / R(4.) - v.d0(5)) * R(2.);
    } else if (D == 1) {
        st[0] = (v.gm(0, 0) + v.gp(0, 0)) / R(2.) - v.d0(0);
        st[1] = ga - v.d0(1);
        st[2] = (v.gm(2, 2) + v.gp(2, 2)) / R(2.) - v.d0(2);
        st[3] = ((v.gm(2, 1) + v.gp(2, 1) + gb * R(2.)) / R(4.) - v.d0(3)) * R(2.);
        st[4] = ((v.gm(2, 0) + v.gp(2, 0) + v.gm(0, 2) + v.gp(0, 2)) / R(4.) - v.d0(4)) * R(2.);
        st[5] = ((gc * R(2.) + v.gm(0, 1) + v.gp(0, 1)) / R(4.) - v.d0(5)) * R(2.);
    } else {
        st[0] = (v.gm(0, 0) + v.gp(0, 0)) / R(2.) - v.d0(0);
        st[1] = (v.gm(1, 1) + v.gp(1, 1)) / R(2.) - v.d0(1);
        st[2] = ga - v.d0(2);
        st[3] = ((gb * R(2.) + v.gm(1, 2) + v.gp(1, 2)) / R(4.) - v.d0(3)) * R(2.);
        st[4] = ((gc * R(2.) + v.gm(0, 2) + v.gp(0, 2)) / R(4.) - v.d0(4)) * R(2.);
        st[5] = ((v.gm(1, 0) + v.gp(1, 0) + v.gm(0, 1) + v.gp(0, 1)) / R(4.) - v.d0(5)) * R(2.);
    }
#pragma unroll
    for (int r = 0; r < 3; r++) out[r] = stress_row<CUB>(m, st, face_row(D, r));
}

// Shared-memory plan of k_elastic_tile: every array sits at a compile-time
// offset from the dynamic base (etile::OFF_*); the material table (sized at
// launch) is last.
template <class R>
struct ETileSmem {
    unsigned char* base;
    __device__ R* u(int slot) const { return reinterpret_cast<R*>(base) + slot * etile::kU<R>; }
    __device__ uint8_t* id(int slot) const { return base + etile::OFF_ID<R> + slot * etile::kIDS; }
    __device__ R* rp() const { return reinterpret_cast<R*>(base + etile::OFF_R<R>); }
    __device__ R* gx(int slot) const { return rp() + slot * etile::kGX; }
    __device__ R* gy() const { return rp() + 2 * etile::kGX; }
    __device__ R* gz() const { return gy() + etile::kGY; }
    __device__ R* d0() const { return gz() + etile::kGZ; }
    __device__ R* fy() const { return d0() + etile::kD0; }
    __device__ R* fz() const { return fy() + etile::kFY; }
    __device__ int* ip() const { return reinterpret_cast<int*>(base + etile::OFF_I<R>); }
    __device__ int* rowoff() const { return ip(); }
    __device__ int* rowj() const { return ip() + etile::UR; }
    __device__ int* colk() const { return ip() + 2 * etile::UR; }
    __device__ uint8_t* idc() const { return base + etile::OFF_IDC<R>; }
    __device__ unsigned long long* bar(int slot) const {
        return reinterpret_cast<unsigned long long*>(base + etile::OFF_BAR<R>) + slot;
    }
    __device__ ElMat<R>* mat() const { return reinterpret_cast<ElMat<R>*>(base + etile::kMatOffset<R>); }
};

// Staging of plane pw into ring slot `slot`.  TMA blocks: one thread arms
// the slot's mbarrier with the byte count and issues one tensor copy per u
// component and one for the ids (no wrap-around needed: the block's halo lies
// inside the grid in every periodic direction).  Other blocks: the u copies
// go out as cp.async (no register or stall while they fly), the ids are
// loaded into registers and stored by etile_stage_finish, which also waits
// for the copies.  Both write the same layout.
constexpr int kStageItems = (etile::UR * etile::UC + etile::NT - 1) / etile::NT;
template <class R>
__device__ inline void etile_stage_issue(const Params& P, const StageIOT<R>& io, const ETileSmem<R>& sm, int slot, int pw,
                                         uint8_t idp[kStageItems], bool tma, const ETileMaps& tm, int j0, int k0) {
    using namespace etile;
    if (tma) {
        if (threadIdx.x == 0) {
            unsigned long long* b = sm.bar(slot);
            mbar_arrive_expect_tx(b, (unsigned)(3 * kUP<R> * sizeof(R) + kIDS));
#pragma unroll
            for (int a = 0; a < 3; a++) tma_load_3d(sm.u(slot) + a * kUP<R>, &tm.u[a], k0 - 2 - UO<R>, j0 - 2, pw, b);
            tma_load_3d(sm.id(slot), &tm.id, k0 - 2 - IO, j0 - 2, pw, b);
        }
        return;
    }
    const int po = pw * P.ny * P.nz;
    R* su = sm.u(slot);
#pragma unroll
    for (int t = 0; t < kStageItems; t++) {
        const int it = threadIdx.x + t * NT;
        if (it < UR * UC) {
            const int ur = it / UC, ucol = it - (it / UC) * UC;
            const int c = po + sm.rowoff()[ur] + sm.colk()[ucol];
            idp[t] = io.mid[c];
#pragma unroll
            for (int a = 0; a < 3; a++) cp_async_elem(&su[a * kUP<R> + ur * UP<R> + ucol + UO<R>], &io.u_in.c[a][c]);
        }
    }
    cp_async_commit();
}
template <class R>
__device__ inline void etile_stage_finish(const ETileSmem<R>& sm, int slot, const uint8_t idp[kStageItems], bool tma,
                                          unsigned phase, const ETileMaps& tm) {
    using namespace etile;
    if (tma) {
        // bounded wait: a copy that never lands sets the run's error flag
        // (reported by gf_check_finite) instead of hanging the block
        if (!mbar_wait_bounded(sm.bar(slot), phase, 1u << 24) && tm.err) atomicOr(tm.err, 1u);
        return;
    }
    uint8_t* sid = sm.id(slot);
#pragma unroll
    for (int t = 0; t < kStageItems; t++) {
        const int it = threadIdx.x + t * NT;
        if (it < UR * UC) {
            const int ur = it / UC, ucol = it - (it / UC) * UC;
            sid[ur * IP + ucol + IO] = idp[t];
        }
    }
    cp_async_wait_all();
}

// Resident blocks per SM the register allocation must allow: the FP32 tile
// needs half the shared memory of the FP64 one, so more blocks fit.
#ifndef GF_ETILE_MINB_F32
#define GF_ETILE_MINB_F32 4
#endif
// The tile of block (bx, by, bz): columns k0 = bx TK.., rows j0 = by TJ..,
// x-planes bz chunk..; smem_raw = the block's dynamic shared memory
// (etile::smem_bytes).  k_elastic_tile runs it once per block; the batched
// phase kernels run it on the work items of many engines.
template <int S, bool CUB, class R>
__device__ __forceinline__ void elastic_tile_body(const Params& P, const StageIOT<R>& io, int chunk, int nmat,
                                                  const ETileMaps& tm, int bx, int by, int bz, unsigned char* smem_raw) {
    using namespace etile;
    const ETileSmem<R> sm{smem_raw};

    const int tid = threadIdx.x;
    const int k0 = bx * TK, j0 = by * TJ;
    const int i0 = bz * chunk;
    const int i1 = min(i0 + chunk, P.nx) - 1;            // last plane of the chunk
    const int L = i1 - i0 + 1;
    const int jl = tid / TK, kl = tid - (tid / TK) * TK;
    const int j = j0 + jl, k = k0 + kl;
    const bool valid = (j < P.ny) && (k < P.nz);
    const int r = jl + 1, s = kl + 1;                    // own cell in halo coordinates
    const bool back = P.elasto_back;
    const bool want_strain = io.strain_c[0] != nullptr;
    const bool quirk = valid && (k == P.ny - 1) && (P.ny < P.nz);
    const bool traction_here = P.strain_pulse && P.strain_type == 3 && k == (int)P.source_z;
    const int nyz = P.ny * P.nz;
    // TMA staging when the staged box needs no wrap-around: its rows and
    // columns lie inside the grid in the periodic directions (in the others
    // the values outside are never used: those faces are stress-free)
    const bool tma = tm.on && !(P.per_y && (j0 - 2 < 0 || j0 + TJ + 1 > P.ny - 1))
                     && !(P.per_z && (k0 - 2 < 0 || k0 + TK + 1 > P.nz - 1));
    unsigned phase[2] = {0u, 0u};

    // ---- block set-up: material table, wrapped row/column offsets, barriers, first two planes ----
    if (tid == 0) {
        mbar_init(sm.bar(0), 1);
        mbar_init(sm.bar(1), 1);
        mbar_fence_init();
    }
    for (int it = tid; it < nmat; it += blockDim.x) {
        const DevMatT<R>& d = io.mats[it];
        ElMat<R>& e = sm.mat()[it];
        for (int a = 0; a < 6; a++) for (int b = 0; b < 6; b++) e.cij[a][b] = d.cij[a][b];
        e.dens_dt = d.dens_dt; e.mass_damp = d.mass_damp; e.stiff_damp = d.stiff_damp;
        e.l100_15 = d.l100_15; e.l111_15 = d.l111_15; e.Q11 = d.Q11; e.Q12 = d.Q12; e.Q44 = d.Q44;
        e.l100a1_075 = d.l100a1_075; e.l100a2_075 = d.l100a2_075; e.l111a1_075 = d.l111a1_075; e.l111a2_075 = d.l111a2_075;
        e.F11 = d.F11; e.F12 = d.F12; e.F44h = d.F44h;
        e.flags = d.flags; e.cubic_c = d.cubic_c;
    }
    for (int it = tid; it < UR; it += blockDim.x) {
        int jj = j0 - 2 + it;
        jj = jj < 0 ? jj + P.ny : jj % P.ny;
        sm.rowj()[it] = jj; sm.rowoff()[it] = jj * P.nz;
    }
    for (int it = tid; it < UC; it += blockDim.x) {
        int kk = k0 - 2 + it;
        sm.colk()[it] = kk < 0 ? kk + P.nz : kk % P.nz;
    }
    __syncthreads();
    {
        uint8_t id0[kStageItems], id1[kStageItems];
        etile_stage_issue(P, io, sm, 0, wrapm(i0 - 1, P.nx), id0, tma, tm, j0, k0);
        etile_stage_issue(P, io, sm, 1, wrapm(i0, P.nx), id1, tma, tm, j0, k0);
        etile_stage_finish(sm, 0, id0, tma, phase[0], tm);
        etile_stage_finish(sm, 1, id1, tma, phase[1], tm);
        phase[0] ^= 1u; phase[1] ^= 1u;
    }
    __syncthreads();
    uint8_t idp[kStageItems];          // ids of the plane being staged

    R sa[3] = {R(0.), R(0.), R(0.)};       // lower cell's half of the next x-face stress
    R sxp[3] = {R(0.), R(0.), R(0.)};      // stress on the previous x-face
    R ty[3] = {R(0.), R(0.), R(0.)}, tz[3] = {R(0.), R(0.), R(0.)};
    uint8_t mid_prev = 0;

    for (int q = 0; q <= L + 1; q++) {
        const int p = i0 - 1 + q;                        // plane of this pass
        const int pw = wrapm(p, P.nx);
        const int po = pw * nyz;
        const int cur = q & 1, nxt = cur ^ 1;           // ring slots of planes p and p+1
        const R* uc = sm.u(cur);
        const R* un = sm.u(nxt);
        const uint8_t* ic = sm.id(cur);
        const uint8_t* in = sm.id(nxt);
        R* gxc = sm.gx(cur ^ 1);                    // face p   (computed in the previous pass)
        R* gxn = sm.gx(cur);                        // face p+1
        // ---- A: gradients and eigenstrains of plane p ----
        // four item lists: x-face gradients of face p+1, y- and z-face
        // gradients, the ids and eigenstrains of the plane's cells
        const int f = p + 1;
        const bool fb = (f == 0 || f == P.nx) && !P.per_x;
        auto a_gx = [&](int it) {
            const int rr = it / HK, ss = it - (it / HK) * HK;
            const int uu = (rr + 1) * UP<R> + ss + 1 + UO<R>, ii = (rr + 1) * IP + ss + 1 + IO;
            const bool fr = fb || !(ic[ii] != 0 && in[ii] != 0);
#pragma unroll
            for (int a = 0; a < 3; a++)
                gxn[a * HJ * HK + it] = fr ? R(0.) : qdivR((un[a * kUP<R> + uu] - uc[a * kUP<R> + uu]), P.dx, P.rdx, P.f.rdx);
        };
        auto a_gy = [&](int it) {
            const int rr = it / HK, ss = it - (it / HK) * HK;
            const int u1 = (rr + 1) * UP<R> + ss + 1 + UO<R>, u0 = u1 - UP<R>;
            const int i1 = (rr + 1) * IP + ss + 1 + IO, i0_ = i1 - IP;
            const bool fr = (sm.rowj()[rr + 1] == 0 && !P.per_y) || !(ic[i0_] != 0 && ic[i1] != 0);
#pragma unroll
            for (int a = 0; a < 3; a++)
                sm.gy()[a * GYR * HK + it] = fr ? R(0.) : qdivR((uc[a * kUP<R> + u1] - uc[a * kUP<R> + u0]), P.dy, P.rdy, P.f.rdy);
        };
        auto a_gz = [&](int it) {
            const int rr = it / GZC, ss = it - (it / GZC) * GZC;
            const int u1 = (rr + 1) * UP<R> + ss + 1 + UO<R>, u0 = u1 - 1;
            const int i1 = (rr + 1) * IP + ss + 1 + IO, i0_ = i1 - 1;
            const bool fr = (sm.colk()[ss + 1] == 0 && !P.per_z) || !(ic[i0_] != 0 && ic[i1] != 0);
#pragma unroll
            for (int a = 0; a < 3; a++)
                sm.gz()[a * HJ * GZC + it] = fr ? R(0.) : qdivR((uc[a * kUP<R> + u1] - uc[a * kUP<R> + u0]), P.dz, P.rdz, P.f.rdz);
        };
        auto a_d0 = [&](int it) {
            const int rr = it / HK, ss = it - (it / HK) * HK;
            const uint8_t id = ic[(rr + 1) * IP + ss + 1 + IO];
            sm.idc()[it] = id;
            R e[6] = {R(0.), R(0.), R(0.), R(0.), R(0.), R(0.)};
            if (back && id != 0) eigen_glb_m(P, io, (long)po + sm.rowoff()[rr + 1] + sm.colk()[ss + 1], sm.mat()[id - 1], e);
#pragma unroll
            for (int a = 0; a < 6; a++) sm.d0()[a * HJ * HK + it] = e[a];
        };
        if constexpr (is_mixed<R>::value) {
            // FP32: one pass over the four lists back to back, so that the
            // partial last round of a list does not idle the block and the
            // eigenstrains' global loads overlap the gradient arithmetic
            // (0.521 against 0.535 ms per step on the 128^3 ferroelectric
            // workload; the FP64 tile measured slower that way, 1.040 and
            // 1.092 with each list padded to whole rounds, against 1.033)
            const int n0 = (q <= L) ? HJ * HK : 0, n1 = n0 + GYR * HK, n2 = n1 + HJ * GZC, n3 = n2 + HJ * HK;
            for (int it = tid; it < n3; it += blockDim.x) {
                if (it < n0) a_gx(it);
                else if (it < n1) a_gy(it - n0);
                else if (it < n2) a_gz(it - n1);
                else a_d0(it - n2);
            }
        } else {
            if (q <= L)
                for (int it = tid; it < HJ * HK; it += blockDim.x) a_gx(it);
            for (int it = tid; it < GYR * HK; it += blockDim.x) a_gy(it);
            for (int it = tid; it < HJ * GZC; it += blockDim.x) a_gz(it);
            for (int it = tid; it < HJ * HK; it += blockDim.x) a_d0(it);
        }
        __syncthreads();

        // ---- B1: y- and z-face stresses of the interior plane p; stage plane p+2 ----
        const bool stage_next = q + 1 <= L;
        if (stage_next) etile_stage_issue(P, io, sm, cur, wrapm(p + 2, P.nx), idp, tma, tm, j0, k0);
        if (q >= 1 && q <= L) {
            for (int it = tid; it < FYR * TK + TJ * FZC; it += blockDim.x) {
              if (it < FYR * TK) {
                const int fr_ = it / TK, fc = it - (it / TK) * TK;       // face j0+fr_, column k0+fc
                const int f = j0 + fr_;
                const uint8_t ia = sm.idc()[fr_ * HK + fc + 1], ib = sm.idc()[(fr_ + 1) * HK + fc + 1];
                R o[3] = {R(0.), R(0.), R(0.)};
                if (!(((f == 0 || f == P.ny) && !P.per_y) || !(ia != 0 && ib != 0))) {
                    const int g = (fr_ + 1) * HK + fc + 1;
                    const R ga = sm.gy()[1 * GYR * HK + g], gb = sm.gy()[2 * GYR * HK + g], gc = sm.gy()[g];
                    const TileCell<R> lo{gxc, gxn, sm.gy(), sm.gz(), sm.d0(), fr_, fc + 1};
                    const TileCell<R> hi{gxc, gxn, sm.gy(), sm.gz(), sm.d0(), fr_ + 1, fc + 1};
                    R a1[3], a2[3];
                    side_rows<1, CUB>(lo, sm.mat()[ia - 1], ga, gb, gc, a1);
                    side_rows<1, CUB>(hi, sm.mat()[ib - 1], ga, gb, gc, a2);
#pragma unroll
                    for (int a = 0; a < 3; a++) o[a] = (a1[a] + a2[a]) / R(2.);
                }
#pragma unroll
                for (int a = 0; a < 3; a++) sm.fy()[a * FYR * TK + it] = o[a];
              } else {
                const int iz = it - FYR * TK;
                const int rl = iz / FZC, fc = iz - (iz / FZC) * FZC;      // row j0+rl, face k0+fc
                const int f = k0 + fc;
                const int rr = rl + 1;
                const uint8_t ia = sm.idc()[rr * HK + fc], ib = sm.idc()[rr * HK + fc + 1];
                R o[3] = {R(0.), R(0.), R(0.)};
                if (!(((f == 0 || f == P.nz) && !P.per_z) || !(ia != 0 && ib != 0))) {
                    const int g = rr * GZC + fc + 1;
                    const R ga = sm.gz()[2 * HJ * GZC + g], gb = sm.gz()[1 * HJ * GZC + g], gc = sm.gz()[g];
                    const TileCell<R> lo{gxc, gxn, sm.gy(), sm.gz(), sm.d0(), rr, fc};
                    const TileCell<R> hi{gxc, gxn, sm.gy(), sm.gz(), sm.d0(), rr, fc + 1};
                    R a1[3], a2[3];
                    side_rows<2, CUB>(lo, sm.mat()[ia - 1], ga, gb, gc, a1);
                    side_rows<2, CUB>(hi, sm.mat()[ib - 1], ga, gb, gc, a2);
#pragma unroll
                    for (int a = 0; a < 3; a++) o[a] = (a1[a] + a2[a]) / R(2.);
                }
#pragma unroll
                for (int a = 0; a < 3; a++) sm.fz()[a * TJ * FZC + iz] = o[a];
              }
            }
        }
        __syncthreads();

        // ---- B2: one column per thread ----
        if (valid) {
            const TileCell<R> me{gxc, gxn, sm.gy(), sm.gz(), sm.d0(), r, s};
            const uint8_t id = sm.idc()[r * HK + s];
            // x-face p: between planes p-1 and p
            if (q >= 1) {
                R sx[3] = {R(0.), R(0.), R(0.)};
                const bool fr = ((p == 0 || p == P.nx) && !P.per_x) || !(mid_prev != 0 && id != 0);
                if (!fr) {
                    const int g = r * HK + s;
                    const R ga = gxc[g], gb = gxc[2 * HJ * HK + g], gc = gxc[HJ * HK + g];
                    R sb[3];
                    side_rows<0, CUB>(me, sm.mat()[id - 1], ga, gb, gc, sb);
#pragma unroll
                    for (int a = 0; a < 3; a++) sx[a] = (sa[a] + sb[a]) / R(2.);
                }
                if (q >= 2 && mid_prev != 0) {
                    // cell (p-1, j, k) is complete: its stress divergence
                    const long c = (long)(p - 1) * nyz + (long)j * P.nz + k;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const R tx = qdivR((sx[a] - sxp[a]), P.dx, P.rdx, P.f.rdx);
                        io.force.c[a][c] = tx + ty[a] + tz[a];
                    }
                }
#pragma unroll
                for (int a = 0; a < 3; a++) sxp[a] = sx[a];
            }
            if (q >= 1 && q <= L) {
                if (id != 0) {
                    R s1[3], s2[3];
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        s1[a] = sm.fy()[(a * FYR + jl) * TK + kl];
                        s2[a] = sm.fy()[(a * FYR + jl + 1) * TK + kl];
                    }
#pragma unroll
                    for (int a = 0; a < 3; a++) ty[a] = qdivR((s2[a] - s1[a]), P.dy, P.rdy, P.f.rdy);
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        s1[a] = sm.fz()[(a * TJ + jl) * FZC + kl];
                        s2[a] = sm.fz()[(a * TJ + jl) * FZC + kl + 1];
                    }
                    if (traction_here || quirk) {
                        const uint8_t iu = sm.idc()[r * HK + s + 1];
                        const bool top_free = ((k + 1 == P.nz) && !P.per_z) || !(id != 0 && iu != 0);
                        if (top_free && traction_here) {
                            // surface traction: x -> xz, y -> yz, z -> zz
                            const R tr = stage_drive(io, S).traction;
                            s2[0] = s2[1] = s2[2] = R(0.);
                            if (P.strain_comp == 0) s2[0] = tr; else if (P.strain_comp == 1) s2[1] = tr; else s2[2] = tr;
                        } else if (!top_free && quirk) {
                            // the reference's +z neighbour of k == ny-1 is k = 0
                            // (elastic_dynamic_solver.cpp:1247); creation rejects
                            // decks where that cell is vacuum
                            const int g = r * GZC + s + 1;
                            const R ga = sm.gz()[2 * HJ * GZC + g], gb = sm.gz()[1 * HJ * GZC + g], gc = sm.gz()[g];
                            const GlobalCell<R> nb(P, io, pw, j, 0);
                            R a1[3], a2[3];
                            side_rows<2, CUB>(me, sm.mat()[id - 1], ga, gb, gc, a1);
                            side_rows<2, CUB>(nb, sm.mat()[io.mid[(long)po + (long)j * P.nz] - 1], ga, gb, gc, a2);
#pragma unroll
                            for (int a = 0; a < 3; a++) s2[a] = (a1[a] + a2[a]) / R(2.);
                        }
                    }
#pragma unroll
                    for (int a = 0; a < 3; a++) tz[a] = qdivR((s2[a] - s1[a]), P.dz, P.rdz, P.f.rdz);
                    // cell strain for the magnetic kernels and, in the FP64 form,
                    // the TDGL kernel (the mixed form's TDGL kernel forms its own
                    // from u: fewer bytes, and its FP32 registers hold the stencil)
                    if (want_strain && (sm.mat()[id - 1].flags & (MF_FM | MF_AFM | (is_mixed<R>::value ? 0u : MF_FE)))) {
                        R e[6];
                        e[0] = (me.gm(0, 0) + me.gp(0, 0)) / R(2.);
                        e[1] = (me.gm(1, 1) + me.gp(1, 1)) / R(2.);
                        e[2] = (me.gm(2, 2) + me.gp(2, 2)) / R(2.);
                        e[3] = (me.gm(2, 1) + me.gp(2, 1) + me.gm(1, 2) + me.gp(1, 2)) / R(4.);
                        e[4] = (me.gm(2, 0) + me.gp(2, 0) + me.gm(0, 2) + me.gp(0, 2)) / R(4.);
                        e[5] = (me.gm(1, 0) + me.gp(1, 0) + me.gm(0, 1) + me.gp(0, 1)) / R(4.);
                        if (P.rot) {
                            R t3[3][3] = {{e[0], e[5], e[4]}, {e[5], e[1], e[3]}, {e[4], e[3], e[2]}}, o3[3][3];
                            rot_tensor(Tg2c<R>(P), t3, o3);
                            e[0] = o3[0][0]; e[1] = o3[1][1]; e[2] = o3[2][2]; e[3] = o3[1][2]; e[4] = o3[0][2]; e[5] = o3[0][1];
                        }
                        const long c = (long)po + (long)j * P.nz + k;
#pragma unroll
                        for (int a = 0; a < 6; a++) io.strain_c[a][c] = e[a];
                    }
                } else {
#pragma unroll
                    for (int a = 0; a < 3; a++) ty[a] = tz[a] = R(0.);
                }
            }
            // lower cell's half of x-face p+1
            if (q <= L && id != 0) {
                const int g = r * HK + s;
                const R ga = gxn[g], gb = gxn[2 * HJ * HK + g], gc = gxn[HJ * HK + g];
                side_rows<0, CUB>(me, sm.mat()[id - 1], ga, gb, gc, sa);
            }
            mid_prev = id;
        }
        if (stage_next) {
            etile_stage_finish(sm, cur, idp, tma, phase[cur], tm);
            phase[cur] ^= 1u;
        }
        __syncthreads();
    }
}

template <int S, bool CUB, class R = double>
__global__ void __launch_bounds__(etile::NT, is_mixed<R>::value ? GF_ETILE_MINB_F32 : 2) k_elastic_tile(Params P, StageIOT<R> io, int chunk, int nmat,
                                                                                        const __grid_constant__ ETileMaps tm) {
    GF_EXTERN_SMEM(unsigned char, smem_raw);
    elastic_tile_body<S, CUB, R>(P, io, chunk, nmat, tm, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// The boundary planes of k_elastic_bc applied inside the RK update
// (Params::el_bc_fused: nz >= 5 and no displacement source on plane 0 or
// nz-1), by the thread of the cell each update reads besides step-start
// values: cell c has formed its new u (uo: the stage output for stages 1-3,
// the new step value for the last, with compensation words ucm in FP32) from
// its step-start value ux.  Mur (abc_1D): the thread of k = 1 (k = nz-2)
// writes the new u of k = 0 (k = nz-1) from its own new value, and the
// returned flag tells the k = 0 (nz-1) thread not to write its own.  Liao:
// the k = 0 thread rewrites its step-start u with the last extrapolation
// (stages 1-3) or replaces its new value with the extrapolation and shifts
// the history (last stage).  Displacement source: the source plane's new
// value is replaced (after the Mur update has read it, as k_elastic_bc
// orders them).  Every other read is of step-start values or history,
// which this launch does not write.
template <int S, class R>
__device__ inline bool rk_bc_fused(const Params& P, const StageIOT<R>& io, int c, const R ux[3], R uo[3], R ucm[3]) {
    const int nz = P.nz;
    const int t = c / nz, k = c - t * nz;
    const long plane = (long)P.nx * P.ny;
    bool skip = false;
    if (P.abc_1D) {
        const bool bot = !P.abc_elast_onlytop;
        if ((k == 0 && bot) || k == nz - 1) skip = true;
        if ((k == 1 && bot) || k == nz - 2) {
            const double* cf = (S == 0 || S == 1) ? P.mur_el_half : P.mur_el_full;
            const int nb = (k == 1) ? c - 1 : c + 1;
            R xn[3];
#pragma unroll
            for (int a = 0; a < 3; a++) xn[a] = io.u_x.c[a][nb];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const R cl = (k == 1) ? R(cf[0]) : R(cf[2]), ct = (k == 1) ? R(cf[1]) : R(cf[3]);
                const R cc = (a == 2) ? cl : ct;
                R* so = (S < 3) ? io.u_out.c[a] : io.u_acc.c[a];
                so[nb] = ux[a] + cc * (xn[a] - uo[a]);
                if constexpr (is_mixed<R>::value) { if (S == 3) io.u_cmp.c[a][nb] = R(0); }
            }
        }
    } else if (k == 0) {
        const R w = P.liao_w;
        if (S < 3) {
            R last[3];
#pragma unroll
            for (int a = 0; a < 3; a++) last[a] = io.liao_last[a * plane + t];
#pragma unroll
            for (int a = 0; a < 3; a++) io.u_x.c[a][c] = last[a];
        } else {
            const R c1 = R(4.) * w + R(2.) * (R(1.) - w), c2 = R(6.) * w + (R(1.) - w), c3 = R(4.) * w;
            const unsigned long long step = *io.step;
            R* slot = io.liao_hist + (size_t)(step & 3ull) * 12 * plane;
            const R* h2 = io.liao_hist + (size_t)((step + 3) & 3ull) * 12 * plane;
            const R* h3 = io.liao_hist + (size_t)((step + 2) & 3ull) * 12 * plane;
            const R* h4 = io.liao_hist + (size_t)((step + 1) & 3ull) * 12 * plane;
            R uv[3][4], t2[3], t3[3], t4[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
#pragma unroll
                for (int p = 1; p <= 4; p++) uv[a][p - 1] = io.u_x.c[a][c + p];
                t2[a] = h2[(a * 4 + 1) * plane + t];
                t3[a] = h3[(a * 4 + 2) * plane + t];
                t4[a] = h4[(a * 4 + 3) * plane + t];
            }
#pragma unroll
            for (int a = 0; a < 3; a++) {
#pragma unroll
                for (int p = 1; p <= 4; p++) slot[(a * 4 + (p - 1)) * plane + t] = uv[a][p - 1];
                const R v = c1 * uv[a][0] - c2 * t2[a] + c3 * t3[a] - w * t4[a];
                uo[a] = v;
                ucm[a] = R(0);
                io.liao_last[a * plane + t] = v;
            }
        }
    }
    if (P.strain_pulse && k == (int)P.source_z) {
        const StageDrive& dr = stage_drive(io, S);
        if (dr.usrc_on && io.mid[c] != 0) {
            uo[P.strain_comp] = R(dr.usrc);
            ucm[P.strain_comp] = R(0);
        }
    }
    return skip;
}

// Per cell after k_elastic_tile: velocity increment from the stress
// divergence f with mass and stiffness damping (get_dv_RK*,
// elastic_dynamic_solver.cpp:1295-1329: weights 1, 2, 2, 1 on f - f_store,
// f_store := f in stage 1 only), then the RK4 combination of v and u.  A
// streaming kernel at full occupancy, so these loads and stores overlap
// across many warps instead of waiting inside the tiled kernel's phases.
// Mixed form: one thread updates two cells 256 apart, and every load of both
// cells is issued before the first store (an FP32 access moves half the bytes
// of an FP64 one, so twice the accesses must be in flight to stream at the
// same rate).  The grid covers 512 cells per block.
template <int S>
struct RkCellF32 {
    float f[3], fs[3], vx[3], vin[3], ux[3], vacc[3], uacc[3], vcmp[3], ucmp[3];
    float dens_dt, mass_damp, stiff_damp;
    uint8_t id;
    __device__ void load(const StageIOT<float>& io, int c) {
        id = io.mid[c];
        if (id != 0) {
            const DevMatT<float>& mt = io.mats[id - 1];
            dens_dt = mt.dens_dt; mass_damp = mt.mass_damp; stiff_damp = mt.stiff_damp;
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            f[a] = io.force.c[a][c]; fs[a] = io.force_store.c[a][c];
            vx[a] = io.v_x.c[a][c]; vin[a] = io.v_in.c[a][c]; ux[a] = io.u_x.c[a][c];
            if (S > 0) { vacc[a] = io.v_acc.c[a][c]; uacc[a] = io.u_acc.c[a][c]; }
            if (S == 3) { vcmp[a] = io.v_cmp.c[a][c]; ucmp[a] = io.u_cmp.c[a][c]; }
        }
    }
    __device__ void update(const Params& P, const StageIOT<float>& io, int c, float dt) const {
        float uo[3], ucn[3];    // new u (stage output, or the new step value and its compensation word)
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float dv = 0.f;
            if (id != 0) {
                const float w = (S == 1 || S == 2) ? 2.f : 1.f;
                dv = f[a] * dens_dt + mass_damp * vx[a] + stiff_damp * (f[a] - fs[a]) * w;
                if (S == 0) io.force_store.c[a][c] = f[a];
            }
            const float du = vin[a] * dt;
            if (S < 3) {
                const float cf = (S == 2) ? 1.f : 0.5f;
                io.v_out.c[a][c] = vx[a] + dv * cf;
                uo[a] = ux[a] + du * cf;
                ucn[a] = 0.f;
                io.v_acc.c[a][c] = (S == 0) ? dv * (1.f / 6.f) : vacc[a] + dv * (1.f / 3.f);
                io.u_acc.c[a][c] = (S == 0) ? du * (1.f / 6.f) : uacc[a] + du * (1.f / 3.f);
            } else {
                float sum, err;
                two_sum(vx[a], (vacc[a] + dv * (1.f / 6.f)) + vcmp[a], sum, err);
                io.v_acc.c[a][c] = sum; io.v_cmp.c[a][c] = err;
                two_sum(ux[a], (uacc[a] + du * (1.f / 6.f)) + ucmp[a], sum, err);
                uo[a] = sum; ucn[a] = err;
            }
        }
        const bool skip = P.el_bc_fused ? rk_bc_fused<S, float>(P, io, c, ux, uo, ucn) : false;
        if (!skip) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (S < 3) io.u_out.c[a][c] = uo[a];
                else { io.u_acc.c[a][c] = uo[a]; io.u_cmp.c[a][c] = ucn[a]; }
            }
        }
    }
};

// block bx of the RK update (256 cells per block in FP64, 512 in FP32)
template <int S, class R>
__device__ __forceinline__ void elastic_rk_body(const Params& P, const StageIOT<R>& io, int bx) {
    if constexpr (is_mixed<R>::value) {
        const int c0 = bx * 512 + threadIdx.x, c1 = c0 + 256;
        RkCellF32<S> a, b;
        if (c0 < P.n) a.load(io, c0);
        if (c1 < P.n) b.load(io, c1);
        if (c0 < P.n) a.update(P, io, c0, P.f.dt);
        if (c1 < P.n) b.update(P, io, c1, P.f.dt);
    } else {
        // FP64: every operand of the three components is loaded before the first
        // store (as RkCellF32 does for two cells), so a thread's ~20 loads are in
        // flight together
        const int c = bx * blockDim.x + threadIdx.x;
        if (c >= P.n) return;
        const uint8_t id = io.mid[c];
        double f[3], fs[3], vx[3], vin[3], ux[3], va[3], ua[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            f[a] = io.force.c[a][c]; fs[a] = io.force_store.c[a][c];
            vx[a] = io.v_x.c[a][c]; vin[a] = io.v_in.c[a][c]; ux[a] = io.u_x.c[a][c];
            va[a] = (S > 0) ? io.v_acc.c[a][c] : 0.;
            ua[a] = (S > 0) ? io.u_acc.c[a][c] : 0.;
        }
        double dv[3] = {0., 0., 0.};
        if (id != 0) {
            const DevMatT<R>& mt = io.mats[id - 1];
            const double dens_dt = mt.dens_dt, mass_damp = mt.mass_damp, stiff_damp = mt.stiff_damp;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (S == 1 || S == 2)
                    dv[a] = f[a] * dens_dt + mass_damp * vx[a] + stiff_damp * (f[a] - fs[a]) * 2.;
                else
                    dv[a] = f[a] * dens_dt + mass_damp * vx[a] + stiff_damp * (f[a] - fs[a]);
                if (S == 0) io.force_store.c[a][c] = f[a];
            }
        }
        double uo[3], ucn[3] = {0., 0., 0.};    // new u: the stage output, or the new step value
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double du = vin[a] * P.dt;
            if (S == 0) {
                io.v_out.c[a][c] = vx[a] + dv[a] * 0.5; io.v_acc.c[a][c] = vx[a] + qdiv(dv[a], 6., kInv6);
                uo[a] = ux[a] + du * 0.5;               io.u_acc.c[a][c] = ux[a] + qdiv(du, 6., kInv6);
            } else if (S == 1) {
                io.v_out.c[a][c] = vx[a] + dv[a] * 0.5; io.v_acc.c[a][c] = va[a] + qdiv(dv[a], 3., kInv3);
                uo[a] = ux[a] + du * 0.5;               io.u_acc.c[a][c] = ua[a] + qdiv(du, 3., kInv3);
            } else if (S == 2) {
                io.v_out.c[a][c] = vx[a] + dv[a];       io.v_acc.c[a][c] = va[a] + qdiv(dv[a], 3., kInv3);
                uo[a] = ux[a] + du;                     io.u_acc.c[a][c] = ua[a] + qdiv(du, 3., kInv3);
            } else {
                io.v_acc.c[a][c] = va[a] + qdiv(dv[a], 6., kInv6);
                uo[a] = ua[a] + qdiv(du, 6., kInv6);
            }
        }
        const bool skip = P.el_bc_fused ? rk_bc_fused<S, double>(P, io, c, ux, uo, ucn) : false;
        if (!skip) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (S < 3) io.u_out.c[a][c] = uo[a];
                else io.u_acc.c[a][c] = uo[a];
            }
        }
    }
}

// FP32: 4 blocks per SM (64 registers; the last stage's update with the
// fused boundary planes spills 8 bytes): 1.322 ms per 128^3 ferroelectric
// step against 1.338 with no bound (77 registers at the last stage, 3
// blocks) and 1.342 at 5 blocks (48 registers, 88 bytes of spills)
#ifndef GF_RK_MINB_F32
#define GF_RK_MINB_F32 4
#endif
template <int S, class R = double>
__global__ void __launch_bounds__(256, is_mixed<R>::value ? GF_RK_MINB_F32 : 1) k_elastic_rk(Params P, StageIOT<R> io) {
    elastic_rk_body<S, R>(P, io, blockIdx.x);
}

// cell strain (global frame) of the current step for output (Dexx_glb ...)
template <class R = double>
__global__ void k_cell_strain(Params P, StageIOT<R> io, double* out6) {
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const long nyz = (long)P.ny * P.nz;
    const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const GradView<R> g(P, io);
    R e[6];
    g.strain_glb(i, j, k, e);
    for (int a = 0; a < 6; a++) out6[(long)a * P.n + c] = e[a];
}

// Boundary planes of u after the stage update, one thread per (i,j).
// For stages 0..2 `tgt` is the stage output (F_glb_store); for the last
// stage it is the new step value and `old` the step-start value (the
// reference's history copy Du?_glb_t1).
template <int S, class R>
__device__ __forceinline__ void elastic_bc_body(const Params& P, const StageIOT<R>& io, int bx) {
    const long t = (long)bx * blockDim.x + threadIdx.x;
    if (t >= (long)P.nx * P.ny) return;
    const long i = t / P.ny, j = t - i * P.ny;
    const long nz = P.nz;
    const long plane = (long)P.nx * P.ny;
    const StageDrive& dr = stage_drive(io, S);
    const unsigned long long step = *io.step;      // 0-based step being finished

    if (!P.abc_1D) {
        // Liao 4th-order extrapolation on k = 0.  History slot h holds planes
        // k=1..4 of u at the start of step h (mod 4).
        const R w = P.liao_w;
        const R c1 = R(4.) * w + R(2.) * (R(1.) - w), c2 = R(6.) * w + (R(1.) - w), c3 = R(4.) * w;
        // every load of a stage is issued before its first store
        if (S < 3) {
            // stages 1-3 rewrite u(k=0) with the value of the last full update
            R last[3];
#pragma unroll
            for (int a = 0; a < 3; a++) last[a] = io.liao_last[a * plane + t];
#pragma unroll
            for (int a = 0; a < 3; a++) io.u_x.c[a][cid(P, i, j, 0)] = last[a];
        } else {
            // shift history: slot (step mod 4) <- planes 1..4 of the step-start u;
            // the extrapolation reads that slot as t1 = u(step), i.e. the
            // values just loaded, and three older slots
            R* slot = io.liao_hist + (size_t)(step & 3ull) * 12 * plane;
            const R* h2 = io.liao_hist + (size_t)((step + 3) & 3ull) * 12 * plane;   // t2 = u(step-1)
            const R* h3 = io.liao_hist + (size_t)((step + 2) & 3ull) * 12 * plane;   // t3 = u(step-2)
            const R* h4 = io.liao_hist + (size_t)((step + 1) & 3ull) * 12 * plane;   // t4 = u(step-3)
            R uv[3][4], t2[3], t3[3], t4[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
#pragma unroll
                for (int p = 1; p <= 4; p++) uv[a][p - 1] = io.u_x.c[a][cid(P, i, j, p)];
                t2[a] = h2[(a * 4 + 1) * plane + t];
                t3[a] = h3[(a * 4 + 2) * plane + t];
                t4[a] = h4[(a * 4 + 3) * plane + t];
            }
#pragma unroll
            for (int a = 0; a < 3; a++) {
#pragma unroll
                for (int p = 1; p <= 4; p++) slot[(a * 4 + (p - 1)) * plane + t] = uv[a][p - 1];
                const R v = c1 * uv[a][0] - c2 * t2[a] + c3 * t3[a] - w * t4[a];
                io.u_acc.c[a][cid(P, i, j, 0)] = v;
                io.liao_last[a * plane + t] = v;
                if constexpr (is_mixed<R>::value) io.u_cmp.c[a][cid(P, i, j, 0)] = R(0);
            }
        }
    } else {
        // first-order Mur on k = 0 (unless only the top is absorbing) and k = nz-1
        const double* cf = (S == 0 || S == 1) ? P.mur_el_half : P.mur_el_full;
        const R cl1 = cf[0], ct1 = cf[1], cll = cf[2], ctl = cf[3];
        const long b0 = cid(P, i, j, 0), b1 = cid(P, i, j, 1), t0 = cid(P, i, j, nz - 1), t1 = cid(P, i, j, nz - 2);
        // the three components' operands are loaded before the first store;
        // with nz <= 2, t1 is b0 and the top update reads the bottom's result
        // (the stage target is u_out for stages 1-3 and the new step value
        // u_acc for the last; the source is the step-start u)
        const bool sep = nz > 2;
        R xb0[3], xb1[3], xt0[3], xt1[3], sb1[3], st1[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const R* x = io.u_x.c[a];
            const R* so = (S < 3) ? io.u_out.c[a] : io.u_acc.c[a];
            xb0[a] = x[b0]; xb1[a] = x[b1]; xt0[a] = x[t0]; xt1[a] = x[t1];
            sb1[a] = so[b1];
            st1[a] = sep ? so[t1] : R(0.);
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const R c1st = (a == 2) ? cl1 : ct1, clast = (a == 2) ? cll : ctl;
            R* so = (S < 3) ? io.u_out.c[a] : io.u_acc.c[a];
            if (!P.abc_elast_onlytop) so[b0] = xb1[a] + c1st * (xb0[a] - sb1[a]);
            so[t0] = xt1[a] + clast * (xt0[a] - (sep ? st1[a] : so[t1]));
            if constexpr (is_mixed<R>::value) {
                if (S == 3) {
                    if (!P.abc_elast_onlytop) io.u_cmp.c[a][b0] = R(0);
                    io.u_cmp.c[a][t0] = R(0);
                }
            }
        }
    }

    // displacement source on plane source_z (types 1 and 2)
    if (P.strain_pulse && dr.usrc_on && io.mid[cid(P, i, j, P.source_z)] != 0) {
        R* tgt = (S < 3) ? io.u_out.c[P.strain_comp] : io.u_acc.c[P.strain_comp];
        tgt[cid(P, i, j, P.source_z)] = dr.usrc;
        if constexpr (is_mixed<R>::value)
            if (S == 3) io.u_cmp.c[P.strain_comp][cid(P, i, j, P.source_z)] = R(0);
    }
}

template <int S, class R = double>
__global__ void k_elastic_bc(Params P, StageIOT<R> io) {
    elastic_bc_body<S, R>(P, io, blockIdx.x);
}

}  // namespace gf
