// Yee-grid Maxwell stage kernels (FP64 parity form; the Yee update, plane
// source and Mur boundary also in the FP32 mixed form).
//
//   k_em_fused<S> one thread per Yee vertex, updating the E edges and H
//                 faces that share its index:
//   E edges:      curl H of the stage state, the
//                 4-cell edge averages of permittivity, conductivity, free
//                 current, polarisation current dP/dt (get_dE_RK{1..4},
//                 EMdynamic_solver.cpp:337-2238) and the RK4 combination of
//                 update_DE_RK*/update_DE (:3588-3777).  Edges on a
//                 non-periodic system boundary get no curl term; the Mur
//                 kernel sets them afterwards.
//   H faces:      curl E and the 2-cell average of
//                 Ms dm/dt of the same stage (get_dH_RK{1..4}, :2239-3476)
//                 with update_DH_RK*/update_DH (:3477-3586).
//   k_em_plane<S> hard plane-wave source on z = planeEM_source_z
//                 (update_planeEM*, :3828-3883).
//   k_em_mur<S,F> first-order Mur on the non-periodic faces of direction F
//                 (EMdynamic_AbsorbingBoundary.cpp:58-874); directions run
//                 x, then y, then z, as in the reference.
//
// The reference keeps the J_f source in three cell arrays rewritten every
// stage; here the box test and the per-stage value are evaluated in-kernel.
#pragma once

#include "gf_state.cuh"

namespace gf {

// per-material constants the Yee updates read, staged in shared memory
template <class R>
struct EmMat {
    R er, cond, Ms, Ms1, Ms2;
    uint32_t flags;
    int pad_;
};

// Material class of an E edge: what the update needs from the four cells
// around it, precomputed on the host in the kernel's order of operations
// (coef = (dt/e0) / ((er1+er2+er3+er4)/4), cond = (s1+s2+s3+s4)/4 over
// material cells, pc = ferroelectric cell count or 1, bit q of mask set when
// cell q is not vacuum).  Edges share few distinct classes, so one byte per
// edge and a table in shared memory replace four material-id loads, twelve
// table reads and a division per edge.
template <class R>
struct EmCls {
    R coef, cond, pc;
    uint32_t mask;
    int pad_;
};
constexpr int kEmMaxCls = 256;

// free current J_f of cell (i,j,k), component a; jf = the stage's amplitude
template <class R>
__device__ inline R jf_cell(const Params& P, const StageIOT<R>& io, R jf, int a, int i, int j, int k) {
    if (!P.jf_on || a != P.jf_comp) return R(0.);
    if (i < P.jf_i0 || i > P.jf_i1 || j < P.jf_j0 || j > P.jf_j1 || k < P.jf_k0 || k > P.jf_k1) return R(0.);
    if (P.jf_type == 1 || P.jf_type == 2) return jf * io.jf_kfac[k];
    return jf;
}

// inverse-spin-Hall current density, component C (0 x, 1 y), of cell
// (ci,cj,ck) (magnetic_system::get_J_ISHE_RK*, magnetic_solver.cpp:231-283):
// coeff_Js coeff_L (m_C dm_z - m_z dm_C, summed over FM and both AFM
// sublattices at the source plane) / dt, with the stage state m and its
// increment dm
template <class R>
__device__ inline R ishe_cell(const Params& P, const StageIOT<R>& io, int C, int ci, int cj, int ck) {
    const int sz = io.ishe_src[ck];
    if (sz < 0) return R(0.);
    const int s = (ci * P.ny + cj) * P.nz + sz;
    R sum = R(0.);
    if (P.fm) sum = io.m_in.c[C][s] * io.dm.c[2][s] - io.m_in.c[2][s] * io.dm.c[C][s];
    if (P.afm) {
        sum = sum + io.a1_in.c[C][s] * io.da1.c[2][s] - io.a1_in.c[2][s] * io.da1.c[C][s];
        sum = sum + io.a2_in.c[C][s] * io.da2.c[2][s] - io.a2_in.c[2][s] * io.da2.c[C][s];
    }
    return qdivR(io.ishe_coef[ck] * sum, P.dt, P.rdt, P.f.rdt);
}

// Cells around an E edge, in the reference's order 1..4, and whether the
// edge lies on a non-periodic boundary (then it keeps its value).
struct EdgeGeom {
    bool bnd;
    int cx[4], cy[4], cz[4];
};

template <int C>
__device__ inline EdgeGeom edge_geom(const Params& P, int i, int j, int k) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    EdgeGeom g;
    g.bnd = false;
    if (C == 0) {
        if ((j == 0 || j == ny) && !P.per_y) g.bnd = true;
        if ((k == 0 || k == nz) && !P.per_z) g.bnd = true;
        const int y1 = (j == 0 || j == ny) ? ny - 1 : j - 1, y3 = (j == 0 || j == ny) ? 0 : j;
        const int z1 = (k == 0 || k == nz) ? nz - 1 : k - 1, z2 = (k == 0 || k == nz) ? 0 : k;
        g.cx[0] = g.cx[1] = g.cx[2] = g.cx[3] = i;
        g.cy[0] = y1; g.cy[1] = y1; g.cy[2] = y3; g.cy[3] = y3;
        g.cz[0] = z1; g.cz[1] = z2; g.cz[2] = z1; g.cz[3] = z2;
    } else if (C == 1) {
        if ((i == 0 || i == nx) && !P.per_x) g.bnd = true;
        if ((k == 0 || k == nz) && !P.per_z) g.bnd = true;
        const int x1 = (i == 0 || i == nx) ? nx - 1 : i - 1, x3 = (i == 0 || i == nx) ? 0 : i;
        const int z1 = (k == 0 || k == nz) ? nz - 1 : k - 1, z2 = (k == 0 || k == nz) ? 0 : k;
        g.cx[0] = x1; g.cx[1] = x1; g.cx[2] = x3; g.cx[3] = x3;
        g.cy[0] = g.cy[1] = g.cy[2] = g.cy[3] = j;
        g.cz[0] = z1; g.cz[1] = z2; g.cz[2] = z1; g.cz[3] = z2;
    } else {
        if ((i == 0 || i == nx) && !P.per_x) g.bnd = true;
        if ((j == 0 || j == ny) && !P.per_y) g.bnd = true;
        const int x1 = (i == 0 || i == nx) ? nx - 1 : i - 1, x3 = (i == 0 || i == nx) ? 0 : i;
        const int y1 = (j == 0 || j == ny) ? ny - 1 : j - 1, y2 = (j == 0 || j == ny) ? 0 : j;
        g.cx[0] = x1; g.cx[1] = x1; g.cx[2] = x3; g.cx[3] = x3;
        g.cy[0] = y1; g.cy[1] = y2; g.cy[2] = y1; g.cy[3] = y2;
        g.cz[0] = g.cz[1] = g.cz[2] = g.cz[3] = k;
    }
    return g;
}

// What a Yee update reads at its own index and from its curl stencil.  The
// fused kernel gathers these for all three E edges (then all three H faces)
// of a thread before any of their stores, so that those loads are in flight
// together instead of one component's round trip after another.
template <class R>
struct YeeIn {
    R c[4];          // curl operands: (c0 - c1) / h_a - (c2 - c3) / h_b
    R x, self, acc, cmp;   // step value, stage value, RK accumulator, compensation
    R dm1, dm2;      // H faces: dm of the two face cells
    int c1, c2;      // H faces: the two face cells
    uint8_t t1, t2;  // E edges: material class (t1); H faces: ids of the two cells
};

// accumulator (stages 1..3) and compensation (mixed form, last stage) of index e
template <int S, class R>
__device__ inline void rk_loads(const R* acc, const R* cmp, int e, YeeIn<R>& L) {
    if (S > 0) L.acc = acc[e];
    if constexpr (is_mixed<R>::value) { if (S == 3) L.cmp = cmp[e]; }
}

template <int S, int C, class R>
__device__ inline void edge_load(const Params& P, const StageIOT<R>& io, const EdgeGeom& g, int i, int j, int k, int e,
                                 YeeIn<R>& L) {
    const int ny = P.ny, nz = P.nz;
    L.x = io.E_x.c[C][e];
    rk_loads<S>(io.E_acc.c[C], io.E_cmp.c[C], e, L);
    if (g.bnd) return;
    L.self = (S == 0) ? L.x : io.E_in.c[C][e];
    if (P.em_cls) L.t1 = io.ecls[C][e];
    const R* Hx = io.H_in.c[0];
    const R* Hy = io.H_in.c[1];
    const R* Hz = io.H_in.c[2];
    if (C == 0) {
        L.c[0] = Hz[(i * ny + g.cy[2]) * (nz + 1) + g.cz[3]]; L.c[1] = Hz[(i * ny + g.cy[0]) * (nz + 1) + g.cz[3]];
        L.c[2] = Hy[(i * (ny + 1) + g.cy[2]) * nz + g.cz[1]]; L.c[3] = Hy[(i * (ny + 1) + g.cy[2]) * nz + g.cz[0]];
    } else if (C == 1) {
        L.c[0] = Hx[(g.cx[2] * ny + j) * nz + g.cz[3]]; L.c[1] = Hx[(g.cx[2] * ny + j) * nz + g.cz[2]];
        L.c[2] = Hz[(g.cx[2] * ny + j) * (nz + 1) + g.cz[1]]; L.c[3] = Hz[(g.cx[0] * ny + j) * (nz + 1) + g.cz[1]];
    } else {
        L.c[0] = Hy[(g.cx[2] * (ny + 1) + g.cy[1]) * nz + k]; L.c[1] = Hy[(g.cx[0] * (ny + 1) + g.cy[1]) * nz + k];
        L.c[2] = Hx[(g.cx[2] * ny + g.cy[1]) * nz + k]; L.c[3] = Hx[(g.cx[2] * ny + g.cy[0]) * nz + k];
    }
}

// curl from the gathered operands; component C's two grid spacings are
// (y, z), (z, x), (x, y)
template <int C, class R>
__device__ inline R yee_curl(const Params& P, const YeeIn<R>& L) {
    if (C == 0) return qdivR(L.c[0] - L.c[1], P.dy, P.rdy, P.f.rdy) - qdivR(L.c[2] - L.c[3], P.dz, P.rdz, P.f.rdz);
    if (C == 1) return qdivR(L.c[0] - L.c[1], P.dz, P.rdz, P.f.rdz) - qdivR(L.c[2] - L.c[3], P.dx, P.rdx, P.f.rdx);
    return qdivR(L.c[0] - L.c[1], P.dx, P.rdx, P.f.rdx) - qdivR(L.c[2] - L.c[3], P.dy, P.rdy, P.f.rdy);
}

template <int S, class R>
__device__ inline void rk_x(const YeeIn<R>& L, R d, R* out, R* acc, R* cmp, int e) {
    const R xv = L.x;
    if constexpr (is_mixed<R>::value) {
        if (S == 0) { out[e] = xv + d * 0.5f; acc[e] = d * (1.f / 6.f); }
        else if (S == 1) { out[e] = xv + d * 0.5f; acc[e] = L.acc + d * (1.f / 3.f); }
        else if (S == 2) { out[e] = xv + d; acc[e] = L.acc + d * (1.f / 3.f); }
        else {
            float sum, err;
            two_sum(xv, (L.acc + d * (1.f / 6.f)) + L.cmp, sum, err);
            acc[e] = sum;
            cmp[e] = err;
        }
    } else {
        if (S == 0) { out[e] = xv + d * 0.5; acc[e] = xv + qdiv(d, 6., kInv6); }
        else if (S == 1) { out[e] = xv + d * 0.5; acc[e] = L.acc + qdiv(d, 3., kInv3); }
        else if (S == 2) { out[e] = xv + d; acc[e] = L.acc + qdiv(d, 3., kInv3); }
        else { acc[e] = L.acc + qdiv(d, 6., kInv6); }
    }
}

// E edge update of component C at edge (i,j,k) (index e in C's array), from
// the gathered values L.
template <int S, int C, class R>
__device__ inline void em_E_edge(const Params& P, const StageIOT<R>& io, const StageDrive& dr, const EmMat<R>* mt,
                                 const EmCls<R>* cls, const EdgeGeom& g, const YeeIn<R>& L, int e) {
    const int ny = P.ny, nz = P.nz;
    R dt_r, dt_e0_r;
    if constexpr (is_mixed<R>::value) { dt_r = P.f.dt; dt_e0_r = P.f.dt_e0; } else { dt_r = P.dt; dt_e0_r = P.dt_e0; }
    const int* cx = g.cx;
    const int* cy = g.cy;
    const int* cz = g.cz;

    R d = R(0.);
    if (!g.bnd) {
        const R curl = yee_curl<C>(P, L);
        R Jf = R(0.), dP = R(0.), er = R(0.), cond = R(0.), pc = R(0.);
        // dP/dt of the four cells, loaded before their ids are known
        R qv[4] = {R(0.), R(0.), R(0.), R(0.)};
        if (P.em_fromP) {
#pragma unroll
            for (int q = 0; q < 4; q++) qv[q] = io.q_in.c[C][(cx[q] * ny + cy[q]) * nz + cz[q]];
        }
        R coef;
        if (P.em_cls) {
            const EmCls<R>& kc = cls[L.t1];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (P.em_fromP && ((kc.mask >> q) & 1u)) dP = dP + qv[q] * dt_r;
                if (P.jf_on) Jf = Jf + jf_cell(P, io, R(dr.jf), C, cx[q], cy[q], cz[q]);
            }
            pc = kc.pc; cond = kc.cond; coef = kc.coef;
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int cc = (cx[q] * ny + cy[q]) * nz + cz[q];
                const uint8_t id = io.mid[cc];
                if (id == 0) {
                    er = er + R(1.);
                } else {
                    const EmMat<R>& m = mt[id - 1];
                    if (P.em_fromP) dP = dP + qv[q] * dt_r;
                    if (m.flags & MF_FE) pc = pc + R(1.);
                    er = er + m.er;
                    cond = cond + m.cond;
                }
                if (P.jf_on) Jf = Jf + jf_cell(P, io, R(dr.jf), C, cx[q], cy[q], cz[q]);
            }
            if (pc < R(0.5)) pc = R(1.);
            er = er / R(4.); cond = cond / R(4.);
            coef = dt_e0_r / er;   // (dt / e0) rounded once on the host, as the reference's left-to-right evaluation
        }
        // without free current (or P sources) the term is +0, and x - (+0)
        // is x in every bit, so it is left out
        R rhs = curl;
        if (P.jf_on) rhs = curl - Jf / R(4.);
        if (P.drude) {
            // Drude current: 4-cell mean of the three poles' stage values
            R Jp = R(0.);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int cc = (cx[q] * ny + cy[q]) * nz + cz[q];
                Jp = Jp + io.jp_in[0].c[C][cc] + io.jp_in[1].c[C][cc] + io.jp_in[2].c[C][cc];
            }
            rhs = rhs - Jp / R(4.);
        }
        if (C < 2 && P.spin) {
            // inverse-spin-Hall current: 4-cell mean, x and y edges only
            R Ji = R(0.);
#pragma unroll
            for (int q = 0; q < 4; q++) Ji = Ji + ishe_cell(P, io, C, cx[q], cy[q], cz[q]);
            rhs = rhs - Ji / R(4.);
        }
        rhs = rhs - cond * L.self;
        if (P.em_fromP) {
            // pc counts the ferroelectric cells (1..4): divisions by 1, 2 and 4 are exact
            if constexpr (is_mixed<R>::value)
                dP = dP * (pc == 3.f ? 1.f / 3.f : (pc == 1.f ? 1.f : (pc == 2.f ? 0.5f : 0.25f)));
            else
                dP = qdiv(dP, pc, pc == 3. ? kInv3 : (pc == 1. ? 1. : (pc == 2. ? 0.5 : 0.25)));
            rhs = rhs - qdivR(dP, P.dt, P.rdt, P.f.rdt);
        }
        d = coef * rhs;
    }
    rk_x<S>(L, d, io.E_out.c[C], io.E_acc.c[C], io.E_cmp.c[C], e);
}

// Gather of an H face: curl operands, step value, accumulators, and the
// ids and dm of the two cells either side of the face.
template <int S, int C, class R>
__device__ inline void face_load(const Params& P, const StageIOT<R>& io, int i, int j, int k, int e, YeeIn<R>& L) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const R* Ex = io.E_in.c[0];
    const R* Ey = io.E_in.c[1];
    const R* Ez = io.E_in.c[2];
    L.x = io.H_x.c[C][e];
    rk_loads<S>(io.H_acc.c[C], io.H_cmp.c[C], e, L);
    int a1x = i, a1y = j, a1z = k, a2x = i, a2y = j, a2z = k;
    if (C == 0) {
        L.c[0] = Ez[(i * (ny + 1) + j + 1) * nz + k]; L.c[1] = Ez[(i * (ny + 1) + j) * nz + k];
        L.c[2] = Ey[(i * ny + j) * (nz + 1) + k + 1]; L.c[3] = Ey[(i * ny + j) * (nz + 1) + k];
        a1x = (i == 0) ? (P.per_x ? nx - 1 : 0) : i - 1;
        a2x = (i == nx) ? (P.per_x ? 0 : nx - 1) : i;
    } else if (C == 1) {
        L.c[0] = Ex[(i * (ny + 1) + j) * (nz + 1) + k + 1]; L.c[1] = Ex[(i * (ny + 1) + j) * (nz + 1) + k];
        L.c[2] = Ez[((i + 1) * (ny + 1) + j) * nz + k]; L.c[3] = Ez[(i * (ny + 1) + j) * nz + k];
        a1y = (j == 0) ? (P.per_y ? ny - 1 : 0) : j - 1;
        a2y = (j == ny) ? (P.per_y ? 0 : ny - 1) : j;
    } else {
        L.c[0] = Ey[((i + 1) * ny + j) * (nz + 1) + k]; L.c[1] = Ey[(i * ny + j) * (nz + 1) + k];
        L.c[2] = Ex[(i * (ny + 1) + j + 1) * (nz + 1) + k]; L.c[3] = Ex[(i * (ny + 1) + j) * (nz + 1) + k];
        a1z = (k == 0) ? (P.per_z ? nz - 1 : 0) : k - 1;
        a2z = (k == nz) ? (P.per_z ? 0 : nz - 1) : k;
    }
    L.c1 = (a1x * ny + a1y) * nz + a1z;
    L.c2 = (a2x * ny + a2y) * nz + a2z;
    L.dm1 = P.em_fromM ? io.dm.c[C][L.c1] : R(0.);
    L.dm2 = P.em_fromM ? io.dm.c[C][L.c2] : R(0.);
    L.t1 = io.mid[L.c1];
    L.t2 = io.mid[L.c2];
}

// H face update of component C (index e in C's array), from the gathered
// values L.
template <int S, int C, class R>
__device__ inline void em_H_face(const Params& P, const StageIOT<R>& io, const EmMat<R>* mt, const YeeIn<R>& L, int e) {
    R mdt_mu0_r;
    if constexpr (is_mixed<R>::value) mdt_mu0_r = P.f.mdt_mu0; else mdt_mu0_r = P.mdt_mu0;
    const R curl = yee_curl<C>(P, L);
    R dM1 = R(0.), dM2 = R(0.), cnt = R(0.);
    // Ms dm + Ms1 dm1 + Ms2 dm2 of each face cell (EMdynamic_solver.cpp:2300-2306)
    if (L.t1 != 0) {
        const EmMat<R>& m = mt[L.t1 - 1];
        if (P.em_fromM) {
            dM1 = L.dm1 * m.Ms;
            if (P.afm) dM1 = dM1 + io.da1.c[C][L.c1] * m.Ms1 + io.da2.c[C][L.c1] * m.Ms2;
        }
        if (m.flags & (MF_FM | MF_AFM)) cnt = cnt + R(1.);
    }
    if (L.t2 != 0) {
        const EmMat<R>& m = mt[L.t2 - 1];
        if (P.em_fromM) {
            dM2 = L.dm2 * m.Ms;
            if (P.afm) dM2 = dM2 + io.da1.c[C][L.c2] * m.Ms1 + io.da2.c[C][L.c2] * m.Ms2;
        }
        if (m.flags & (MF_FM | MF_AFM)) cnt = cnt + R(1.);
    }
    if (cnt < R(0.5)) cnt = R(1.);
    // -dt/mu0 rounded once on the host; cnt is 1 or 2, so the division is exact
    const R dMs = dM1 + dM2;
    const R d = mdt_mu0_r * curl - (cnt == R(2.) ? dMs * R(0.5) : dMs);
    rk_x<S>(L, d, io.H_out.c[C], io.H_acc.c[C], io.H_cmp.c[C], e);
}

// All six Yee components of one stage: thread (i,j,k) on the vertex grid
// (nx+1)(ny+1)(nz+1) updates every E edge and H face with index (i,j,k)
// inside that component's staggered extent.  E reads only the stage H and
// H only the stage E and dm, so the six updates are independent.  The grid
// is (blocks over the (j,k) vertex plane) x (nx+1 planes); the material
// constants are staged in shared memory.
// Blocks per SM of the launch bound: room for the gathered operands of three
// components without spills (FP64: 80 registers, 24 warps per SM; FP32: 64
// registers, 32 warps).  Measured on the 128x128x96 magnetoelastic film
// against 8, 6, 5, 4, 3 and 2: FP64 (3) 0.365 ms per step vs 0.43-0.76, FP32
// (4) 0.253 ms vs 0.26-0.34.
#ifndef GF_EM_MINB_F32
#define GF_EM_MINB_F32 4
#endif
#ifndef GF_EM_MINB_F64
#define GF_EM_MINB_F64 3
#endif
// block (bx, by): 256 vertices of the (j, k) plane bx of vertex plane by;
// mt, cl = the block's shared-memory tables (kMaxMat and kEmMaxCls entries),
// filled here behind a barrier
template <int S, class R>
__device__ __forceinline__ void em_fused_body(const Params& P, const StageIOT<R>& io, int nmat, const EmCls<R>* __restrict__ cls_g,
                                              int ncls, int bx, int by, EmMat<R>* mt, EmCls<R>* cl) {
    for (int q = threadIdx.x; q < nmat; q += blockDim.x) {
        const DevMatT<R>& d = io.mats[q];
        mt[q].er = d.er; mt[q].cond = d.cond; mt[q].Ms = d.Ms; mt[q].Ms1 = d.Ms1; mt[q].Ms2 = d.Ms2; mt[q].flags = d.flags;
    }
    for (int q = threadIdx.x; q < ncls; q += blockDim.x) cl[q] = cls_g[q];
    __syncthreads();
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int t = bx * blockDim.x + threadIdx.x;
    if (t >= (ny + 1) * (nz + 1)) return;
    const int i = by;
    const int j = t / (nz + 1), k = t - (t / (nz + 1)) * (nz + 1);
    const StageDrive& dr = stage_drive(io, S);
    // E edges: gather all three, then update (the stores follow every load)
    {
        const bool on0 = i < nx, on1 = j < ny, on2 = k < nz;
        const int e0 = (i * (ny + 1) + j) * (nz + 1) + k, e1 = (i * ny + j) * (nz + 1) + k, e2 = (i * (ny + 1) + j) * nz + k;
        const EdgeGeom g0 = edge_geom<0>(P, i, j, k), g1 = edge_geom<1>(P, i, j, k), g2 = edge_geom<2>(P, i, j, k);
        YeeIn<R> L0, L1, L2;
        if (on0) edge_load<S, 0, R>(P, io, g0, i, j, k, e0, L0);
        if (on1) edge_load<S, 1, R>(P, io, g1, i, j, k, e1, L1);
        if (on2) edge_load<S, 2, R>(P, io, g2, i, j, k, e2, L2);
        if (on0) em_E_edge<S, 0, R>(P, io, dr, mt, cl, g0, L0, e0);
        if (on1) em_E_edge<S, 1, R>(P, io, dr, mt, cl, g1, L1, e1);
        if (on2) em_E_edge<S, 2, R>(P, io, dr, mt, cl, g2, L2, e2);
    }
    // H faces, the same way
    {
        const bool on0 = j < ny && k < nz, on1 = i < nx && k < nz, on2 = i < nx && j < ny;
        const int e0 = (i * ny + j) * nz + k, e1 = (i * (ny + 1) + j) * nz + k, e2 = (i * ny + j) * (nz + 1) + k;
        YeeIn<R> L0, L1, L2;
        if (on0) face_load<S, 0, R>(P, io, i, j, k, e0, L0);
        if (on1) face_load<S, 1, R>(P, io, i, j, k, e1, L1);
        if (on2) face_load<S, 2, R>(P, io, i, j, k, e2, L2);
        if (on0) em_H_face<S, 0, R>(P, io, mt, L0, e0);
        if (on1) em_H_face<S, 1, R>(P, io, mt, L1, e1);
        if (on2) em_H_face<S, 2, R>(P, io, mt, L2, e2);
    }
}

template <int S, class R = double>
__global__ void __launch_bounds__(256, is_mixed<R>::value ? GF_EM_MINB_F32 : GF_EM_MINB_F64) k_em_fused(Params P, StageIOT<R> io, int nmat,
                                                                                      const EmCls<R>* __restrict__ cls_g, int ncls) {
    __shared__ EmMat<R> mt[kMaxMat];
    __shared__ EmCls<R> cl[kEmMaxCls];
    em_fused_body<S, R>(P, io, nmat, cls_g, ncls, blockIdx.x, blockIdx.y, mt, cl);
}

// Drude polarisation current, per cell: dJp_n = (e0 wp_n^2 E_cell c_n -
// Jp_n / tau_n) dt for the three poles (get_dJp_RK{1..4},
// EMdynamic_solver.cpp:4318-4452) with E_cell the 4-edge mean of the stage E
// (update_DE_cell, :3813-3826), and the RK4 combination of update_Jp_RK*/
// update_Jp (:4454-4524).
template <int S, class R = double>
__global__ void __launch_bounds__(256) k_drude(Params P, StageIOT<R> io) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const uint8_t id = io.mid[c];
    const int nyz = P.ny * P.nz;
    const int i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
    const int ny = P.ny, nz = P.nz;
    R dJ[3][3] = {{R(0.), R(0.), R(0.)}, {R(0.), R(0.), R(0.)}, {R(0.), R(0.), R(0.)}};
    R dt_r;
    if constexpr (is_mixed<R>::value) dt_r = P.f.dt; else dt_r = P.dt;
    if (id != 0) {
        const DevMatT<R>& mt = io.mats[id - 1];
        const int ex = (i * (ny + 1) + j) * (nz + 1) + k;
        const int ey = (i * ny + j) * (nz + 1) + k;
        const int ez = (i * (ny + 1) + j) * nz + k;
        const R* Ex = io.E_in.c[0];
        const R* Ey = io.E_in.c[1];
        const R* Ez = io.E_in.c[2];
        const R Ec[3] = {(Ex[ex] + Ex[ex + nz + 1] + Ex[ex + 1] + Ex[ex + nz + 1 + 1]) / R(4.),
                              (Ey[ey] + Ey[ey + ny * (nz + 1)] + Ey[ey + 1] + Ey[ey + ny * (nz + 1) + 1]) / R(4.),
                              (Ez[ez] + Ez[ez + (ny + 1) * nz] + Ez[ez + nz] + Ez[ez + (ny + 1) * nz + nz]) / R(4.)};
#pragma unroll
        for (int pole = 0; pole < 3; pole++)
#pragma unroll
            for (int a = 0; a < 3; a++)
                dJ[pole][a] = (R(kE0) * mt.wp[pole] * mt.wp[pole] * Ec[a] * mt.comp[pole] - mt.rtau[pole] * io.jp_in[pole].c[a][c]) * dt_r;
    }
    if constexpr (is_mixed<R>::value) {
#pragma unroll
        for (int pole = 0; pole < 3; pole++)
#pragma unroll
            for (int a = 0; a < 3; a++)
                rk_mixed<S>(io.jp_x[pole].c[a][c], dJ[pole][a], io.jp_out[pole].c[a], io.jp_acc[pole].c[a], io.jp_cmp[pole].c[a], c);
    } else {
#pragma unroll
        for (int pole = 0; pole < 3; pole++)
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const double d = dJ[pole][a];
                double* out = io.jp_out[pole].c[a];
                double* acc = io.jp_acc[pole].c[a];
                const double xv = io.jp_x[pole].c[a][c];
                if (S == 0) { out[c] = xv + d * 0.5; acc[c] = xv + qdiv(d, 6., kInv6); }
                else if (S == 1) { out[c] = xv + d * 0.5; acc[c] = acc[c] + qdiv(d, 3., kInv3); }
                else if (S == 2) { out[c] = xv + d; acc[c] = acc[c] + qdiv(d, 3., kInv3); }
                else { acc[c] = acc[c] + qdiv(d, 6., kInv6); }
            }
    }
}

// Perfect electric conductor: E = 0 on every edge with a PEC cell among its
// four cells, edges on non-periodic system faces excepted (DE?_ifPEC,
// EMdynamic_initialize.cpp:160-330), after the Mur update (update_DE_PEC,
// EMdynamic_solver.cpp:4526-4556).  The reference zeroes both the step value
// and the stage value, so stages 1-3 also clear the step-start buffer.
template <class R>
__device__ inline bool pec_cell(const StageIOT<R>& io, int c) {
    const uint8_t id = io.mid[c];
    return id != 0 && (io.mats[id - 1].flags & MF_PEC);
}
template <int S, class R = double>
__global__ void __launch_bounds__(256) k_em_pec(Params P, StageIOT<R> io) {
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (ny + 1) * (nz + 1)) return;
    const int i = blockIdx.y;
    const int j = t / (nz + 1), k = t - (t / (nz + 1)) * (nz + 1);
    for (int C = 0; C < 3; C++) {
        if ((C == 0 && i >= nx) || (C == 1 && j >= ny) || (C == 2 && k >= nz)) continue;
        // the two directions across the edge and their wrapped cell indices
        int lo[3] = {i, j, k}, hi[3] = {i, j, k};
        bool skip = false;
        for (int d = 0; d < 3; d++) {
            if (d == C) continue;
            const int nd = d == 0 ? nx : (d == 1 ? ny : nz);
            const int per = d == 0 ? P.per_x : (d == 1 ? P.per_y : P.per_z);
            const int v = d == 0 ? i : (d == 1 ? j : k);
            if (v == 0 || v == nd) {
                if (!per) { skip = true; break; }
                lo[d] = nd - 1; hi[d] = 0;
            } else { lo[d] = v - 1; hi[d] = v; }
        }
        if (skip) continue;
        bool pec = false;
        for (int q = 0; q < 4; q++) {
            int x[3];
            int bit = 0;
            for (int d = 0; d < 3; d++) {
                if (d == C) { x[d] = d == 0 ? i : (d == 1 ? j : k); continue; }
                x[d] = ((q >> bit) & 1) ? hi[d] : lo[d];
                bit++;
            }
            pec = pec || pec_cell(io, (x[0] * ny + x[1]) * nz + x[2]);
        }
        if (!pec) continue;
        const int e = C == 0 ? (i * (ny + 1) + j) * (nz + 1) + k
                             : (C == 1 ? (i * ny + j) * (nz + 1) + k : (i * (ny + 1) + j) * nz + k);
        if (S < 3) { io.E_out.c[C][e] = R(0.); io.E_x.c[C][e] = R(0.); }
        else io.E_acc.c[C][e] = R(0.);
        if constexpr (is_mixed<R>::value) io.E_cmp.c[C][e] = R(0.);
    }
}

// hard plane-wave source: E on z = plane_z, all three components, i<nx, j<ny
template <int S, class R = double>
__global__ void k_em_plane(Params P, StageIOT<R> io) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)P.nx * P.ny) return;
    const long i = t / P.ny, j = t - i * P.ny;
    const long nx = P.nx, ny = P.ny, nz = P.nz, z = P.plane_z;
    const StageDrive& dr = stage_drive(io, S);
    R* tx = (S < 3) ? io.E_out.c[0] : io.E_acc.c[0];
    R* ty = (S < 3) ? io.E_out.c[1] : io.E_acc.c[1];
    R* tz = (S < 3) ? io.E_out.c[2] : io.E_acc.c[2];
    tx[(i * (ny + 1) + j) * (nz + 1) + z] = dr.plane[0];
    ty[(i * ny + j) * (nz + 1) + z] = dr.plane[1];
    tz[(i * (ny + 1) + j) * nz + z] = dr.plane[2];
    if constexpr (is_mixed<R>::value) {
        if (S == 3) {
            io.E_cmp.c[0][(i * (ny + 1) + j) * (nz + 1) + z] = R(0);
            io.E_cmp.c[1][(i * ny + j) * (nz + 1) + z] = R(0);
            io.E_cmp.c[2][(i * (ny + 1) + j) * nz + z] = R(0);
        }
    }
    (void)nx;
}

// Mur boundary on the two faces normal to direction F (0 x, 1 y, 2 z).
// For S < 3:  out(b) = X(b_in) + c * (X(b) - out(b_in))   (stage store)
// For S = 3:  new(b) = old(b_in) + c * (old(b) - new(b_in))
// where X / old is the step-start value and out / new the value written.
template <int S, int F, class R>
__device__ __forceinline__ void em_mur_body(const Params& P, const StageIOT<R>& io, int bx) {
    const long nx = P.nx, ny = P.ny, nz = P.nz;
    const long t = (long)bx * blockDim.x + threadIdx.x;
    const bool half = (S == 0 || S == 1);
    // two tangential components per face; index range per component
    if (F == 0) {
        // Ey (j<ny, k<=nz) then Ez (j<=ny, k<nz) at i = 0 and i = nx
        const R cfx = half ? P.c_x_half : P.c_x;
        const long n1 = ny * (nz + 1), n2 = (ny + 1) * nz;
        if (t >= n1 + n2) return;
        const int comp = (t < n1) ? 1 : 2;
        const long r = (t < n1) ? t : t - n1;
        long e0, e1, eN, eN1;   // b=0, b_in=1, b=nx, b_in=nx-1
        if (comp == 1) {
            const long j = r / (nz + 1), k = r - j * (nz + 1);
            e0 = (0 * ny + j) * (nz + 1) + k; e1 = (1 * ny + j) * (nz + 1) + k;
            eN = (nx * ny + j) * (nz + 1) + k; eN1 = ((nx - 1) * ny + j) * (nz + 1) + k;
        } else {
            const long j = r / nz, k = r - j * nz;
            e0 = (0 * (ny + 1) + j) * nz + k; e1 = (1 * (ny + 1) + j) * nz + k;
            eN = (nx * (ny + 1) + j) * nz + k; eN1 = ((nx - 1) * (ny + 1) + j) * nz + k;
        }
        const R* X = io.E_x.c[comp];
        R* O = (S < 3) ? io.E_out.c[comp] : io.E_acc.c[comp];
        if (!P.pec_xy) {
            // both faces' operands before the first store; with one cell
            // across, eN1 is e0 and the second update reads the first's result
            const R x1 = X[e1], x0 = X[e0], o1 = O[e1], xN1 = X[eN1], xN = X[eN];
            const R oN1 = (nx > 1) ? O[eN1] : R(0.);
            O[e0] = x1 + cfx * (x0 - o1);
            O[eN] = xN1 + cfx * (xN - ((nx > 1) ? oN1 : O[eN1]));
        } else { O[e0] = R(0.); O[eN] = R(0.); }
        if constexpr (is_mixed<R>::value) if (S == 3) { io.E_cmp.c[comp][e0] = R(0); io.E_cmp.c[comp][eN] = R(0); }
    } else if (F == 1) {
        // Ex (i<nx, k<=nz) then Ez (i<=nx, k<nz) at j = 0 and j = ny
        const R cfy = half ? P.c_y_half : P.c_y;
        const long n1 = nx * (nz + 1), n2 = (nx + 1) * nz;
        if (t >= n1 + n2) return;
        const int comp = (t < n1) ? 0 : 2;
        const long r = (t < n1) ? t : t - n1;
        long e0, e1, eN, eN1;
        if (comp == 0) {
            const long i = r / (nz + 1), k = r - i * (nz + 1);
            e0 = (i * (ny + 1) + 0) * (nz + 1) + k; e1 = (i * (ny + 1) + 1) * (nz + 1) + k;
            eN = (i * (ny + 1) + ny) * (nz + 1) + k; eN1 = (i * (ny + 1) + ny - 1) * (nz + 1) + k;
        } else {
            const long i = r / nz, k = r - i * nz;
            e0 = (i * (ny + 1) + 0) * nz + k; e1 = (i * (ny + 1) + 1) * nz + k;
            eN = (i * (ny + 1) + ny) * nz + k; eN1 = (i * (ny + 1) + ny - 1) * nz + k;
        }
        const R* X = io.E_x.c[comp];
        R* O = (S < 3) ? io.E_out.c[comp] : io.E_acc.c[comp];
        if (!P.pec_xy) {
            // both faces' operands before the first store; with one cell
            // across, eN1 is e0 and the second update reads the first's result
            const R x1 = X[e1], x0 = X[e0], o1 = O[e1], xN1 = X[eN1], xN = X[eN];
            const R oN1 = (ny > 1) ? O[eN1] : R(0.);
            O[e0] = x1 + cfy * (x0 - o1);
            O[eN] = xN1 + cfy * (xN - ((ny > 1) ? oN1 : O[eN1]));
        } else { O[e0] = R(0.); O[eN] = R(0.); }
        if constexpr (is_mixed<R>::value) if (S == 3) { io.E_cmp.c[comp][e0] = R(0); io.E_cmp.c[comp][eN] = R(0); }
    } else {
        // Ex (i<nx, j<=ny) then Ey (i<=nx, j<ny) at k = 0 and k = nz
        const R ctop = half ? P.c_top_half : P.c_top, cbot = half ? P.c_bot_half : P.c_bot;
        const long n1 = nx * (ny + 1), n2 = (nx + 1) * ny;
        if (t >= n1 + n2) return;
        const int comp = (t < n1) ? 0 : 1;
        const long r = (t < n1) ? t : t - n1;
        long base;
        if (comp == 0) { const long i = r / (ny + 1), j = r - i * (ny + 1); base = (i * (ny + 1) + j) * (nz + 1); }
        else { const long i = r / ny, j = r - i * ny; base = (i * ny + j) * (nz + 1); }
        const long e0 = base, e1 = base + 1, eN = base + nz, eN1 = base + nz - 1;
        const R* X = io.E_x.c[comp];
        R* O = (S < 3) ? io.E_out.c[comp] : io.E_acc.c[comp];
        if (!P.pec_z) {
            // both faces' operands before the first store; with one cell
            // across, e1 is eN and the bottom update reads the top's result
            const R xN1 = X[eN1], xN = X[eN], oN1 = O[eN1], x1 = X[e1], x0 = X[e0];
            const R o1 = (nz > 1) ? O[e1] : R(0.);
            O[eN] = xN1 + ctop * (xN - oN1);
            if (!P.abc_1D || !P.abc_em_onlytop) O[e0] = x1 + cbot * (x0 - ((nz > 1) ? o1 : O[e1]));
            else O[e0] = R(0.);
        } else { O[e0] = R(0.); O[eN] = R(0.); }
        if constexpr (is_mixed<R>::value) if (S == 3) { io.E_cmp.c[comp][e0] = R(0); io.E_cmp.c[comp][eN] = R(0); }
    }
}

template <int S, int F, class R = double>
__global__ void k_em_mur(Params P, StageIOT<R> io) {
    em_mur_body<S, F, R>(P, io, blockIdx.x);
}

}  // namespace gf
