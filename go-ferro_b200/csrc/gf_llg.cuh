// Ferromagnetic LLG stage kernel (FP64 parity form and FP32 mixed form).
//
// One thread per cell.  For every ferromagnetic cell it evaluates the
// effective field and the LLG increment exactly as magnetic_system::
// get_dm_RK{1..4} (magnetic_solver.cpp:3-229) does — anisotropy, magneto-
// elastic, harmonic-mean exchange with the interface slopes of
// get_m_spatial_derivative_local (magnetic_solver.cpp:1638-1831), interfacial
// DMI, static, external, non-uniform external and Maxwell back-action field —
// and applies the RK4 combination of update_m_RK{1,2,3} / get_dm / update_m
// (magnetic_solver.cpp:1448-1458, 1515-1636) in the same pass.
//
// The reference reads six precomputed exchange-coefficient arrays Aij_* and
// three interface-mask arrays per stage (magnetic_initialize.cpp:136-524);
// here both are derived from the one-byte material ids of the cell and its
// six neighbours and a per-pair harmonic-mean table, which removes ~60 bytes
// of reads per cell and stage.
#pragma once

#include "gf_elastic.cuh"

namespace gf {

template <class R>
struct LLGTablesT {
    R Aij[kMaxMat + 1][kMaxMat + 1];   // 2*A1*A2/(A1+A2) for ids (1-based)
    R AijA[2][kMaxMat + 1][kMaxMat + 1];   // the same for the AFM sublattice exchange constants
};
using LLGTables = LLGTablesT<double>;

__device__ inline bool is_fm(const DevMat* mats, uint8_t id) {
    return id != 0 && (mats[id - 1].flags & MF_FM);
}

// static strain plus the cell strain of the stage displacement, crystal
// frame (exxt0_crt + Dexx_crt, magnetic_solver.cpp:89-96); the dynamic part
// is written by k_elastic_tile earlier in the same stage
template <class R>
__device__ inline void cell_strain_total(const Params& P, const StageIOT<R>& io, long i, long j, long k, long c, R e[6]) {
    R d[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
    if (P.elastic) for (int a = 0; a < 6; a++) d[a] = io.strain_c[a][c];
    for (int a = 0; a < 6; a++) {
        R t = io.eps0_c[a] ? io.eps0_c[a][c] : R(0);
        e[a] = t + d[a];
    }
}

// per-material LLG constants, staged in shared memory
template <class R>
struct LLGMat {
    R Aex, dA, ex_coef, dmi_coef, K1c, K2c, B1c, B2c, precess, alpha_precess, Ms;
    int aniso;
    uint32_t fm;
};

// One thread per cell of the ferromagnetic bounding box; cells outside it
// hold their initial m in all four buffers and are never touched.  Grid:
// (blocks over the box's (j,k) plane) x (box planes in i).  R = float is the
// mixed form: FP32 stencil, compensated step value, |m| = 1 after every stage.
#ifndef GF_LLG_MINB_F32
#define GF_LLG_MINB_F32 4
#endif
#ifndef GF_LLG_MINB_F64
#define GF_LLG_MINB_F64 4
#endif
template <int S, class R = double>
// (256, 4): 64 registers, 32 resident warps per SM for its neighbour-load
// latency; measured faster than 98 registers at 16 warps despite a few spills
// (with the RK operands gathered before the first store, on the 128x128x96
// magnetoelastic film: FP64 0.225 ms per step at 4 blocks, 0.238 at 3, 0.285
// at 2; FP32 0.145 at 4)
__global__ void __launch_bounds__(256, is_mixed<R>::value ? GF_LLG_MINB_F32 : GF_LLG_MINB_F64) k_llg_fm(Params P, StageIOT<R> io, const LLGTablesT<R>* __restrict__ tab, int nmat) {
    __shared__ LLGMat<R> mt[kMaxMat];
    __shared__ R sA[kMaxMat + 1][kMaxMat + 1];
    for (int q = threadIdx.x; q < nmat; q += blockDim.x) {
        const DevMatT<R>& d = io.mats[q];
        mt[q] = LLGMat<R>{d.Aex, d.dA, d.ex_coef, d.dmi_coef, d.K1c, d.K2c, d.B1c, d.B2c, d.precess, d.alpha_precess, d.Ms,
                          d.aniso, (d.flags & MF_FM) ? 1u : 0u};
    }
    for (int q = threadIdx.x; q < (nmat + 1) * (nmat + 1); q += blockDim.x) {
        const int a = q / (nmat + 1), b = q - (q / (nmat + 1)) * (nmat + 1);
        sA[a][b] = tab->Aij[a][b];
    }
    __syncthreads();
    const int bjk = (int)(P.fm_bj * P.fm_bk);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bjk) return;
    const int bj = t / (int)P.fm_bk;
    const int i = (int)P.fm_i0 + blockIdx.y, j = (int)P.fm_j0 + bj, k = (int)P.fm_k0 + (t - bj * (int)P.fm_bk);
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int c = (i * ny + j) * nz + k;
    auto fm_at = [&](uint8_t q) { return q != 0 && mt[q - 1].fm != 0u; };
    const R zero = R(0);

    const uint8_t id = io.mid[c];
    const bool fm_cell = fm_at(id);
    R dmx = zero, dmy = zero, dmz = zero;
    const R mxc = io.m_in.c[0][c], myc = io.m_in.c[1][c], mzc = io.m_in.c[2][c];
    if (fm_cell) {
        const LLGMat<R>& mat = mt[id - 1];
        R mx, my, mz;
        glb2crt(P, mxc, myc, mzc, mx, my, mz);

        R exx = zero, eyy = zero, ezz = zero, eyz = zero, exz = zero, exy = zero;
        if (P.elasto_on) {
            R e[6];
            cell_strain_total(P, io, i, j, k, c, e);
            exx = e[0]; eyy = e[1]; ezz = e[2]; eyz = e[3]; exz = e[4]; exy = e[5];
        }

        // ---- one-sided differences with interface slopes ----
        const R A = mat.Aex;
        const R dA = mat.dA;   // D/2./A
        // neighbour ids and linear indices with periodic wrap at array ends
        const int ib = (i == 0) ? nx - 1 : i - 1, iF = (i == nx - 1) ? 0 : i + 1;
        const int jb = (j == 0) ? ny - 1 : j - 1, jF = (j == ny - 1) ? 0 : j + 1;
        const int kb = (k == 0) ? nz - 1 : k - 1, kF = (k == nz - 1) ? 0 : k + 1;
        const int cxb = (ib * ny + j) * nz + k, cxf = (iF * ny + j) * nz + k;
        const int cyb = (i * ny + jb) * nz + k, cyf = (i * ny + jF) * nz + k;
        const int czb = (i * ny + j) * nz + kb, czf = (i * ny + j) * nz + kF;
        // the six neighbours' m is loaded whether or not the face is a surface
        // (the wrapped indices are always inside the array), so these loads do
        // not wait for the neighbour ids
        R nm[6][3];
        {
            const int ncell[6] = {cxb, cxf, cyb, cyf, czb, czf};
#pragma unroll
            for (int f = 0; f < 6; f++)
#pragma unroll
                for (int a = 0; a < 3; a++) nm[f][a] = io.m_in.c[a][ncell[f]];
        }
        const uint8_t idxb = io.mid[cxb], idxf = io.mid[cxf], idyb = io.mid[cyb], idyf = io.mid[cyf];
        const uint8_t idzb = io.mid[czb], idzf = io.mid[czf];
        // a face is an FM surface when the neighbour across it is not FM, or
        // it is a non-periodic system boundary
        const bool sxb = (i == 0 && !P.per_x) || !fm_at(idxb);
        const bool sxf = (i == nx - 1 && !P.per_x) || !fm_at(idxf);
        const bool syb = (j == 0 && !P.per_y) || !fm_at(idyb);
        const bool syf = (j == ny - 1 && !P.per_y) || !fm_at(idyf);
        const bool szb = (k == 0 && !P.per_z) || !fm_at(idzb);
        const bool szf = (k == nz - 1 && !P.per_z) || !fm_at(idzf);

        R dxb[3], dxf[3], dyb[3], dyf[3], dzb[3], dzf[3];
        if (sxb) { dxb[0] = -dA * mzc; dxb[1] = zero; dxb[2] = dA * mxc; }
        else { dxb[0] = qdivR((mxc - nm[0][0]), P.dx, P.rdx, P.f.rdx); dxb[1] = qdivR((myc - nm[0][1]), P.dx, P.rdx, P.f.rdx); dxb[2] = qdivR((mzc - nm[0][2]), P.dx, P.rdx, P.f.rdx); }
        if (sxf) { dxf[0] = -dA * mzc; dxf[1] = zero; dxf[2] = dA * mxc; }
        else { dxf[0] = qdivR((nm[1][0] - mxc), P.dx, P.rdx, P.f.rdx); dxf[1] = qdivR((nm[1][1] - myc), P.dx, P.rdx, P.f.rdx); dxf[2] = qdivR((nm[1][2] - mzc), P.dx, P.rdx, P.f.rdx); }
        if (syb) { dyb[0] = zero; dyb[1] = -dA * mzc; dyb[2] = dA * myc; }
        else { dyb[0] = qdivR((mxc - nm[2][0]), P.dy, P.rdy, P.f.rdy); dyb[1] = qdivR((myc - nm[2][1]), P.dy, P.rdy, P.f.rdy); dyb[2] = qdivR((mzc - nm[2][2]), P.dy, P.rdy, P.f.rdy); }
        if (syf) { dyf[0] = zero; dyf[1] = -dA * mzc; dyf[2] = dA * myc; }
        else { dyf[0] = qdivR((nm[3][0] - mxc), P.dy, P.rdy, P.f.rdy); dyf[1] = qdivR((nm[3][1] - myc), P.dy, P.rdy, P.f.rdy); dyf[2] = qdivR((nm[3][2] - mzc), P.dy, P.rdy, P.f.rdy); }
        if (szb) { dzb[0] = zero; dzb[1] = zero; dzb[2] = zero; }
        else { dzb[0] = qdivR((mxc - nm[4][0]), P.dz, P.rdz, P.f.rdz); dzb[1] = qdivR((myc - nm[4][1]), P.dz, P.rdz, P.f.rdz); dzb[2] = qdivR((mzc - nm[4][2]), P.dz, P.rdz, P.f.rdz); }
        if (szf) { dzf[0] = zero; dzf[1] = zero; dzf[2] = zero; }
        else { dzf[0] = qdivR((nm[5][0] - mxc), P.dz, P.rdz, P.f.rdz); dzf[1] = qdivR((nm[5][1] - myc), P.dz, P.rdz, P.f.rdz); dzf[2] = qdivR((nm[5][2] - mzc), P.dz, P.rdz, P.f.rdz); }

        const R dmxdx = (dxb[0] + dxf[0]) * R(0.5);
        const R dmzdx = (dxb[2] + dxf[2]) * R(0.5);
        const R dmydy = (dyb[1] + dyf[1]) * R(0.5);
        const R dmzdy = (dyb[2] + dyf[2]) * R(0.5);

        // exchange coefficients per face
        const R Axf = sxf ? A : sA[id][idxf];
        const R Axb = sxb ? A : sA[id][idxb];
        const R Ayf = syf ? A : sA[id][idyf];
        const R Ayb = syb ? A : sA[id][idyb];
        const R Azf = szf ? A : sA[id][idzf];
        const R Azb = szb ? A : sA[id][idzb];

        R Hex[3];
        for (int a = 0; a < 3; a++) {
            const R d2xf = qdivR(dxf[a], P.dx, P.rdx, P.f.rdx), d2xb = -qdivR(dxb[a], P.dx, P.rdx, P.f.rdx);
            const R d2yf = qdivR(dyf[a], P.dy, P.rdy, P.f.rdy), d2yb = -qdivR(dyb[a], P.dy, P.rdy, P.f.rdy);
            const R d2zf = qdivR(dzf[a], P.dz, P.rdz, P.f.rdz), d2zb = -qdivR(dzb[a], P.dz, P.rdz, P.f.rdz);
            Hex[a] = mat.ex_coef * (Axf * d2xf + Axb * d2xb + Ayf * d2yf + Ayb * d2yb + Azf * d2zf + Azb * d2zb);
        }

        // ---- anisotropy (crystal frame) ----
        R hax = zero, hay = zero, haz = zero;
        if (mat.aniso == 1) {
            hax = R(-2.) * (mat.K1c * (my * my + mz * mz) + mat.K2c * my * my * mz * mz) * mx;
            hay = R(-2.) * (mat.K1c * (mx * mx + mz * mz) + mat.K2c * mx * mx * mz * mz) * my;
            haz = R(-2.) * (mat.K1c * (mx * mx + my * my) + mat.K2c * mx * mx * my * my) * mz;
        } else if (mat.aniso == 2) {
            haz = R(2.) * mat.K1c * mz;
        }
        R Hax, Hay, Haz;
        crt2glb(P, hax, hay, haz, Hax, Hay, Haz);

        // ---- magnetoelastic ----
        const R hex_ = R(-2.) * (mat.B1c * (exx)*mx + mat.B2c * ((exy)*my + (exz)*mz));
        const R hey_ = R(-2.) * (mat.B1c * (eyy)*my + mat.B2c * ((exy)*mx + (eyz)*mz));
        const R hez_ = R(-2.) * (mat.B1c * (ezz)*mz + mat.B2c * ((exz)*mx + (eyz)*my));
        R Hmx, Hmy, Hmz;
        crt2glb(P, hex_, hey_, hez_, Hmx, Hmy, Hmz);

        // ---- interfacial DMI ----
        const R Hdx = mat.dmi_coef * dmzdx;
        const R Hdy = mat.dmi_coef * dmzdy;
        const R Hdz = -mat.dmi_coef * (dmxdx + dmydy);

        const StageDrive& dr = stage_drive(io, S);
        R hnx = zero, hny = zero, hnz = zero;
        if (P.has_hext_nonunif) { hnx = io.Hnu.c[0][c]; hny = io.Hnu.c[1][c]; hnz = io.Hnu.c[2][c]; }
        R Hx = io.Hstat.c[0][c] + Hax + Hmx + Hex[0] + Hdx + R(dr.Hext[0]) + hnx;
        R Hy = io.Hstat.c[1][c] + Hay + Hmy + Hex[1] + Hdy + R(dr.Hext[1]) + hny;
        R Hz = io.Hstat.c[2][c] + Haz + Hmz + Hex[2] + Hdz + R(dr.Hext[2]) + hnz;

        if (P.em_back_M) {
            // cell-centred Maxwell H of the stage state (EMdynamic_solver.cpp:3780-3810)
            const int hx0 = (i * ny + j) * nz + k, hx1 = ((i + 1) * ny + j) * nz + k;
            const int hy0 = (i * (ny + 1) + j) * nz + k, hy1 = (i * (ny + 1) + j + 1) * nz + k;
            const int hz0 = (i * ny + j) * (nz + 1) + k, hz1 = hz0 + 1;
            Hx = Hx + (io.H_in.c[0][hx0] + io.H_in.c[0][hx1]) / R(2.);
            Hy = Hy + (io.H_in.c[1][hy0] + io.H_in.c[1][hy1]) / R(2.);
            // with the 1-D magnetostatic model the cell's Maxwell H_z is
            // -Ms m_z - H_stat,z of the stage state (:3793-3804; the
            // sublattice terms are zero in a ferromagnetic cell)
            if (P.mag1d_em) Hz = Hz + (-R(1.) * mat.Ms * mzc - io.Hstat.c[2][c]);
            else Hz = Hz + (io.H_in.c[2][hz0] + io.H_in.c[2][hz1]) / R(2.);
        }

        const R precess = mat.precess;
        const R px = myc * Hz - mzc * Hy;
        const R py = mzc * Hx - mxc * Hz;
        const R pz = mxc * Hy - myc * Hx;
        const R qx = myc * pz - mzc * py;
        const R qy = mzc * px - mxc * pz;
        const R qz = mxc * py - myc * px;
        dmx = precess * px + mat.alpha_precess * qx;
        dmy = precess * py + mat.alpha_precess * qy;
        dmz = precess * pz + mat.alpha_precess * qz;
    }
    // RK operands of the three components, loaded before the first store
    R mx0[3], ma[3], mcm[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        mx0[a] = io.m_x.c[a][c];
        ma[a] = (S > 0) ? io.m_acc.c[a][c] : R(0.);
        mcm[a] = R(0.);
        if constexpr (is_mixed<R>::value) { if (S == 3) mcm[a] = io.m_cmp.c[a][c]; }
    }
    if (P.em_fromM || P.spin) { io.dm.c[0][c] = dmx; io.dm.c[1][c] = dmy; io.dm.c[2][c] = dmz; }

    if constexpr (is_mixed<R>::value) {
        // mixed form: compensated RK4, then |m| = 1 (ferromagnetic cells only;
        // the others hold m = 0)
        const float d[3] = {dmx, dmy, dmz};
        if (S < 3) {
            const float cf = (S == 2) ? 1.f : 0.5f;
            float o[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                o[a] = mx0[a] + d[a] * cf;
                io.m_acc.c[a][c] = (S == 0) ? d[a] * (1.f / 6.f) : ma[a] + d[a] * (1.f / 3.f);
            }
            if (fm_cell) renorm3(o[0], o[1], o[2]);
#pragma unroll
            for (int a = 0; a < 3; a++) io.m_out.c[a][c] = o[a];
            // the next magnetostatic source, Ms m of this stage's output
            // (k_mag_source_f32 forms the same product from memory)
            if (io.msrc) {
                const float Ms = fm_cell ? mt[id - 1].Ms : 0.f;
#pragma unroll
                for (int a = 0; a < 3; a++) io.msrc[(long)a * P.n + c] = fm_cell ? Ms * o[a] : 0.f;
            }
        } else {
            float x[3], cm[3];
#pragma unroll
            for (int a = 0; a < 3; a++)
                two_sum(mx0[a], (ma[a] + d[a] * (1.f / 6.f)) + mcm[a], x[a], cm[a]);
            if (fm_cell) renorm_pair(x, cm);
#pragma unroll
            for (int a = 0; a < 3; a++) { io.m_acc.c[a][c] = x[a]; io.m_cmp.c[a][c] = cm[a]; }
            if (io.msrc) {
                const float Ms = fm_cell ? mt[id - 1].Ms : 0.f;
#pragma unroll
                for (int a = 0; a < 3; a++) io.msrc[(long)a * P.n + c] = fm_cell ? Ms * x[a] : 0.f;
            }
        }
    } else {
        // ---- RK4 combination; the magnetic increment is summed before it is
        //      added to m (magnetic_solver.cpp:1453-1455, 1601-1603) ----
        const double d[3] = {dmx, dmy, dmz};
        double o[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double xv = mx0[a];
            if (S == 0) { o[a] = xv + d[a] * 0.5; io.m_out.c[a][c] = o[a]; io.m_acc.c[a][c] = qdiv(d[a], 6., kInv6); }
            else if (S == 1) { o[a] = xv + d[a] * 0.5; io.m_out.c[a][c] = o[a]; io.m_acc.c[a][c] = ma[a] + qdiv(d[a], 3., kInv3); }
            else if (S == 2) { o[a] = xv + d[a]; io.m_out.c[a][c] = o[a]; io.m_acc.c[a][c] = ma[a] + qdiv(d[a], 3., kInv3); }
            else { o[a] = xv + (ma[a] + qdiv(d[a], 6., kInv6)); io.m_acc.c[a][c] = o[a]; }
        }
        // the next magnetostatic source, Ms m of this stage's output (the
        // product k_mag_source forms, magnetostatic_solver.cpp:129-131)
        if (io.msrc) {
            const double Ms = fm_cell ? mt[id - 1].Ms : 0.;
#pragma unroll
            for (int a = 0; a < 3; a++) io.msrc[(long)a * P.n + c] = fm_cell ? Ms * o[a] : 0.;
        }
    }
}

// ---------------------------------------------------------------------------
// Two-sublattice antiferromagnet (magnetic_system::get_dm_AFM_RK{1..4},
// magnetic_AFM_solver.cpp:3-1713, with get_m_AFM{1,2}_spatial_derivative_local
// :1837-2219 and the RK4 combination update_m_AFM_RK*/get_dm_AFM/update_m_AFM
// :1715-1835).  One thread per cell of the AFM bounding box evaluates both
// sublattices: uniaxial anisotropy 2K1/(mu0 Ms)(u.m)u, magnetoelastic field
// with factor -1, harmonic-mean exchange whose slope is 0 at AFM surfaces
// (no DMI), the inter-sublattice field -J/(mu0 Ms_s) m_other, static and
// external field and the Maxwell back-action; the exchange tables and
// surface masks of magnetic_initialize.cpp:632-1071 are derived from the
// material ids.
// ---------------------------------------------------------------------------
template <class R>
struct AFMMat {
    R Aex[2], K1c[2], B1c[2], B2c[2], J[2], ex[2], prec[2], aprec[2];
    R u[3];
    uint32_t afm;
    int pad_;
};

template <int S, class R = double>
__global__ void __launch_bounds__(256, 2) k_llg_afm(Params P, StageIOT<R> io, const LLGTablesT<R>* __restrict__ tab, int nmat) {
    __shared__ AFMMat<R> mt[kMaxMat];
    __shared__ R sA[2][kMaxMat + 1][kMaxMat + 1];
    for (int q = threadIdx.x; q < nmat; q += blockDim.x) {
        const DevMatT<R>& d = io.mats[q];
        AFMMat<R>& m = mt[q];
        for (int s = 0; s < 2; s++) {
            m.Aex[s] = d.aAex[s]; m.K1c[s] = d.aK1c[s]; m.B1c[s] = d.aB1c[s]; m.B2c[s] = d.aB2c[s];
            m.J[s] = d.aJ[s]; m.ex[s] = d.aex[s]; m.prec[s] = d.aprec[s]; m.aprec[s] = d.aaprec[s];
        }
        m.u[0] = d.au[0]; m.u[1] = d.au[1]; m.u[2] = d.au[2];
        m.afm = (d.flags & MF_AFM) ? 1u : 0u;
    }
    for (int q = threadIdx.x; q < 2 * (nmat + 1) * (nmat + 1); q += blockDim.x) {
        const int s = q / ((nmat + 1) * (nmat + 1)), r = q - s * (nmat + 1) * (nmat + 1);
        const int a = r / (nmat + 1), b = r - (r / (nmat + 1)) * (nmat + 1);
        sA[s][a][b] = tab->AijA[s][a][b];
    }
    __syncthreads();
    const int bjk = (int)(P.afm_bj * P.afm_bk);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bjk) return;
    const int bj = t / (int)P.afm_bk;
    const int i = (int)P.afm_i0 + blockIdx.y, j = (int)P.afm_j0 + bj, k = (int)P.afm_k0 + (t - bj * (int)P.afm_bk);
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int c = (i * ny + j) * nz + k;
    auto afm_at = [&](uint8_t q) { return q != 0 && mt[q - 1].afm != 0u; };

    const uint8_t id = io.mid[c];
    R dm[2][3] = {{R(0.), R(0.), R(0.)}, {R(0.), R(0.), R(0.)}};
    if (afm_at(id)) {
        const AFMMat<R>& mat = mt[id - 1];
        R exx = R(0.), eyy = R(0.), ezz = R(0.), eyz = R(0.), exz = R(0.), exy = R(0.);
        if (P.elasto_on) {
            R e[6];
            cell_strain_total(P, io, i, j, k, c, e);
            exx = e[0]; eyy = e[1]; ezz = e[2]; eyz = e[3]; exz = e[4]; exy = e[5];
        }
        const int ib = (i == 0) ? nx - 1 : i - 1, iF = (i == nx - 1) ? 0 : i + 1;
        const int jb = (j == 0) ? ny - 1 : j - 1, jF = (j == ny - 1) ? 0 : j + 1;
        const int kb = (k == 0) ? nz - 1 : k - 1, kF = (k == nz - 1) ? 0 : k + 1;
        const int nb[6] = {(ib * ny + j) * nz + k, (iF * ny + j) * nz + k, (i * ny + jb) * nz + k,
                           (i * ny + jF) * nz + k, (i * ny + j) * nz + kb, (i * ny + j) * nz + kF};
        uint8_t nid[6];
#pragma unroll
        for (int f = 0; f < 6; f++) nid[f] = io.mid[nb[f]];
        // AFM surface: the neighbour across the face is not AFM, or it is a
        // non-periodic system boundary (XOR masks, magnetic_initialize.cpp:632-860)
        const bool surf[6] = {(i == 0 && !P.per_x) || !afm_at(nid[0]), (i == nx - 1 && !P.per_x) || !afm_at(nid[1]),
                              (j == 0 && !P.per_y) || !afm_at(nid[2]), (j == ny - 1 && !P.per_y) || !afm_at(nid[3]),
                              (k == 0 && !P.per_z) || !afm_at(nid[4]), (k == nz - 1 && !P.per_z) || !afm_at(nid[5])};
        R Hem[3] = {R(0.), R(0.), R(0.)};
        if (P.em_back_M) {
            // cell-centred Maxwell H of the stage state (EMdynamic_solver.cpp:3780-3810)
            const int hx0 = (i * ny + j) * nz + k, hx1 = ((i + 1) * ny + j) * nz + k;
            const int hy0 = (i * (ny + 1) + j) * nz + k, hy1 = (i * (ny + 1) + j + 1) * nz + k;
            const int hz0 = (i * ny + j) * (nz + 1) + k, hz1 = hz0 + 1;
            Hem[0] = (io.H_in.c[0][hx0] + io.H_in.c[0][hx1]) / R(2.);
            Hem[1] = (io.H_in.c[1][hy0] + io.H_in.c[1][hy1]) / R(2.);
            if (P.mag1d_em) {
                // the 1-D model's H_z of the stage state (:3793-3804)
                const DevMatT<R>& dm_ = io.mats[id - 1];
                const R mzc = P.fm ? io.m_in.c[2][c] : R(0.);
                Hem[2] = -R(1.) * dm_.Ms * mzc - R(1.) * dm_.Ms1 * io.a1_in.c[2][c] - R(1.) * dm_.Ms2 * io.a2_in.c[2][c]
                         - io.Hstat.c[2][c];
            } else {
                Hem[2] = (io.H_in.c[2][hz0] + io.H_in.c[2][hz1]) / R(2.);
            }
        }
        const StageDrive& dr = stage_drive(io, S);
        const double h[3] = {P.dx, P.dy, P.dz}, rh[3] = {P.rdx, P.rdy, P.rdz};
        const float rhf[3] = {P.f.rdx, P.f.rdy, P.f.rdz};
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const F3T<R>& ms = s ? io.a2_in : io.a1_in;
            const F3T<R>& mo = s ? io.a1_in : io.a2_in;
            const R mgx = ms.c[0][c], mgy = ms.c[1][c], mgz = ms.c[2][c];
            const R mg[3] = {mgx, mgy, mgz};
            R mx, my, mz;
            glb2crt(P, mgx, mgy, mgz, mx, my, mz);
            // exchange: slopes to the six neighbours (0 at surfaces), then
            // the second-difference terms d?/dx2_f = fwd/dx, _b = -bwd/dx
            R Hex[3];
            {
                R Aij[6];
#pragma unroll
                for (int f = 0; f < 6; f++) Aij[f] = surf[f] ? mat.Aex[s] : sA[s][id][nid[f]];
                R acc[3] = {R(0.), R(0.), R(0.)};
                R d2[6][3];
#pragma unroll
                for (int dir = 0; dir < 3; dir++) {
                    const int fb = 2 * dir, ff = 2 * dir + 1;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const R bwd = surf[fb] ? R(0.) : qdivR(mg[a] - ms.c[a][nb[fb]], h[dir], rh[dir], rhf[dir]);
                        const R fwd = surf[ff] ? R(0.) : qdivR(ms.c[a][nb[ff]] - mg[a], h[dir], rh[dir], rhf[dir]);
                        d2[ff][a] = qdivR(fwd, h[dir], rh[dir], rhf[dir]);
                        d2[fb][a] = -qdivR(bwd, h[dir], rh[dir], rhf[dir]);
                    }
                }
#pragma unroll
                for (int a = 0; a < 3; a++)
                    acc[a] = Aij[1] * d2[1][a] + Aij[0] * d2[0][a] + Aij[3] * d2[3][a] + Aij[2] * d2[2][a]
                             + Aij[5] * d2[5][a] + Aij[4] * d2[4][a];
#pragma unroll
                for (int a = 0; a < 3; a++) Hex[a] = mat.ex[s] * acc[a];
            }
            // uniaxial anisotropy (crystal frame)
            const R udotm = mx * mat.u[0] + my * mat.u[1] + mz * mat.u[2];
            R Hax, Hay, Haz;
            crt2glb(P, R(2.) * mat.K1c[s] * udotm * mat.u[0], R(2.) * mat.K1c[s] * udotm * mat.u[1],
                    R(2.) * mat.K1c[s] * udotm * mat.u[2], Hax, Hay, Haz);
            // magnetoelastic field, factor -1
            const R B1 = mat.B1c[s], B2 = mat.B2c[s];
            R Hmx, Hmy, Hmz;
            crt2glb(P, -R(1.) * (B1 * (exx)*mx + B2 * ((exy)*my + (exz)*mz)), -R(1.) * (B1 * (eyy)*my + B2 * ((exy)*mx + (eyz)*mz)),
                    -R(1.) * (B1 * (ezz)*mz + B2 * ((exz)*mx + (eyz)*my)), Hmx, Hmy, Hmz);
            // inter-sublattice exchange with the other sublattice's stage state
            const R Hix = mat.J[s] * mo.c[0][c], Hiy = mat.J[s] * mo.c[1][c], Hiz = mat.J[s] * mo.c[2][c];
            R Hx = io.Hstat.c[0][c] + Hax + Hmx + Hex[0] + Hix + R(dr.Hext_afm[0]);
            R Hy = io.Hstat.c[1][c] + Hay + Hmy + Hex[1] + Hiy + R(dr.Hext_afm[1]);
            R Hz = io.Hstat.c[2][c] + Haz + Hmz + Hex[2] + Hiz + R(dr.Hext_afm[2]);
            if (P.em_back_M) { Hx = Hx + Hem[0]; Hy = Hy + Hem[1]; Hz = Hz + Hem[2]; }
            const R px = mgy * Hz - mgz * Hy;
            const R py = mgz * Hx - mgx * Hz;
            const R pz = mgx * Hy - mgy * Hx;
            const R qx = mgy * pz - mgz * py;
            const R qy = mgz * px - mgx * pz;
            const R qz = mgx * py - mgy * px;
            dm[s][0] = mat.prec[s] * px + mat.aprec[s] * qx;
            dm[s][1] = mat.prec[s] * py + mat.aprec[s] * qy;
            dm[s][2] = mat.prec[s] * pz + mat.aprec[s] * qz;
        }
    }
    // RK operands of both sublattices, loaded before the first store
    R sx[2][3], sa[2][3], sc[2][3];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int a = 0; a < 3; a++) {
            sx[s][a] = (s ? io.a2_x : io.a1_x).c[a][c];
            sa[s][a] = (S > 0) ? (s ? io.a2_acc : io.a1_acc).c[a][c] : R(0.);
            sc[s][a] = R(0.);
            if constexpr (is_mixed<R>::value) { if (S == 3) sc[s][a] = (s ? io.a2_cmp : io.a1_cmp).c[a][c]; }
        }
    if (P.em_fromM || P.spin) {
#pragma unroll
        for (int a = 0; a < 3; a++) { io.da1.c[a][c] = dm[0][a]; io.da2.c[a][c] = dm[1][a]; }
    }
    const bool afm_cell = afm_at(id);
    if constexpr (is_mixed<R>::value) {
        // mixed form: compensated RK4 of both sublattices, then |m_s| = 1
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const F3T<R>& O = s ? io.a2_out : io.a1_out;
            const F3T<R>& A = s ? io.a2_acc : io.a1_acc;
            const F3T<R>& Cm = s ? io.a2_cmp : io.a1_cmp;
            if (S < 3) {
                const float cf = (S == 2) ? 1.f : 0.5f;
                float o[3];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    o[a] = sx[s][a] + dm[s][a] * cf;
                    A.c[a][c] = (S == 0) ? dm[s][a] * (1.f / 6.f) : sa[s][a] + dm[s][a] * (1.f / 3.f);
                }
                if (afm_cell) renorm3(o[0], o[1], o[2]);
#pragma unroll
                for (int a = 0; a < 3; a++) O.c[a][c] = o[a];
            } else {
                float x[3], cm[3];
#pragma unroll
                for (int a = 0; a < 3; a++)
                    two_sum(sx[s][a], (sa[s][a] + dm[s][a] * (1.f / 6.f)) + sc[s][a], x[a], cm[a]);
                if (afm_cell) renorm_pair(x, cm);
#pragma unroll
                for (int a = 0; a < 3; a++) { A.c[a][c] = x[a]; Cm.c[a][c] = cm[a]; }
            }
        }
    } else {
        // RK4 combination; the increment is summed before it is added to m
        // (get_dm_AFM / update_m_AFM, magnetic_AFM_solver.cpp:1715-1835)
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const F3& O = s ? io.a2_out : io.a1_out;
            const F3& A = s ? io.a2_acc : io.a1_acc;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const double d = dm[s][a];
                const double xv = sx[s][a];
                if (S == 0) { O.c[a][c] = xv + d * 0.5; A.c[a][c] = qdiv(d, 6., kInv6); }
                else if (S == 1) { O.c[a][c] = xv + d * 0.5; A.c[a][c] = sa[s][a] + qdiv(d, 3., kInv3); }
                else if (S == 2) { O.c[a][c] = xv + d; A.c[a][c] = sa[s][a] + qdiv(d, 3., kInv3); }
                else { A.c[a][c] = xv + (sa[s][a] + qdiv(d, 6., kInv6)); }
            }
        }
    }
}

// Prescribed-m test mode (if_prescribed_m; update_prescribed_m_half /
// _full / update_prescribed_m, magnetic_solver.cpp:1891-1960): after the
// update of stage S the ferromagnetic cells of plane k = 0 take the stage
// drive's prescribed m — the stage output for S < 3, the new step value for
// S = 3 (in the mixed form with its compensation word cleared).  One thread
// per (i, j).
template <int S, class R>
__global__ void k_prescribed_m(Params P, StageIOT<R> io) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)P.nx * P.ny) return;
    const long i = t / P.ny, j = t - i * P.ny;
    const long c = cid(P, i, j, 0);
    const uint8_t id = io.mid[c];
    if (id == 0 || !(io.mats[id - 1].flags & MF_FM)) return;
    const StageDrive& dr = stage_drive(io, S);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        R* tgt = (S < 3) ? io.m_out.c[a] : io.m_acc.c[a];
        tgt[c] = R(dr.pm[a]);
        if constexpr (is_mixed<R>::value) { if (S == 3) io.m_cmp.c[a][c] = R(0); }
    }
}

// z component of the cell-centred Maxwell H when the 1-D magnetostatic
// model meets M-sourced Maxwell fields (update_DH_cell, EMdynamic_solver.cpp:
// 3793-3804): -Ms m_z - Ms1 m1_z - Ms2 m2_z - H_stat,z of the cell's current
// step value, zero in vacuum; written over the face mean that k_em_cell
// leaves in out (cells c0 .. c0 + count - 1; mz, mz1, mz2 null where the run
// has no such magnet)
template <class R>
__global__ void k_em_cell_hz_1d(const DevMatT<R>* __restrict__ mats, const uint8_t* __restrict__ mid, const R* __restrict__ mz,
                                const R* __restrict__ mz1, const R* __restrict__ mz2, const R* __restrict__ hz,
                                double* __restrict__ out, long c0, long count) {
    const long c = c0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c0 + count) return;
    const uint8_t id = mid[c];
    if (id == 0) { out[c] = 0.; return; }
    const DevMatT<R>& m = mats[id - 1];
    const R z = mz ? mz[c] : R(0.), z1 = mz1 ? mz1[c] : R(0.), z2 = mz2 ? mz2[c] : R(0.);
    out[c] = (double)(-R(1.) * m.Ms * z - R(1.) * m.Ms1 * z1 - R(1.) * m.Ms2 * z2 - hz[c]);
}

}  // namespace gf
