// Ferromagnetic LLG stage kernel (FP64).
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

struct LLGTables {
    double Aij[kMaxMat + 1][kMaxMat + 1];   // 2*A1*A2/(A1+A2) for ids (1-based)
};

__device__ inline bool is_fm(const DevMat* mats, uint8_t id) {
    return id != 0 && (mats[id - 1].flags & MF_FM);
}

// static strain plus the cell strain of the stage displacement, crystal
// frame (exxt0_crt + Dexx_crt, magnetic_solver.cpp:89-96); the dynamic part
// is written by k_elastic_tile earlier in the same stage
__device__ inline void cell_strain_total(const Params& P, const StageIO& io, long i, long j, long k, long c, double e[6]) {
    double d[6] = {0., 0., 0., 0., 0., 0.};
    if (P.elastic) for (int a = 0; a < 6; a++) d[a] = io.strain_c[a][c];
    for (int a = 0; a < 6; a++) {
        double t = io.eps0_c[a] ? io.eps0_c[a][c] : 0.;
        e[a] = t + d[a];
    }
}

// One thread per cell of the ferromagnetic bounding box; cells outside it
// hold their initial m in all four buffers and are never touched.
template <int S>
__global__ void __launch_bounds__(256) k_llg_fm(Params P, StageIO io, const LLGTables* __restrict__ tab) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long bjk = P.fm_bj * P.fm_bk;
    if (t >= P.fm_bi * bjk) return;
    const long bi = t / bjk, r = t - bi * bjk, bj = r / P.fm_bk;
    const long i = P.fm_i0 + bi, j = P.fm_j0 + bj, k = P.fm_k0 + (r - bj * P.fm_bk);
    const long c = cid(P, i, j, k);

    const uint8_t id = io.mid[c];
    double dmx = 0., dmy = 0., dmz = 0.;
    const double mxc = io.m_in.c[0][c], myc = io.m_in.c[1][c], mzc = io.m_in.c[2][c];
    if (is_fm(io.mats, id)) {
        const DevMat& mat = io.mats[id - 1];
        double mx, my, mz;
        glb2crt(P, mxc, myc, mzc, mx, my, mz);

        double exx = 0., eyy = 0., ezz = 0., eyz = 0., exz = 0., exy = 0.;
        if (P.elasto_on) {
            double e[6];
            cell_strain_total(P, io, i, j, k, c, e);
            exx = e[0]; eyy = e[1]; ezz = e[2]; eyz = e[3]; exz = e[4]; exy = e[5];
        }

        // ---- one-sided differences with interface slopes ----
        const double A = mat.Aex;
        const double dA = mat.dA;   // D/2./A
        // neighbour ids and linear indices with periodic wrap at array ends
        const long ib = (i == 0) ? P.nx - 1 : i - 1, iF = (i == P.nx - 1) ? 0 : i + 1;
        const long jb = (j == 0) ? P.ny - 1 : j - 1, jF = (j == P.ny - 1) ? 0 : j + 1;
        const long kb = (k == 0) ? P.nz - 1 : k - 1, kF = (k == P.nz - 1) ? 0 : k + 1;
        const long cxb = cid(P, ib, j, k), cxf = cid(P, iF, j, k);
        const long cyb = cid(P, i, jb, k), cyf = cid(P, i, jF, k);
        const long czb = cid(P, i, j, kb), czf = cid(P, i, j, kF);
        // a face is an FM surface when the neighbour across it is not FM, or
        // it is a non-periodic system boundary
        const bool sxb = (i == 0 && !P.per_x) || !is_fm(io.mats, io.mid[cxb]);
        const bool sxf = (i == P.nx - 1 && !P.per_x) || !is_fm(io.mats, io.mid[cxf]);
        const bool syb = (j == 0 && !P.per_y) || !is_fm(io.mats, io.mid[cyb]);
        const bool syf = (j == P.ny - 1 && !P.per_y) || !is_fm(io.mats, io.mid[cyf]);
        const bool szb = (k == 0 && !P.per_z) || !is_fm(io.mats, io.mid[czb]);
        const bool szf = (k == P.nz - 1 && !P.per_z) || !is_fm(io.mats, io.mid[czf]);

        double dxb[3], dxf[3], dyb[3], dyf[3], dzb[3], dzf[3];
        if (sxb) { dxb[0] = -dA * mzc; dxb[1] = 0.; dxb[2] = dA * mxc; }
        else { dxb[0] = qdiv((mxc - io.m_in.c[0][cxb]), P.dx, P.rdx); dxb[1] = qdiv((myc - io.m_in.c[1][cxb]), P.dx, P.rdx); dxb[2] = qdiv((mzc - io.m_in.c[2][cxb]), P.dx, P.rdx); }
        if (sxf) { dxf[0] = -dA * mzc; dxf[1] = 0.; dxf[2] = dA * mxc; }
        else { dxf[0] = qdiv((io.m_in.c[0][cxf] - mxc), P.dx, P.rdx); dxf[1] = qdiv((io.m_in.c[1][cxf] - myc), P.dx, P.rdx); dxf[2] = qdiv((io.m_in.c[2][cxf] - mzc), P.dx, P.rdx); }
        if (syb) { dyb[0] = 0.; dyb[1] = -dA * mzc; dyb[2] = dA * myc; }
        else { dyb[0] = qdiv((mxc - io.m_in.c[0][cyb]), P.dy, P.rdy); dyb[1] = qdiv((myc - io.m_in.c[1][cyb]), P.dy, P.rdy); dyb[2] = qdiv((mzc - io.m_in.c[2][cyb]), P.dy, P.rdy); }
        if (syf) { dyf[0] = 0.; dyf[1] = -dA * mzc; dyf[2] = dA * myc; }
        else { dyf[0] = qdiv((io.m_in.c[0][cyf] - mxc), P.dy, P.rdy); dyf[1] = qdiv((io.m_in.c[1][cyf] - myc), P.dy, P.rdy); dyf[2] = qdiv((io.m_in.c[2][cyf] - mzc), P.dy, P.rdy); }
        if (szb) { dzb[0] = 0.; dzb[1] = 0.; dzb[2] = 0.; }
        else { dzb[0] = qdiv((mxc - io.m_in.c[0][czb]), P.dz, P.rdz); dzb[1] = qdiv((myc - io.m_in.c[1][czb]), P.dz, P.rdz); dzb[2] = qdiv((mzc - io.m_in.c[2][czb]), P.dz, P.rdz); }
        if (szf) { dzf[0] = 0.; dzf[1] = 0.; dzf[2] = 0.; }
        else { dzf[0] = qdiv((io.m_in.c[0][czf] - mxc), P.dz, P.rdz); dzf[1] = qdiv((io.m_in.c[1][czf] - myc), P.dz, P.rdz); dzf[2] = qdiv((io.m_in.c[2][czf] - mzc), P.dz, P.rdz); }

        const double dmxdx = (dxb[0] + dxf[0]) * 0.5;
        const double dmzdx = (dxb[2] + dxf[2]) * 0.5;
        const double dmydy = (dyb[1] + dyf[1]) * 0.5;
        const double dmzdy = (dyb[2] + dyf[2]) * 0.5;

        // exchange coefficients per face
        const double Axf = sxf ? A : tab->Aij[id][io.mid[cxf]];
        const double Axb = sxb ? A : tab->Aij[id][io.mid[cxb]];
        const double Ayf = syf ? A : tab->Aij[id][io.mid[cyf]];
        const double Ayb = syb ? A : tab->Aij[id][io.mid[cyb]];
        const double Azf = szf ? A : tab->Aij[id][io.mid[czf]];
        const double Azb = szb ? A : tab->Aij[id][io.mid[czb]];

        double Hex[3];
        for (int a = 0; a < 3; a++) {
            const double d2xf = qdiv(dxf[a], P.dx, P.rdx), d2xb = -qdiv(dxb[a], P.dx, P.rdx);
            const double d2yf = qdiv(dyf[a], P.dy, P.rdy), d2yb = -qdiv(dyb[a], P.dy, P.rdy);
            const double d2zf = qdiv(dzf[a], P.dz, P.rdz), d2zb = -qdiv(dzb[a], P.dz, P.rdz);
            Hex[a] = mat.ex_coef * (Axf * d2xf + Axb * d2xb + Ayf * d2yf + Ayb * d2yb + Azf * d2zf + Azb * d2zb);
        }

        // ---- anisotropy (crystal frame) ----
        double hax = 0., hay = 0., haz = 0.;
        if (mat.aniso == 1) {
            hax = -2. * (mat.K1c * (my * my + mz * mz) + mat.K2c * my * my * mz * mz) * mx;
            hay = -2. * (mat.K1c * (mx * mx + mz * mz) + mat.K2c * mx * mx * mz * mz) * my;
            haz = -2. * (mat.K1c * (mx * mx + my * my) + mat.K2c * mx * mx * my * my) * mz;
        } else if (mat.aniso == 2) {
            haz = 2. * mat.K1c * mz;
        }
        double Hax, Hay, Haz;
        crt2glb(P, hax, hay, haz, Hax, Hay, Haz);

        // ---- magnetoelastic ----
        const double hex_ = -2. * (mat.B1c * (exx)*mx + mat.B2c * ((exy)*my + (exz)*mz));
        const double hey_ = -2. * (mat.B1c * (eyy)*my + mat.B2c * ((exy)*mx + (eyz)*mz));
        const double hez_ = -2. * (mat.B1c * (ezz)*mz + mat.B2c * ((exz)*mx + (eyz)*my));
        double Hmx, Hmy, Hmz;
        crt2glb(P, hex_, hey_, hez_, Hmx, Hmy, Hmz);

        // ---- interfacial DMI ----
        const double Hdx = mat.dmi_coef * dmzdx;
        const double Hdy = mat.dmi_coef * dmzdy;
        const double Hdz = -mat.dmi_coef * (dmxdx + dmydy);

        const StageDrive& dr = stage_drive(io, S);
        double hnx = 0., hny = 0., hnz = 0.;
        if (P.has_hext_nonunif) { hnx = io.Hnu.c[0][c]; hny = io.Hnu.c[1][c]; hnz = io.Hnu.c[2][c]; }
        double Hx = io.Hstat.c[0][c] + Hax + Hmx + Hex[0] + Hdx + dr.Hext[0] + hnx;
        double Hy = io.Hstat.c[1][c] + Hay + Hmy + Hex[1] + Hdy + dr.Hext[1] + hny;
        double Hz = io.Hstat.c[2][c] + Haz + Hmz + Hex[2] + Hdz + dr.Hext[2] + hnz;

        if (P.em_back_M) {
            // cell-centred Maxwell H of the stage state (EMdynamic_solver.cpp:3780-3810)
            const long hx0 = (i * P.ny + j) * P.nz + k, hx1 = ((i + 1) * P.ny + j) * P.nz + k;
            const long hy0 = (i * (P.ny + 1) + j) * P.nz + k, hy1 = (i * (P.ny + 1) + j + 1) * P.nz + k;
            const long hz0 = (i * P.ny + j) * (P.nz + 1) + k, hz1 = hz0 + 1;
            Hx = Hx + (io.H_in.c[0][hx0] + io.H_in.c[0][hx1]) / 2.;
            Hy = Hy + (io.H_in.c[1][hy0] + io.H_in.c[1][hy1]) / 2.;
            Hz = Hz + (io.H_in.c[2][hz0] + io.H_in.c[2][hz1]) / 2.;
        }

        const double precess = mat.precess;
        const double px = myc * Hz - mzc * Hy;
        const double py = mzc * Hx - mxc * Hz;
        const double pz = mxc * Hy - myc * Hx;
        const double qx = myc * pz - mzc * py;
        const double qy = mzc * px - mxc * pz;
        const double qz = mxc * py - myc * px;
        dmx = precess * px + mat.alpha_precess * qx;
        dmy = precess * py + mat.alpha_precess * qy;
        dmz = precess * pz + mat.alpha_precess * qz;
    }
    if (P.em_fromM) { io.dm.c[0][c] = dmx; io.dm.c[1][c] = dmy; io.dm.c[2][c] = dmz; }

    // ---- RK4 combination; the magnetic increment is summed before it is
    //      added to m (magnetic_solver.cpp:1453-1455, 1601-1603) ----
    const double d[3] = {dmx, dmy, dmz};
    for (int a = 0; a < 3; a++) {
        const double xv = io.m_x.c[a][c];
        if (S == 0) { io.m_out.c[a][c] = xv + d[a] * 0.5; io.m_acc.c[a][c] = qdiv(d[a], 6., kInv6); }
        else if (S == 1) { io.m_out.c[a][c] = xv + d[a] * 0.5; io.m_acc.c[a][c] = io.m_acc.c[a][c] + qdiv(d[a], 3., kInv3); }
        else if (S == 2) { io.m_out.c[a][c] = xv + d[a]; io.m_acc.c[a][c] = io.m_acc.c[a][c] + qdiv(d[a], 3., kInv3); }
        else { io.m_acc.c[a][c] = xv + (io.m_acc.c[a][c] + qdiv(d[a], 6., kInv6)); }
    }
}

}  // namespace gf
