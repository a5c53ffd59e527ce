// Device-side data layout and helpers shared by every kernel of the engine.
//
// Storage is the reference's matrix3d order (matrix.h:46-52): one array per
// vector component, index (i*dimy + j)*dimz + k, z fastest.  Material ids are
// one byte per cell (0 = vacuum, id-1 indexes the material table), in place
// of the reference's unsigned int material_cell (global.h:92).
//
// The FP64 parity kernels are compiled with -fmad=false and evaluate every
// expression in the reference's operation order, so that each multiply and
// add is rounded exactly as in the reference's host build.
#pragma once

#include <cstdint>

namespace gf {

constexpr double kMu0 = 1.256637061e-6;     // magnetic_system.h:14, EMdynamic_system.h:12
constexpr double kE0 = 8.854187817e-12;     // EMdynamic_system.h:13
constexpr double kC0 = 2.99792458e8;        // EMdynamic_system.h:14
constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxMat = 32;

enum MatFlag : uint32_t { MF_FM = 1u, MF_AFM = 2u, MF_FE = 4u, MF_PEC = 8u };

// Real type of the mixed-precision form: state and stencils in FP32.
template <class R> struct is_mixed { static constexpr bool value = false; };
template <> struct is_mixed<float> { static constexpr bool value = true; };

// Per-material constants, precomputed on the host with the same expressions
// (and operation order) the reference evaluates inside its cell loops.  The
// FP64 table is converted member by member for the mixed form: after the
// four integers every member is a real of type R.
template <class R>
struct DevMatT {
    uint32_t flags;
    int aniso;          // anisotropy_type
    int cubic_c;        // 1: rotated stiffness has the cubic sparsity pattern
    int pad_;
    // FM LLG (magnetic_solver.cpp:84-87, 164-185, 206-208)
    R Ms, K1c, K2c, B1c, B2c, Aex, dA;   // dA = D/2./A
    R ex_coef;                            // 2./mu0/Ms
    R dmi_coef;                           // 2.*D/mu0/Ms
    R alpha, precess, alpha_precess;      // precess = -gyro/(1+a^2)*dt
    // AFM sublattices s = 0, 1 (magnetic_AFM_solver.cpp:106-112, 181-191)
    R Ms1, Ms2;
    R aAex[2];                 // Aex_AFM
    R aK1c[2], aB1c[2], aB2c[2];   // K1/mu0/Ms, B1/mu0/Ms, B2/mu0/Ms
    R aJ[2];                   // -1*J_AFM/mu0/Ms
    R aex[2];                  // 2./mu0/Ms
    R aprec[2], aaprec[2];     // -gyro/(1+a^2)*dt and alpha times it
    R au[3];                   // uniaxial axis (crystal frame, normalised)
    // elastic (elastic_dynamic_solver.cpp:1295-1297)
    R cij[6][6];
    R dens_dt, mass_damp, stiff_damp;
    // dynamic eigenstrain (elastic_dynamic_solver.cpp:24-61)
    R l100_15, l111_15, l100a1_075, l100a2_075, l111a1_075, l111a2_075;
    R Q11, Q12, Q44;
    // ferroelectric TDGL (ferroelectric_solver.cpp:704-717)
    R a1, a11, a12, a111, a112, a123, a1111, a1112, a1122, a1123;
    R tv1, tv2, tv3, G11;
    R fe_coef, fe_damp;                    // -dt/m, fe_coef*gamma
    // flexoelectric coupling (ferroelectric_solver.cpp:800-833,
    // elastic_dynamic_solver.cpp:63-70; read.cpp:182-198)
    R tv4, tv5, tv6, tv7, tv8;
    R f11, f12, f44x2;                     // f44x2 = 2 f44
    R F11, F12, F44h;                      // F44h = F44 / 2
    // electromagnetic
    R er, cond;
    R comp[3], wp[3], rtau[3];
};
using DevMat = DevMatT<double>;
constexpr int kDevMatReals = (int)((sizeof(DevMatT<double>) - 16) / sizeof(double));
static_assert(sizeof(DevMatT<double>) == 16 + kDevMatReals * sizeof(double), "DevMatT<double> layout");
static_assert(sizeof(DevMatT<float>) == 16 + kDevMatReals * sizeof(float), "DevMatT<float> layout");

// Grid, switches and scalars that every kernel needs (passed by value).
struct Params {
    int nx, ny, nz;
    int per_x, per_y, per_z;
    long n;
    double dx, dy, dz, dt;
    double rdx, rdy, rdz, rdt;   // correctly rounded reciprocals (host 1./dx ...), for qdiv
    double dt_e0, mdt_mu0;       // dt / e0 and -dt / mu0, rounded as the reference does
    int rot;                 // if_OrientRotate
    double Tg2c[3][3], Tc2g[3][3];
    // active physics
    int fm, afm, fe, elastic, em;
    // bounding boxes of the ferromagnetic and antiferromagnetic cells (the
    // LLG kernels cover only them)
    long fm_i0, fm_j0, fm_k0, fm_bi, fm_bj, fm_bk;
    long afm_i0, afm_j0, afm_k0, afm_bi, afm_bj, afm_bk;
    int elasto_on, elasto_back;   // if_elasto_on_pORm, if_elasto_backaction_from_pORm
    int em_fromM, em_fromP, em_back_M, em_back_P;
    int has_eig0, has_strain0, has_hext_nonunif;
    int estat;                 // E_stat may be nonzero (Estat.in, the electrostatic solve or an upload); 0: it is all +0
    int abc_1D, abc_elast_onlytop, abc_em_onlytop, pec_xy, pec_z;
    int prescribed_m;             // if_prescribed_m: k = 0 ferromagnetic cells precess on a prescribed cone
    uint32_t fe_mask, fm_mask;   // bit id-1 set when material id is ferroelectric / ferromagnetic
    int spin;                 // spin pumping: inverse-spin-Hall current in the Yee E update
    int em_cls;               // the Yee E update reads per-edge material classes (StageIOT::ecls)
    int drude;                // some material has a Drude pole (omega_plasma != 0)
    int pec;                  // some material is a perfect electric conductor
    int mag_1D;
    int mag1d_em;             // if_mag_1Dmodel with M-sourced Maxwell fields: the cell-centred Maxwell H_z is the 1-D field
    int el_bc_fused;          // the elastic RK update also applies the boundary planes (no k_elastic_bc launch)
    int flexo;                // if_flexo with ferroelectrics: StageIOT::sg / pge are set
    int elastostatic;         // if_elastostatic: the TDGL field adds the static strain and eigenstrain
    double liao_w;
    // elastic boundary coefficients (elastodynamics_AbsorbingBoundary.cpp)
    double vs_long_1st, vs_tran_1st, vs_long_last, vs_tran_last;
    double mur_el_half[4], mur_el_full[4];    // long_1st tran_1st long_last tran_last
    unsigned source_z;
    int strain_pulse, strain_type;
    int strain_comp;                           // 0,1,2 for x,y,z
    // EM Mur coefficients (EMdynamic_initialize.cpp:48-56)
    double c_top_half, c_bot_half, c_x_half, c_y_half;
    double c_top, c_bot, c_x, c_y;
    long plane_z;                               // planeEM_source_z
    int planeEM;
    // J_f box (EMdynamic_initialize.cpp:60-68)
    int jf_on, jf_type, jf_comp;
    long jf_i0, jf_i1, jf_j0, jf_j1, jf_k0, jf_k1;
    // FP32 copies of the constants the mixed-form stencils use
    struct {
        float rdx, rdy, rdz, rdt, dt, dt_e0, mdt_mu0;
        float Tg2c[3][3], Tc2g[3][3];
    } f;
};

// Values that depend on time, computed on the host for every step with the
// reference's expressions (magnetic_solver.cpp:1833-1861,
// ferroelectric_solver.cpp:2001-2029, elastic_dynamic_solver.cpp:1195-1223
// and 3059-3284, EMdynamic_solver.cpp:3828-4316).  Index s = RK stage 0..3.
struct StageDrive {
    double Hext[3];        // external H seen by the ferromagnet
    double Hext_afm[3];    // external H seen by the antiferromagnet (differs with a prescribed table)
    double Eext[3];
    double traction;       // surface traction on the source plane (type 3)
    double usrc;           // displacement written on the source plane after the update
    double jf;             // J_f amplitude factor for the stage (types 1,2 times a per-k factor)
    double plane[3];       // plane-wave E written after the update
    double pm[3];          // prescribed m of the k = 0 ferromagnetic cells after the update (if_prescribed_m)
    int usrc_on;
    int pad_;
};
struct StepDrive {
    double t;
    StageDrive st[4];
};

constexpr double kInv3 = 1. / 3.;
constexpr double kInv6 = 1. / 6.;

// x / d rounded to nearest, for a divisor d that is fixed for the run, given
// rd = RN(1/d) (computed once on the host by IEEE division).  This is
// Markstein's correction step (P. W. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990): if q is within one ulp of x/d and rd is the correctly rounded
// reciprocal, the residual r = x - d*q is exact in one FMA and RN(q + r*rd)
// is the correctly rounded quotient.  q0 = RN(x*rd) can be up to two ulps
// off, so a first correction makes it faithful and a second rounds it
// correctly.  The identity needs normal residuals, which holds for every
// field value here (|x| far above 1e-290); a zero x keeps its sign.  Five
// FP64 operations and no branch, against the general division's reciprocal
// refinement and slow-path test.
__device__ __forceinline__ double qdiv(double x, double d, double rd) {
    const double q0 = __dmul_rn(x, rd);
    double r = __fma_rn(-q0, d, x);
    const double q1 = __fma_rn(r, rd, q0);
    r = __fma_rn(-q1, d, x);
    const double q2 = __fma_rn(r, rd, q1);
    return x == 0. ? q0 : q2;
}

// Division by a run constant d: qdiv in the FP64 form (rd = RN(1/d)); in the
// mixed form a multiplication by the FP32 reciprocal rdf (within one ulp of
// the FP32 quotient).
__device__ __forceinline__ double qdivR(double x, double d, double rd, float) { return qdiv(x, d, rd); }
__device__ __forceinline__ float qdivR(float x, double, double, float rdf) { return x * rdf; }

// frame-rotation matrices in the kernel's precision
template <class R> __device__ __forceinline__ const auto& Tg2c(const Params& P) {
    if constexpr (is_mixed<R>::value) return P.f.Tg2c; else return P.Tg2c;
}
template <class R> __device__ __forceinline__ const auto& Tc2g(const Params& P) {
    if constexpr (is_mixed<R>::value) return P.f.Tc2g; else return P.Tc2g;
}

__host__ __device__ inline long cid(const Params& P, long i, long j, long k) {
    return (i * P.ny + j) * P.nz + k;
}

// 3x3 frame rotations (mathlib.cpp:45-125); identity when rot == 0
template <class R>
__device__ inline void glb2crt(const Params& P, R x, R y, R z, R& a, R& b, R& c) {
    if (P.rot) {
        const auto& T = Tg2c<R>(P);
        a = T[0][0] * x + T[0][1] * y + T[0][2] * z;
        b = T[1][0] * x + T[1][1] * y + T[1][2] * z;
        c = T[2][0] * x + T[2][1] * y + T[2][2] * z;
    } else { a = x; b = y; c = z; }
}
template <class R>
__device__ inline void crt2glb(const Params& P, R x, R y, R z, R& a, R& b, R& c) {
    if (P.rot) {
        const auto& T = Tc2g<R>(P);
        a = T[0][0] * x + T[0][1] * y + T[0][2] * z;
        b = T[1][0] * x + T[1][1] * y + T[1][2] * z;
        c = T[2][0] * x + T[2][1] * y + T[2][2] * z;
    } else { a = x; b = y; c = z; }
}
// symmetric tensor rotation out[i][j] = sum_kl T[i][k] T[j][l] in[k][l]
template <class R>
__device__ inline void rot_tensor(const R T[3][3], const R in[3][3], R out[3][3]) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            R acc = R(0);
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) acc = acc + T[i][k] * T[j][l] * in[k][l];
            out[i][j] = acc;
        }
}

}  // namespace gf
