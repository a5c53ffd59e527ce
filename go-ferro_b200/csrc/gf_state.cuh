// Device pointers that one RK stage of one step reads and writes.
//
// Every state field F keeps four device arrays per component:
//   X  — value at the start of the step (the reference's F_glb),
//   A  — RK4 accumulator; after the last stage it holds the new step value,
//        and the engine swaps the roles of X and A (two captured graphs,
//        one per parity of the step counter),
//   S0, S1 — stage states (the reference's F_glb_store), ping-ponged so a
//        stencil can read stage s while stage s+1 is written.
// Stage s reads `in` (X for s=0, S0, S1, S0) and writes `out` (S0, S1, S0,
// and for the last stage the A buffer in place).  This replaces the
// reference's five arrays per component (F_glb, F_glb_store, dF_rk1..4).
//
// The mixed-precision form (R = float) keeps the same four arrays in FP32
// plus a compensation word C per scalar: the step value is X + C.  Stages
// 1-3 accumulate only the weighted increments in A; the last stage adds
// A + C to X with an error-free sum, stores the rounded sum as the new step
// value and its rounding error as the new C.
#pragma once

#include "gf_common.cuh"

namespace gf {

template <class R> struct F3T { R* c[3]; };
using F3 = F3T<double>;

template <class R>
struct StageIOT {
    using F3 = F3T<R>;
    // ferromagnet m and its stage increment (read by the Maxwell H update)
    F3 m_in, m_x, m_acc, m_out, dm;
    // antiferromagnet sublattices m1, m2 and their stage increments
    F3 a1_in, a1_x, a1_acc, a1_out, da1;
    F3 a2_in, a2_x, a2_acc, a2_out, da2;
    // ferroelectric p and q = dp/dt
    F3 p_in, p_x, p_acc, p_out, q_in, q_x, q_acc, q_out;
    // elastic displacement u and velocity v
    F3 u_in, u_x, u_acc, u_out, v_in, v_x, v_acc, v_out;
    F3 force_store;   // stage-1 stress divergence (stiffness damping)
    F3 force;         // stress divergence of the stage, k_elastic_tile -> k_elastic_rk
    // Yee E and H: component c of E lives on the c-edges, of H on the c-faces
    F3 E_in, E_x, E_acc, E_out, H_in, H_x, H_acc, H_out;
    // Drude polarisation currents of the three poles (cell arrays)
    F3 jp_in[3], jp_x[3], jp_acc[3], jp_out[3];
    // compensation words of the mixed form (null in the FP64 form)
    F3 m_cmp, p_cmp, q_cmp, u_cmp, v_cmp, E_cmp, H_cmp, a1_cmp, a2_cmp, jp_cmp[3];
    // static and external fields
    F3 Hstat, Estat, Hnu;
    // face-normal displacement gradients of the current state, written by
    // k_face_grad for the strain output: fg[3*d + a] = d u_a / d x_d on the
    // cell's -d face
    R* fg[9];
    // crystal-frame cell strain of the stage displacement (Dexx_crt ...),
    // written by k_elastic_tile for ferromagnetic and ferroelectric cells and
    // read by the LLG and TDGL kernels of the same stage; null when unused
    R* strain_c[6];
    // optional static inputs (null when absent): static strain and static
    // eigenstrain in the crystal frame
    const R* eps0_c[6];
    const R* eig0_c[6];
    // Liao absorbing-boundary history: 4 slots of planes k=1..4 of u
    // (3 comps), plus the last boundary value written on plane 0
    R* liao_hist;
    R* liao_last;
    // input of the next magnetostatic transform (M = Ms m of the stage
    // output), written by the ferromagnet's LLG kernel when it covers the
    // whole grid and the run has no antiferromagnet; null otherwise (a
    // separate source kernel then forms it)
    R* msrc;
    // flexoelectric scratch (null without flexoelectricity), written by
    // k_flexo_prep at the start of each stage from the stage state: sg = the
    // global-frame cell strain of the stage displacement (Dexx_glb ...), pge =
    // the polarisation-gradient combinations the dynamic eigenstrain uses
    // (dpx/dx, dpy/dy, dpz/dz, dpy/dz + dpz/dy, dpx/dz + dpz/dx,
    // dpy/dx + dpx/dy; zero outside ferroelectric cells)
    R* sg[6];
    R* pge[6];
    // geometry / materials / time
    const uint8_t* mid;
    const DevMatT<R>* mats;
    const StepDrive* drive;
    const unsigned long long* step;   // index of the step being computed (0-based)
    unsigned long long drive_mask;    // drive ring holds drive_mask+1 steps
    const R* jf_kfac;            // per-k spatial factor of J_f types 1,2
    // spin pumping: per-k coefficient coeff_Js * coeff_L of the inverse-spin-
    // Hall current and the source plane of layer k (-1: no current)
    const R* ishe_coef;
    const int* ishe_src;
    // material class of every E edge, per component (Params::em_cls)
    const uint8_t* ecls[3];
};
using StageIO = StageIOT<double>;

// time-dependent values of RK stage s of the step being computed
template <class R>
__device__ inline const StageDrive& stage_drive(const StageIOT<R>& io, int s) {
    return io.drive[(*io.step) & io.drive_mask].st[s];
}

// ---------------------------------------------------------------------------
// Mixed-form RK4 helpers (R = float)
// ---------------------------------------------------------------------------

// a + b = s + e exactly (Knuth's TwoSum: six additions, no assumption on the
// magnitudes of a and b).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    const float bp = s - a;
    const float ap = s - bp;
    e = (a - ap) + (b - bp);
}

// RK4 combination of one state scalar: stage states X + d/2, X + d/2, X + d;
// A accumulates d1/6 + d2/3 + d3/3; the last stage forms A + d4/6 + C and adds
// it to X error-free, so the step value keeps about 48 significant bits while
// every array stays FP32.
template <int S>
__device__ __forceinline__ void rk_mixed(float xv, float d, float* out, float* acc, float* cmp, int e) {
    if (S == 0) { out[e] = xv + d * 0.5f; acc[e] = d * (1.f / 6.f); }
    else if (S == 1) { out[e] = xv + d * 0.5f; acc[e] = acc[e] + d * (1.f / 3.f); }
    else if (S == 2) { out[e] = xv + d; acc[e] = acc[e] + d * (1.f / 3.f); }
    else {
        float sum, err;
        two_sum(xv, (acc[e] + d * (1.f / 6.f)) + cmp[e], sum, err);
        acc[e] = sum;
        cmp[e] = err;
    }
}

// rk_mixed with the accumulator (stages 1..3) and compensation (last stage)
// already loaded into av and cv, so that a kernel can issue the loads of
// several scalars before the first of their stores
template <int S>
__device__ __forceinline__ void rk_mixed_v(float xv, float av, float cv, float d, float* out, float* acc, float* cmp,
                                           int e) {
    if (S == 0) { out[e] = xv + d * 0.5f; acc[e] = d * (1.f / 6.f); }
    else if (S == 1) { out[e] = xv + d * 0.5f; acc[e] = av + d * (1.f / 3.f); }
    else if (S == 2) { out[e] = xv + d; acc[e] = av + d * (1.f / 3.f); }
    else {
        float sum, err;
        two_sum(xv, (av + d * (1.f / 6.f)) + cv, sum, err);
        acc[e] = sum;
        cmp[e] = err;
    }
}

// |m| = 1 for a stage state (FP32)
__device__ __forceinline__ void renorm3(float& x, float& y, float& z) {
    // a zero vector stays zero (a ferromagnetic cell the deck leaves at m = 0
    // keeps it, as the reference's unnormalised update does)
    const float s2 = x * x + y * y + z * z;
    const float inv = s2 > 0.f ? 1.f / sqrtf(s2) : 0.f;
    x = x * inv; y = y * inv; z = z * inv;
}

// |x + c| = 1 for a compensated step value.  delta = |x + c|^2 - 1 is formed
// from exact squares (FMA residuals) and error-free sums, so its leading bits
// survive although it lies far below one ulp of 1; then x + c is scaled by
// 1 - delta/2 + 3 delta^2/8 and re-split into a rounded value and its error.
__device__ inline void renorm_pair(float x[3], float c[3]) {
    float p[3], e[3];
#pragma unroll
    for (int a = 0; a < 3; a++) { p[a] = x[a] * x[a]; e[a] = __fmaf_rn(x[a], x[a], -p[a]); }
    float s1, t1, s2, t2;
    two_sum(p[0], p[1], s1, t1);
    two_sum(s1, p[2], s2, t2);
    const float xc = x[0] * c[0] + x[1] * c[1] + x[2] * c[2];
    const float delta = (s2 - 1.f) + (((t1 + t2) + (e[0] + e[1] + e[2])) + 2.f * xc);
    if (!(fabsf(delta) < 1e-3f)) {
        // far from unit length (not reached from a unit initial state): plain scaling
        float v[3] = {x[0] + c[0], x[1] + c[1], x[2] + c[2]};
        renorm3(v[0], v[1], v[2]);
#pragma unroll
        for (int a = 0; a < 3; a++) { x[a] = v[a]; c[a] = 0.f; }
        return;
    }
    const float g = delta * (-0.5f + 0.375f * delta);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float sum, err;
        two_sum(x[a], c[a] + g * x[a], sum, err);
        x[a] = sum;
        c[a] = err;
    }
}

}  // namespace gf
