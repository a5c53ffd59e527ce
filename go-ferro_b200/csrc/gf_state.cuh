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
#pragma once

#include "gf_common.cuh"

namespace gf {

struct F3 { double* c[3]; };

struct StageIO {
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
    // static and external fields
    F3 Hstat, Estat, Hnu;
    // face-normal displacement gradients of the current state, written by
    // k_face_grad for the strain output: fg[3*d + a] = d u_a / d x_d on the
    // cell's -d face
    double* fg[9];
    // crystal-frame cell strain of the stage displacement (Dexx_crt ...),
    // written by k_elastic_tile for ferromagnetic and ferroelectric cells and
    // read by the LLG and TDGL kernels of the same stage; null when unused
    double* strain_c[6];
    // optional static inputs (null when absent): static strain and static
    // eigenstrain in the crystal frame
    const double* eps0_c[6];
    const double* eig0_c[6];
    // Liao absorbing-boundary history: 4 slots of planes k=1..4 of u
    // (3 comps), plus the last boundary value written on plane 0
    double* liao_hist;
    double* liao_last;
    // geometry / materials / time
    const uint8_t* mid;
    const DevMat* mats;
    const StepDrive* drive;
    const unsigned long long* step;   // index of the step being computed (0-based)
    unsigned long long drive_mask;    // drive ring holds drive_mask+1 steps
    const double* jf_kfac;            // per-k spatial factor of J_f types 1,2
};

// time-dependent values of RK stage s of the step being computed
__device__ inline const StageDrive& stage_drive(const StageIO& io, int s) {
    return io.drive[(*io.step) & io.drive_mask].st[s];
}

}  // namespace gf
