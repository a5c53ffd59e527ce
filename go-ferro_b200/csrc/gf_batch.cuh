// Batched sweep kernels of the mixed form: the stage kernels of many engines
// (uneven grids) in one launch per stage phase.
//
// A stage of a ferroelectric + elastodynamics + FDTD engine is a few phases
// whose kernels depend only on the phases before:
//   A: elastic tile (stress divergence), TDGL, Yee update
//   B: elastic RK update, the first Mur boundary of E  (read A's outputs)
//   C: elastic boundary planes (after the RK update), the second Mur boundary
//   D: the third Mur boundary
// (the Mur faces of x, y and z share their corner edges and read the planes
// next to them, so an engine's directions run in order x, y, z, one phase
// each, as the per-engine kernels do).
// k_batch_phase<S, PH> runs a phase of stage S for every engine of a batch:
// its blocks are work items (engine, kind, block coordinates) in a list built
// on the host, longest kinds first; each block reads its engine's parameters
// and stage buffers from the engine table (read-only, cached) and runs the
// kind's body —
// the same device functions the per-engine kernels run (elastic_tile_body,
// fe_body, em_fused_body, elastic_rk_body, em_mur_body, elastic_bc_body), so
// the arithmetic is the per-engine kernels'.  Small grids share the GPU
// within one launch instead of occupying it one after another.
#pragma once

#include "gf_elastic.cuh"
#include "gf_em.cuh"
#include "gf_fe.cuh"

namespace gf {

enum BatchKind : int { BK_TILE = 0, BK_EM = 1, BK_FE = 2, BK_RK = 3, BK_MUR_X = 4, BK_MUR_Y = 5, BK_MUR_Z = 6, BK_BC = 7 };

// one engine of a batch, in device memory
struct BatchInst {
    Params P;
    StageIOT<float> io[2][4];          // [step parity][stage]
    const EmCls<float>* cls;
    int ncls, nmat, el_chunk, el_cubic;
    unsigned long long* step;          // the engine's step counter
};

// one block of a phase launch
struct BatchItem {
    int inst, kind, bx, by, bz;
};

// PH: 0 = phase A (all of its kinds), 1 = the later phases (RK update, Mur
// and elastic boundaries), 3 = phase A tile items only, 4 = phase A Yee
// items only, 5 = phase A TDGL items only (one body per kernel: no register
// pressure from the others)
#ifndef GF_BATCH_TILE_MINB
#define GF_BATCH_TILE_MINB 3
#endif
template <int S, int PH>
__global__ void __launch_bounds__(256, PH == 3 ? GF_BATCH_TILE_MINB : 4) k_batch_phase(const BatchInst* __restrict__ insts, const BatchItem* __restrict__ items,
                                                        int parity, const __grid_constant__ ETileMaps tm) {
    GF_EXTERN_SMEM(unsigned char, smem_raw);
    const BatchItem it = items[blockIdx.x];
    const BatchInst& g = insts[it.inst];
    const Params& P = g.P;
    const StageIOT<float>& io = g.io[parity][S];
    auto tile = [&]() {
        if (g.el_cubic) elastic_tile_body<S, true, float>(P, io, g.el_chunk, g.nmat, tm, it.bx, it.by, it.bz, smem_raw);
        else elastic_tile_body<S, false, float>(P, io, g.el_chunk, g.nmat, tm, it.bx, it.by, it.bz, smem_raw);
    };
    auto yee = [&]() {
        EmMat<float>* mt = reinterpret_cast<EmMat<float>*>(smem_raw);
        EmCls<float>* cl = reinterpret_cast<EmCls<float>*>(smem_raw + kMaxMat * sizeof(EmMat<float>));
        em_fused_body<S, float>(P, io, g.nmat, g.cls, g.ncls, it.bx, it.by, mt, cl);
    };
    if constexpr (PH == 0) {
        if (it.kind == BK_TILE) tile();
        else if (it.kind == BK_EM) yee();
        else if (it.kind == BK_FE) fe_body<S, float, false>(P, io, it.bx, it.by);
    } else if constexpr (PH == 3) {
        tile();
    } else if constexpr (PH == 4) {
        yee();
    } else if constexpr (PH == 5) {
        fe_body<S, float, false>(P, io, it.bx, it.by);
    } else {
        if (it.kind == BK_RK) elastic_rk_body<S, float>(P, io, it.bx);
        else if (it.kind == BK_MUR_X) em_mur_body<S, 0, float>(P, io, it.bx);
        else if (it.kind == BK_MUR_Y) em_mur_body<S, 1, float>(P, io, it.bx);
        else if (it.kind == BK_MUR_Z) em_mur_body<S, 2, float>(P, io, it.bx);
        else if (it.kind == BK_BC) elastic_bc_body<S, float>(P, io, it.bx);
    }
}

// every engine's step counter + 1 (after the fourth stage)
static __global__ void k_batch_step_inc(const BatchInst* __restrict__ insts, int count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) *insts[t].step = *insts[t].step + 1ull;
}

// shared memory of a phase-A block: the elastic tile's, or the Yee
// kernel's two tables
inline size_t batch_smem_bytes(int nmat) {
    const size_t em = kMaxMat * sizeof(EmMat<float>) + kEmMaxCls * sizeof(EmCls<float>);
    const size_t tile = etile::smem_bytes<float>(nmat);
    return tile > em ? tile : em;
}

}  // namespace gf
