// Batched sweep kernels of the mixed form: the stage kernels of many engines
// (uneven grids) in one launch per stage phase.
//
// A stage of a ferroelectric + elastodynamics + FDTD engine is a few phases
// whose kernels depend only on the phases before:
//   A: elastic tile (stress divergence), TDGL, Yee update
//   B: elastic RK update, the first Mur boundary of E  (read A's outputs)
//   C: elastic boundary planes (after the RK update; none where the RK
//      update applies them itself, Params::el_bc_fused), the second Mur
//      boundary
//   D: the third Mur boundary
// (the Mur faces of x, y and z share their corner edges and read the planes
// next to them, so an engine's directions run in order x, y, z, one phase
// each, as the per-engine kernels do).
// k_batch_phase<S, PH> runs a phase of stage S for every engine of a batch
// (k_batch_persistent runs all phases of all four stages in one cooperative
// launch, with grid barriers between them):
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
// work item `it` of a phase-PH list, run by the whole block
template <int S, int PH>
__device__ __forceinline__ void batch_item(const BatchInst* __restrict__ insts, const BatchItem it, int parity, const ETileMaps& tm,
                                           unsigned char* smem_raw) {
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

template <int S, int PH>
__global__ void __launch_bounds__(256, PH == 3 ? GF_BATCH_TILE_MINB : 4) k_batch_phase(const BatchInst* __restrict__ insts, const BatchItem* __restrict__ items,
                                                        int parity, const __grid_constant__ ETileMaps tm) {
    GF_EXTERN_SMEM(unsigned char, smem_raw);
    batch_item<S, PH>(insts, items[blockIdx.x], parity, tm, smem_raw);
}

// Grid-wide barrier of a cooperative launch (every block resident):
// bar[0] counts the blocks that arrived, bar[1] is the generation.  The last
// block to arrive resets the count and advances the generation; the others
// poll the generation.  Writes before the barrier are made visible to
// every block after it by the fences around the arrival.  The poll is
// bounded (2^22 polls of >= 64 ns): a block that gives up sets bit 2 of
// *err and returns false, and the kernel then returns (every later barrier
// gives up the same way), so a fault cannot hang the GPU.
__device__ inline bool batch_grid_sync(unsigned* bar, unsigned* err) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned polls = 0;
            while (*gen == g0) {
                if (++polls > (1u << 22)) {
                    if (err) atomicOr(err, 2u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// one work item of kind K as a function of its own (not inlined), so that
// the persistent kernel, which holds every kind of every stage, allocates
// registers per kind instead of for all of them at once
template <int S, int K>
__device__ __noinline__ void batch_kind_call(const BatchInst* __restrict__ insts, const BatchItem it, int parity, const ETileMaps* tm,
                                             unsigned char* smem_raw) {
    const BatchInst& g = insts[it.inst];
    const Params& P = g.P;
    const StageIOT<float>& io = g.io[parity][S];
    if constexpr (K == BK_TILE) {
        if (g.el_cubic) elastic_tile_body<S, true, float>(P, io, g.el_chunk, g.nmat, *tm, it.bx, it.by, it.bz, smem_raw);
        else elastic_tile_body<S, false, float>(P, io, g.el_chunk, g.nmat, *tm, it.bx, it.by, it.bz, smem_raw);
    } else if constexpr (K == BK_EM) {
        EmMat<float>* mt = reinterpret_cast<EmMat<float>*>(smem_raw);
        EmCls<float>* cl = reinterpret_cast<EmCls<float>*>(smem_raw + kMaxMat * sizeof(EmMat<float>));
        em_fused_body<S, float>(P, io, g.nmat, g.cls, g.ncls, it.bx, it.by, mt, cl);
    } else if constexpr (K == BK_FE) {
        fe_body<S, float, false>(P, io, it.bx, it.by);
    } else if constexpr (K == BK_RK) {
        elastic_rk_body<S, float>(P, io, it.bx);
    } else if constexpr (K == BK_MUR_X) {
        em_mur_body<S, 0, float>(P, io, it.bx);
    } else if constexpr (K == BK_MUR_Y) {
        em_mur_body<S, 1, float>(P, io, it.bx);
    } else if constexpr (K == BK_MUR_Z) {
        em_mur_body<S, 2, float>(P, io, it.bx);
    } else {
        elastic_bc_body<S, float>(P, io, it.bx);
    }
}
template <int S>
__device__ __forceinline__ void batch_item_call(const BatchInst* __restrict__ insts, const BatchItem it, int parity, const ETileMaps* tm,
                                                unsigned char* smem_raw) {
    switch (it.kind) {
        case BK_TILE: batch_kind_call<S, BK_TILE>(insts, it, parity, tm, smem_raw); break;
        case BK_EM: batch_kind_call<S, BK_EM>(insts, it, parity, tm, smem_raw); break;
        case BK_FE: batch_kind_call<S, BK_FE>(insts, it, parity, tm, smem_raw); break;
        case BK_RK: batch_kind_call<S, BK_RK>(insts, it, parity, tm, smem_raw); break;
        case BK_MUR_X: batch_kind_call<S, BK_MUR_X>(insts, it, parity, tm, smem_raw); break;
        case BK_MUR_Y: batch_kind_call<S, BK_MUR_Y>(insts, it, parity, tm, smem_raw); break;
        case BK_MUR_Z: batch_kind_call<S, BK_MUR_Z>(insts, it, parity, tm, smem_raw); break;
        default: batch_kind_call<S, BK_BC>(insts, it, parity, tm, smem_raw); break;
    }
}

// stage S of the persistent step: phase A's items, then those of phases
// B, C and D (L holds them in that order), each phase ended by a grid
// barrier; blocks take items in strides of the grid
template <int S>
__device__ __forceinline__ bool batch_persist_stage(const BatchInst* __restrict__ insts, const BatchItem* __restrict__ A, int nA,
                                                    const BatchItem* __restrict__ L, int nB, int nC, int nD, int parity,
                                                    const ETileMaps& tm, unsigned char* smem_raw, unsigned* bar) {
    for (int i = blockIdx.x; i < nA; i += gridDim.x) {
        batch_item_call<S>(insts, A[i], parity, &tm, smem_raw);
        __syncthreads();   // the next item reuses the shared memory
    }
    if (!batch_grid_sync(bar, tm.err)) return false;
    const int n[3] = {nB, nC, nD};
    for (int q = 0; q < 3; q++) {
        if (n[q] == 0) continue;
        for (int i = blockIdx.x; i < n[q]; i += gridDim.x) batch_item_call<S>(insts, L[i], parity, &tm, smem_raw);
        L += n[q];
        if (!batch_grid_sync(bar, tm.err)) return false;
    }
    return true;
}

#ifdef GF_MIXED_TU
// One RK4 step of every engine of a batch in one cooperative launch: the
// four stages' phases over the work lists of the phase mode, separated by
// grid barriers instead of launches, then the engines' step counters.
// Launch with every block resident (cudaLaunchAttributeCooperative, at
// most the occupancy times the SM count).
#ifndef GF_BATCH_PERSIST_MINB
#define GF_BATCH_PERSIST_MINB 4
#endif
__global__ void __launch_bounds__(256, GF_BATCH_PERSIST_MINB) k_batch_persistent(const BatchInst* __restrict__ insts, int ninst,
                                                                             const BatchItem* __restrict__ A, int nA,
                                                                             const BatchItem* __restrict__ L, int nB, int nC, int nD,
                                                                             int parity, const __grid_constant__ ETileMaps tm,
                                                                             unsigned* bar) {
    GF_EXTERN_SMEM(unsigned char, smem_raw);
    if (!batch_persist_stage<0>(insts, A, nA, L, nB, nC, nD, parity, tm, smem_raw, bar)) return;
    if (!batch_persist_stage<1>(insts, A, nA, L, nB, nC, nD, parity, tm, smem_raw, bar)) return;
    if (!batch_persist_stage<2>(insts, A, nA, L, nB, nC, nD, parity, tm, smem_raw, bar)) return;
    if (!batch_persist_stage<3>(insts, A, nA, L, nB, nC, nD, parity, tm, smem_raw, bar)) return;
    // after the last barrier no block reads a step counter any more
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < ninst; t += blockDim.x) *insts[t].step = *insts[t].step + 1ull;
}
#endif  // GF_MIXED_TU

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
