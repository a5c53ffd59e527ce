// Kernel launch helper: every launch of the engine goes through launch(), so
// that launch failures are checked in one place.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace gf {

inline unsigned blocks_for(long n, int threads) {
    long b = (n + threads - 1) / threads;
    return (unsigned)(b > 0 ? b : 1);
}

template <class Kernel, class... Args>
inline cudaError_t launch(Kernel k, dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    k<<<grid, block, smem, s>>>(args...);
    return cudaGetLastError();
}

// Asynchronous 8-byte global -> shared copy (cp.async, sm_80 and later).
// The data is visible to the issuing thread after cp_async_wait_all() and
// to the block after a barrier that follows it.
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// one element of a real array (8 bytes for FP64, 4 for FP32)
__device__ __forceinline__ void cp_async_elem(double* smem_dst, const double* gsrc) { cp_async8(smem_dst, gsrc); }
__device__ __forceinline__ void cp_async_elem(float* smem_dst, const float* gsrc) { cp_async4(smem_dst, gsrc); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Dynamic shared memory of a block-cooperative kernel (128-byte aligned:
// TMA destinations sit at fixed offsets from it).
#define GF_EXTERN_SMEM(T, name) extern __shared__ __align__(128) T name[]

// ---- mbarrier and TMA (cp.async.bulk.tensor) helpers, sm_90 and later ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes initialised mbarriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// wait for phase `parity` of the barrier to complete, giving up after
// `limit` polls (each try_wait itself blocks for a bounded time)
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned limit) {
    for (unsigned i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// one tiled 3-D tensor copy global -> this CTA's shared memory, completing
// on `bar` (no multicast); x is the innermost coordinate and must put the
// box start on a 16-byte boundary
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Launch of a block-cooperative kernel (one that synchronises its threads
// with __syncthreads and carries per-thread state across the barriers).
template <class Kernel, class... Args>
inline cudaError_t launch_tiled(Kernel k, dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    return launch(k, grid, block, smem, s, args...);
}

}  // namespace gf
