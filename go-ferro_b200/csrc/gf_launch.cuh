// Kernel launch helper: every launch of the engine goes through launch(), so
// that launch failures are checked in one place.
#pragma once

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

// Dynamic shared memory of a block-cooperative kernel.
#define GF_EXTERN_SMEM(T, name) extern __shared__ T name[]

// Launch of a block-cooperative kernel (one that synchronises its threads
// with __syncthreads and carries per-thread state across the barriers).
template <class Kernel, class... Args>
inline cudaError_t launch_tiled(Kernel k, dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    return launch(k, grid, block, smem, s, args...);
}

}  // namespace gf
