// dq_common.cuh — small shared device helpers: complex arithmetic, warp and
// block reductions, the bounded "last block reduces" ticket.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dq {

struct cd { double x, y; };   // complex128, same layout as dq_cdouble / cuDoubleComplex

__host__ __device__ __forceinline__ cd cmk(double x, double y) { cd r; r.x = x; r.y = y; return r; }
__device__ __forceinline__ cd cadd(cd a, cd b) { return cmk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cd csub(cd a, cd b) { return cmk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cd cmul(cd a, cd b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ cd cscale(cd a, double s) { return cmk(a.x * s, a.y * s); }
__device__ __forceinline__ cd cconj(cd a) { return cmk(a.x, -a.y); }
__device__ __forceinline__ double cabs2(cd a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ cd cdiv(cd a, cd b) {
    double d = b.x * b.x + b.y * b.y;
    return cmk((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block of a per-thread double; result valid in thread 0.
// `scratch` needs blockDim.x/32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) scratch[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        r = lane < nw ? scratch[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Ticket for the "last block finishes the reduction" pattern.  Every block
// publishes its partial, fences, and takes a ticket; the block that draws
// the last ticket sums all partials in block order (deterministic) and resets
// the counter for the next launch.  No block ever waits on another.
// a GPU-scope acquire load (the partner of a fence + atomic by another block)
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool last_block_ticket(unsigned int* counter, unsigned int nblocks) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(counter, 1u);
        is_last = (t == nblocks - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// Raises a kernel's dynamic shared-memory limit to at least `bytes` and never
// lowers it.  The limit is one attribute of the function for the whole device,
// shared by every context and call there, so a context with a smaller Krylov
// dimension or window must not shrink what another one launches with.
template <typename F>
inline cudaError_t raise_smem_limit(F* f, int bytes) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
    if (a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace dq
