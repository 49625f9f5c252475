// dq_batched.cuh — data structures and device helpers of the batched
// ensemble workspace, shared by the ensemble path (dq_batched.cu) and the
// adjoint (dq_adjoint.cu).
#pragma once
#include <cuda.h>

#include <functional>
#include <vector>

#include "dq_internal.h"

namespace dq {

constexpr int kBThreads = 256;
constexpr int kMaxTC = 64;
constexpr int kMaxCtasPerChunk = 4096;
// CTAs per SM of the streaming per-row kernels (noise, axpy, combine): one
// wave of 256-thread CTAs at their ~64 registers per thread (4 resident per
// SM); measured on the tube, 2, 3, 8 and 16 were all slower (small systems
// take twice as many, see batched_set_tiling)
constexpr int kStreamCtasPerSm = 4;
constexpr int kMCheckStride = 4;   // adaptive Krylov dimension: checks at m_min, m_min + 4, ... below m

// ---- vector access of TPT consecutive complex values ----------------------
template <typename Real, int TPT> struct VL;
template <> struct VL<float, 1> { using T = float2; };
template <> struct VL<float, 2> { using T = float4; };
template <> struct VL<double, 1> { using T = double2; };
template <> struct VL<float, 4> { using T = float4; };   // two per value

template <typename Real, int TPT>
struct CV { Real v[2 * TPT]; };   // interleaved (re, im) per trajectory

template <typename Real, int TPT, bool kLdg>
__device__ __forceinline__ CV<Real, TPT> ldv(const Real* base, size_t idx) {
    using T = typename VL<Real, TPT>::T;
    const T* p = reinterpret_cast<const T*>(base + 2 * idx);
    CV<Real, TPT> v;
    if constexpr (TPT == 4) {
        static_assert(sizeof(Real) == 4, "4 trajectories per lane: complex64 only");
        const T a = kLdg ? __ldg(p) : p[0];
        const T b = kLdg ? __ldg(p + 1) : p[1];
        v.v[0] = a.x; v.v[1] = a.y; v.v[2] = a.z; v.v[3] = a.w;
        v.v[4] = b.x; v.v[5] = b.y; v.v[6] = b.z; v.v[7] = b.w;
        return v;
    }
    T t = kLdg ? __ldg(p) : *p;
    if constexpr (TPT == 2) {
        v.v[0] = t.x; v.v[1] = t.y; v.v[2] = t.z; v.v[3] = t.w;
    } else {
        v.v[0] = t.x; v.v[1] = t.y;
    }
    return v;
}

// last read of a value before it is overwritten: evict-first (ld.global.cs)
template <typename Real, int TPT>
__device__ __forceinline__ CV<Real, TPT> ldv_cs(const Real* base, size_t idx) {
    using T = typename VL<Real, TPT>::T;
    const T* p = reinterpret_cast<const T*>(base + 2 * idx);
    CV<Real, TPT> v;
    if constexpr (TPT == 4) {
        const T a = __ldcs(p), b = __ldcs(p + 1);
        v.v[0] = a.x; v.v[1] = a.y; v.v[2] = a.z; v.v[3] = a.w;
        v.v[4] = b.x; v.v[5] = b.y; v.v[6] = b.z; v.v[7] = b.w;
        return v;
    }
    const T t = __ldcs(p);
    if constexpr (TPT == 2) {
        v.v[0] = t.x; v.v[1] = t.y; v.v[2] = t.z; v.v[3] = t.w;
    } else {
        v.v[0] = t.x; v.v[1] = t.y;
    }
    return v;
}

template <typename Real, int TPT>
__device__ __forceinline__ void stv(Real* base, size_t idx, const CV<Real, TPT>& v) {
    using T = typename VL<Real, TPT>::T;
    T t;
    if constexpr (TPT == 4) {
        T* q = reinterpret_cast<T*>(base + 2 * idx);
        q[0] = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
        q[1] = make_float4(v.v[4], v.v[5], v.v[6], v.v[7]);
        return;
    } else if constexpr (TPT == 2) {
        t.x = v.v[0]; t.y = v.v[1]; t.z = v.v[2]; t.w = v.v[3];
    } else {
        t.x = v.v[0]; t.y = v.v[1];
    }
    *reinterpret_cast<T*>(base + 2 * idx) = t;
}

// acc += c * y for TPT complex values; packed FP32x2 FMA on sm_100 for the
// complex64 path (one instruction per complex element)
template <typename Real, int TPT>
__device__ __forceinline__ void cfma(CV<Real, TPT>& acc, Real c, const CV<Real, TPT>& y) {
    if constexpr (sizeof(Real) == 4) {
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            const float2 r = __ffma2_rn(make_float2(c, c), make_float2(y.v[2 * t], y.v[2 * t + 1]),
                                        make_float2(acc.v[2 * t], acc.v[2 * t + 1]));
            acc.v[2 * t] = r.x;
            acc.v[2 * t + 1] = r.y;
        }
    } else {
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            acc.v[2 * t] = fma(c, y.v[2 * t], acc.v[2 * t]);
            acc.v[2 * t + 1] = fma(c, y.v[2 * t + 1], acc.v[2 * t + 1]);
        }
    }
}

struct BatchedScalars {
    double* alpha;    // [kMaxL][B] complex (2 doubles)
    double* beta;     // [kMaxL][B]
    double* sc;       // [kMaxL][B]; q_j = sc_j r_j
    double* yt;       // [kMaxL][B] complex combine weights y_{j-1} sc_j
    double* nav;      // [B] ||H q_{m+1}||
    double* norm2;    // [B] ||psi||^2 of the stored (unnormalised) psi
    double* partial;  // 2 regions of [chunks][gx][TC][2]
    unsigned int* tickets;  // [8][chunks] + step ticket
    int* status;      // [1]
    int* step;        // [1] current step index
    double* corr;     // [(max_steps+1)][chunks][2]
    // adaptive Krylov dimension (null when the dimension is fixed): the
    // dimension chosen per trajectory (0 = not yet), per chunk whether every
    // trajectory has chosen (its remaining iterations exit at once) and the
    // largest choice
    int* mtraj;       // [B]
    int* cdone;       // [chunks]
    int* mchunk;      // [chunks]
};

// Iteration kernels return at once for a chunk whose trajectories all chose
// their Krylov dimension (uniform over the chunk's CTAs, before any barrier).
__device__ __forceinline__ bool chunk_converged(const BatchedScalars& S, int chunk) {
    return S.cdone != nullptr && S.cdone[chunk] != 0;
}

// Thread -> (row lane, trajectory lane) map and the CTA's row range.
template <int TPT>
struct Tile {
    int tr, rl, RPC, b0, r0, r1, chunk, bx;
    // chunk_fast: consecutive blocks take the chunks of one row range (the
    // linear block id runs over chunks first), so the pieces of every site's
    // trajectory row are read at about the same time; bx is the row-range
    // index either way (the reduction's partial slot).
    __device__ __forceinline__ Tile(int TC, int rows_per_cta, int n, int cy0 = 0, bool chunk_fast = false) {
        const int TPR = TC / TPT;
        tr = threadIdx.x % TPR;
        rl = threadIdx.x / TPR;
        RPC = blockDim.x / TPR;
        if (chunk_fast) {
            const int L = blockIdx.y * gridDim.x + blockIdx.x;
            chunk = L % gridDim.y + cy0;
            bx = L / gridDim.y;
        } else {
            chunk = blockIdx.y + cy0;
            bx = blockIdx.x;
        }
        b0 = chunk * TC + tr * TPT;
        r0 = bx * rows_per_cta;
        r1 = min(n, r0 + rows_per_cta);
    }
};

}  // namespace dq

// Row-blocked column-union form of the off-diagonal couplings: block k holds
// rows [kR, kR+R); its entries are the sorted union of those rows' neighbour
// columns, each with R coefficients (zero where a row lacks that column), so
// one gathered trajectory row serves R output rows.
struct BlockFmt {
    int R = 0, nb = 0;
    int max_block = 0;       // most union entries (records) of one block
    size_t nunion = 0;
    bool packed = false;     // 16-byte records {col, c0, c1, c2}, blocks padded to 4 entries
    int* bptr = nullptr;     // nb + 1
    int* bcol = nullptr;     // nunion
    void* bcoef = nullptr;   // nunion x R (Real)
};

struct dq::BatchedState {
    int B = 0, TC = 0, TPT = 2, chunks = 0, gx = 0, rpc = 0, ctas_per_sm = 2;
    int R = 4, gxs = 0, bpc = 0;          // SpMM: rows per block, CTAs per chunk, blocks per CTA
    int staged = 0;                       // 1: TMA-staged shared-memory window SpMM
    int groups = 1;                       // trajectory groups iterated one after another
    int halo = 0, wmask = 0, rpc_win = 0, gxw = 0, bw = 0;   // window geometry, matrix bandwidth
    size_t win_smem = 0;
    std::vector<CUtensorMap> tmaps;       // one per slab (window variant)
    // fused iteration (staged = 2): second SpMM output buffer, tensor maps of
    // slabs 0..m and of wB (boxes of f_sr rows), halo blocks, stages, grid
    void* wB = nullptr;
    std::vector<CUtensorMap> fmaps;
    int f_sr = 0, f_hb = 0, f_D = 2, f_rpc = 0, f_gx = 0, f_rb = 1;   // f_rb: blocks per warp (staged = 4)
    size_t f_smem = 0;
    ::BlockFmt fmt[5];                    // R = 1, 2, 3, 4, 8 (built on demand)
    bool fmt_borrowed = false;            // fmt belongs to another workspace
    int sms = 148;
    bool mixed = true;
    void* slabs = nullptr;      // (m+2) slabs (slab 0 = w)
    void* diag = nullptr;       // Real [n][B]
    double* eps = nullptr;      // [n][B]
    double* deps = nullptr;     // [n][B]
    double* zzD = nullptr;      // ZZ noise sums of a block of steps [kZZBlock][n][B]
    int* zz_start = nullptr;    // first step of that block
    dq::BatchedScalars s{};
    double* scal_mem = nullptr;
    size_t partial_cap = 0;     // doubles per partial region
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace dq {

// ---------------------------------------------------------------------------
// per-chunk reduction of TC complex partials per block
// ---------------------------------------------------------------------------
// ar/ai: this thread's partials for its TPT trajectories.  Threads of the
// same trajectory lane are summed in shared memory; the block partial goes to
// partial[chunk][blockIdx.x][TC]; the last block of the chunk sums the
// gridDim.x partials in block order.  Returns true in that block, with the
// chunk's totals in red_out[0..TC).
// chunk_reduce_s takes its shared scratch (kBThreads * 2 double2) from the
// caller; chunk_reduce declares it.
template <int TPT>
__device__ __forceinline__ bool chunk_reduce_s(const double (&ar)[TPT], const double (&ai)[TPT], int TC,
                                               double* partial, unsigned int* ticket, double2* red_out, int chunk,
                                               double2* sm, int bx = -1) {
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
#pragma unroll
    for (int t = 0; t < TPT; ++t) sm[rl * TC + tr * TPT + t] = make_double2(ar[t], ai[t]);
    __syncthreads();
    double* mypart = partial + ((size_t)chunk * gridDim.x + (bx < 0 ? (int)blockIdx.x : bx)) * TC * 2;
    if (threadIdx.x < TC) {
        double sr = 0.0, si = 0.0;
        for (int r = 0; r < RPC; ++r) {
            double2 v = sm[r * TC + threadIdx.x];
            sr += v.x;
            si += v.y;
        }
        mypart[2 * threadIdx.x] = sr;
        mypart[2 * threadIdx.x + 1] = si;
    }
    bool last = last_block_ticket(ticket + chunk, gridDim.x);
    if (last) {
        // all threads of the last block: `per` threads per trajectory each sum
        // a strided share of the block partials, then the shares are added in
        // a fixed order (deterministic, no serial walk over every partial)
        const int per = blockDim.x / TC;
        const int tl = threadIdx.x % TC, part = threadIdx.x / TC;
        const double* base = partial + (size_t)chunk * gridDim.x * TC * 2;
        double sr = 0.0, si = 0.0;
#pragma unroll 4
        for (unsigned int g = part; g < gridDim.x; g += per) {
            const double2 v = __ldcg(reinterpret_cast<const double2*>(base + ((size_t)g * TC + tl) * 2));
            sr += v.x;
            si += v.y;
        }
        __syncthreads();   // sm is reused for the shares
        sm[part * TC + tl] = make_double2(sr, si);
        __syncthreads();
        if (threadIdx.x < TC) {
            double ar2 = 0.0, ai2 = 0.0;
            for (int q = 0; q < per; ++q) {
                ar2 += sm[q * TC + threadIdx.x].x;
                ai2 += sm[q * TC + threadIdx.x].y;
            }
            red_out[threadIdx.x] = make_double2(ar2, ai2);
        }
        if (threadIdx.x == 0) ticket[chunk] = 0;
        __syncthreads();
    }
    return last;
}

template <int TPT>
__device__ __forceinline__ bool chunk_reduce(const double (&ar)[TPT], const double (&ai)[TPT], int TC,
                                             double* partial, unsigned int* ticket, double2* red_out, int chunk,
                                             int bx = -1) {
    __shared__ double2 sm[kBThreads * 2];
    return chunk_reduce_s<TPT>(ar, ai, TC, partial, ticket, red_out, chunk, sm, bx);
}

}  // namespace dq

namespace dq {
// host functions of dq_batched.cu used by the adjoint
BatchedState* batched_alloc_ws(dq_ctx* c, int B, bool mixed, dq_status* st);
void batched_free_ws(BatchedState* bs);
dq_status batched_iteration(dq_ctx* c, BatchedState* ws, int j);
dq_status batched_mirror_tiling(dq_ctx* c, BatchedState* dst);
dq_status batched_step_eager(dq_ctx* c, const std::function<void()>* after_noise, bool skip_pop);
}  // namespace dq
