// dq_batched.cu — the batched ensemble form: B trajectories share the
// coupling CSR, so the Krylov SpMV of the reference (cusparseZcsrmv,
// lanczosClass.cu:620-661, once per trajectory) becomes one SpMM that streams
// the off-diagonal structure once per iteration for all trajectories and adds
// every trajectory's fluctuating diagonal in registers.
//
// HBM layout (site-major, trajectory-minor, so one CSR column index fetches a
// contiguous run of trajectories):
//   slab j (j = 1..m+1): r_j[site][traj], complex64 (mixed) or complex128
//                        (fp64); q_j = sc_j[traj] * r_j (unnormalised Lanczos
//                        residuals, slab 1 = psi itself)
//   slab 0             : w[site][traj], SpMM output of the current iteration
//   d[site][traj]      : this step's diagonal, real (float or double)
//   eps, deps          : FP64 static energies and OU offsets [site][traj]
// Per-trajectory FP64 scalars live in [j][traj] arrays.
//
// Tiling: blockIdx.y picks a chunk of TC trajectories; blockIdx.x owns a
// CONTIGUOUS range of rows, so the neighbour rows one row gathers are the
// ones its predecessors just gathered and stay in L1.  A thread owns TPT
// consecutive trajectories of one row at a time (8- or 16-byte vector
// loads).  TC, TPT and CTAs per SM are chosen by dq_autotune.
// Per-trajectory reductions (alpha, beta, norms, correlation) go through
// per-chunk partials and a per-chunk last-block ticket: deterministic, no
// extra launch, no block ever waits for another.
//
// One time step (propagate.cu:199-259 for all trajectories at once):
//   k_noise_b, m x {k_spmm, k_axpy_beta}, k_spmm (norm), k_pade_b,
//   k_combine_b, k_pop_b
// captured once into a CUDA graph and replayed per step; the step index lives
// in device memory.
#include <climits>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cudaTypedefs.h>

#include "dq_batched.cuh"
#include "dq_internal.h"
#include "dq_rng.cuh"
#include "dq_tma.cuh"

namespace dq {

// The dynamic shared memory of a kernel begins right after its static shared
// memory, and only 16-byte alignment of that start is guaranteed, whatever the
// declaration says; TMA destinations need 128 bytes.  The TMA-fed kernels
// therefore round the start up themselves, from 128 bytes of padding that
// their launches add to the dynamic size (kSmemAlignPad).
constexpr size_t kSmemAlignPad = 128;
__device__ __forceinline__ unsigned char* align_smem128(unsigned char* p) {
    const uint32_t a = smem_u32(p);
    return p + ((128u - (a & 127u)) & 127u);
}

// Budget of the bounded mbarrier waits in SM cycles: kWaitCycles (about 2 s)
// unless a test lowers it through dq_debug_set_wait_cycles.  A negative value
// is a test mode: each ring-SpMM CTA first waits |value| cycles on a barrier
// that no copy completes, so its wait runs out for certain.  The drains after
// a timeout always use kWaitCycles.
__device__ long long g_dq_wait_cycles = kWaitCycles;

// the budget of the forms without the forced-timeout mode
__device__ __forceinline__ long long wait_budget() {
    const long long b = g_dq_wait_cycles;
    return b > 0 ? b : kWaitCycles;
}

// ---------------------------------------------------------------------------
__global__ void k_traj_init_b(int n, int B, int traj0, uint64_t seed, const double* __restrict__ h0,
                              const double* __restrict__ static_eps, double sigma_static,
                              const double* __restrict__ sigma, int noise, double* __restrict__ eps,
                              double* __restrict__ deps) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        for (int b = threadIdx.x; b < B; b += blockDim.x) {
            const size_t x = (size_t)i * B + b;
            const int g = traj0 + b;   // trajectory index of the whole ensemble (Philox key)
            double e;
            if (static_eps) e = static_eps[i];
            else e = __dadd_rn(__dmul_rn(sigma_static, normal(seed, P_STATIC, g, 0, i, 0)), h0[i]);
            eps[x] = e;
            deps[x] = (noise == DQ_NOISE_OU) ? __dmul_rn(sigma[i], normal(seed, P_OU_INIT, g, 0, i, 0)) : 0.0;
        }
    }
}

// ZZ noise sums of kZZBlock consecutive steps [start, start + kZZBlock) for
// every (site, trajectory): zzD[t][site][traj] = sum_osc c cos(omega (start +
// t) dt + phi), in oscillator order as two fused multiply-adds per term
// (gpuSysHelper.cu:134-177 sums c cos(omega t + phi) every step).  One
// thread per trajectory pair of a site draws both phases of an oscillator from
// one Philox block and reuses their sin/cos for all kZZBlock steps; the
// steps' factors (c cos(omega t), c sin(omega t)) come from a shared table
// filled 32 oscillators at a time.  The kernel leaves at once when the step
// about to run already lies in the stored block (start is *zz_start).
constexpr int kZZBlock = 16;
constexpr int kZZTile = 32;
constexpr int kZZThreads = 128;

__global__ void __launch_bounds__(kZZThreads, 4) k_zz_block_b(int n, int B, int traj0, uint64_t seed, ZZParams zz,
                                                          BatchedScalars S, const int* __restrict__ zz_start,
                                                          double* __restrict__ zzD) {
    const int step = *S.step, start = *zz_start;
    if (step >= start && step - start < kZZBlock) return;   // uniform over the grid
    __shared__ double fc[kZZTile][kZZBlock], fs[kZZTile][kZZBlock];
    const int hp = (B + 1) / 2;   // trajectory pairs per site
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = x < (long long)n * hp;
    const int site = active ? (int)(x / hp) : 0;
    const int b = active ? 2 * (int)(x % hp) : 0;
    const bool has1 = b + 1 < B;
    double a0[kZZBlock], a1[kZZBlock];
#pragma unroll
    for (int t = 0; t < kZZBlock; ++t) { a0[t] = 0.0; a1[t] = 0.0; }
    for (int o0 = 0; o0 < zz.n_osc; o0 += kZZTile) {
        const int no = min(kZZTile, zz.n_osc - o0);
        __syncthreads();
        for (int e = threadIdx.x; e < no * kZZBlock; e += blockDim.x) {
            const int o = e / kZZBlock, t = e % kZZBlock;
            zz_factors(zz.omega[o0 + o], zz.coeff[o0 + o], step + t, zz.dt, fc[o][t], fs[o][t]);
        }
        __syncthreads();
        if (active) {
            for (int o = 0; o < no; ++o) {
                float u0, u1;
                zz_phase_pair(seed, (uint32_t)((traj0 + b) >> 1), (uint32_t)site, (uint32_t)(o0 + o), u0, u1);
                double s0, c0, s1, c1;
                own_sincos_2pi((double)u0, s0, c0);
                own_sincos_2pi((double)u1, s1, c1);
#pragma unroll
                for (int t = 0; t < kZZBlock; ++t) {
                    const double cc = fc[o][t], cs = fs[o][t];
                    a0[t] = __fma_rn(-cs, s0, __fma_rn(cc, c0, a0[t]));
                    a1[t] = __fma_rn(-cs, s1, __fma_rn(cc, c1, a1[t]));
                }
            }
        }
    }
    if (!active) return;
    const size_t se = (size_t)n * B, xi = (size_t)site * B + b;
#pragma unroll
    for (int t = 0; t < kZZBlock; ++t) {
        zzD[t * se + xi] = a0[t];
        if (has1) zzD[t * se + xi + 1] = a1[t];
    }
}

// Records the block k_zz_block_b computed (run after it, so that no block of
// that kernel reads the new start).
__global__ void k_zz_mark(BatchedScalars S, int* zz_start) {
    const int step = *S.step, start = *zz_start;
    if (!(step >= start && step - start < kZZBlock)) *zz_start = step;
}

template <typename Real>
__global__ void k_set_psi0_b(int n, int B, const cd* __restrict__ psi0, Real* __restrict__ r1) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const cd p = psi0[i];
        for (int b = threadIdx.x; b < B; b += blockDim.x) {
            const size_t x = (size_t)i * B + b;
            r1[2 * x] = (Real)p.x;
            r1[2 * x + 1] = (Real)p.y;
        }
    }
}

// OU / Gaussian update of every trajectory's diagonal for this step
// (gpuSysHelper.cu:32-128 with Philox keys instead of shared cuRAND states)
template <typename Real, int TPT>
__global__ void __launch_bounds__(kBThreads) k_noise_b(int n, int B, int traj0, int TC, int rpc, int noise, int ns,
                                                      double subdt,
                                                      double sqrt_subdt, uint64_t seed,
                                                      const double* __restrict__ sigma,
                                                      const double* __restrict__ invtau,
                                                      const double* __restrict__ coeff,
                                                      const double* __restrict__ eps, double* __restrict__ deps,
                                                      Real* __restrict__ d, BatchedScalars S,
                                                      const double* __restrict__ zzD, const int* __restrict__ zz_start) {
    const Tile<TPT> T(TC, rpc, n, 0, true);
    const int step = *S.step;
    if (noise == DQ_NOISE_ZZ) {
        // eps + this step's row of the block of noise sums (k_zz_block_b)
        const double* D = zzD + (size_t)(step - *zz_start) * n * B;
        for (int row = T.r0 + T.rl; row < T.r1; row += T.RPC) {
            const size_t x = (size_t)row * B + T.b0;
#pragma unroll
            for (int t = 0; t < TPT; ++t) d[x + t] = (Real)__dadd_rn(D[x + t], eps[x + t]);
        }
        return;
    }
    for (int row = T.r0 + T.rl; row < T.r1; row += T.RPC) {
        if constexpr (TPT == 2) {
            // trajectories b0, b0+1 form one Philox pair (b0 is even)
            const size_t x = (size_t)row * B + T.b0;
            double v0, v1;
            if (noise == DQ_NOISE_OU) {
                double c0 = deps[x], c1 = deps[x + 1];
                ou_update_pair(c0, c1, invtau[row], coeff[row], subdt, sqrt_subdt, ns, seed, (traj0 + T.b0) >> 1, step,
                               row);
                deps[x] = c0;
                deps[x + 1] = c1;
                v0 = __dadd_rn(c0, eps[x]);
                v1 = __dadd_rn(c1, eps[x + 1]);
            } else if (noise == DQ_NOISE_GAUSS) {
                double z0, z1;
                normal_pair(seed, P_GAUSS, (traj0 + T.b0) >> 1, step, row, 0, z0, z1);
                v0 = __dadd_rn(__dmul_rn(z0, sigma[row]), eps[x]);
                v1 = __dadd_rn(__dmul_rn(z1, sigma[row]), eps[x + 1]);
            } else {
                v0 = eps[x];
                v1 = eps[x + 1];
            }
            d[x] = (Real)v0;
            d[x + 1] = (Real)v1;
        } else {
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                const int b = T.b0 + t;
                const size_t x = (size_t)row * B + b;
                double v;
                if (noise == DQ_NOISE_OU) {
                    double cur =
                        ou_update(deps[x], invtau[row], coeff[row], subdt, sqrt_subdt, ns, seed, traj0 + b, step, row);
                    deps[x] = cur;
                    v = __dadd_rn(cur, eps[x]);
                } else if (noise == DQ_NOISE_GAUSS) {
                    double xi = normal(seed, P_GAUSS, traj0 + b, step, row, 0);
                    v = __dadd_rn(__dmul_rn(xi, sigma[row]), eps[x]);
                } else {
                    v = eps[x];
                }
                d[x] = (Real)v;
            }
        }
    }
}

template <typename Real, int R>
__device__ __forceinline__ void ld_coef(const Real* __restrict__ base, int e, Real (&c)[R]) {
    const Real* p = base + (size_t)e * R;
    if constexpr (R == 1) {
        c[0] = __ldg(p);
    } else if constexpr (sizeof(Real) * R == 8) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        c[0] = t.x;
        c[1] = t.y;
    } else {
        constexpr int NV = (int)(sizeof(Real) * R / 16);
        constexpr int PER = 16 / (int)sizeof(Real);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(p) + v);
            union { float4 f; Real r[PER]; } u;
            u.f = t;
#pragma unroll
            for (int k = 0; k < PER; ++k) c[v * PER + k] = u.r[k];
        }
    }
}

// acc[i] += sum_p coef[p][i] * gather(col[p]) over the union entries
// [pb, pe) of one row block.  The columns and coefficients of the next G
// entries are loaded while the current G gather and accumulate, so the
// index loads leave the gather's dependency chain.
template <typename Real, int TPT, int R, int G, typename Gather>
__device__ __forceinline__ void union_loop(int pb, int pe, const int* __restrict__ bcol,
                                           const Real* __restrict__ bcoef, CV<Real, TPT> (&acc)[R],
                                           Gather gather) {
    if (pb >= pe) return;
    int cc[G];
    Real cf[G][R];
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const int p = min(pb + q, pe - 1);
        cc[q] = __ldg(bcol + p);
        ld_coef<Real, R>(bcoef, p, cf[q]);
    }
    for (int p0 = pb; p0 < pe; p0 += G) {
        const bool more = p0 + G < pe;
        int nc[G];
        Real nf[G][R];
        if (more) {
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int p = min(p0 + G + q, pe - 1);
                nc[q] = __ldg(bcol + p);
                ld_coef<Real, R>(bcoef, p, nf[q]);
            }
        }
        CV<Real, TPT> y[G];
#pragma unroll
        for (int q = 0; q < G; ++q) y[q] = gather(cc[q]);
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if (p0 + q < pe) {
#pragma unroll
                for (int i = 0; i < R; ++i) cfma<Real, TPT>(acc[i], cf[q][i], y[q]);
            }
        }
        if (more) {
#pragma unroll
            for (int q = 0; q < G; ++q) {
                cc[q] = nc[q];
#pragma unroll
                for (int i = 0; i < R; ++i) cf[q][i] = nf[q][i];
            }
        }
    }
}

template <int R> struct UnionGroup { static constexpr int G = R >= 4 ? 2 : 4; };

// Packed form (complex64, R <= 3): one 16-byte record {col, c0, c1, c2} per
// union entry, the block's record count a multiple of 4.  Two groups of four
// records alternate so the next group loads while the current one gathers.
template <int TPT, int R, typename Gather>
__device__ __forceinline__ void union_loop_packed(int pb, int pe, const float4* __restrict__ rec,
                                                  CV<float, TPT> (&acc)[R], Gather gather) {
    if (pb >= pe) return;
    float4 A[4], Bq[4];
    auto process = [&](const float4 (&E)[4]) {
        CV<float, TPT> y[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) y[q] = gather(__float_as_int(E[q].x));
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            cfma<float, TPT>(acc[0], E[q].y, y[q]);
            if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], E[q].z, y[q]);
            if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], E[q].w, y[q]);
        }
    };
#pragma unroll
    for (int q = 0; q < 4; ++q) A[q] = __ldg(rec + pb + q);
    for (int p0 = pb;; p0 += 8) {
        const bool hasB = p0 + 4 < pe;
        if (hasB) {
#pragma unroll
            for (int q = 0; q < 4; ++q) Bq[q] = __ldg(rec + p0 + 4 + q);
        }
        process(A);
        if (!hasB) break;
        const bool hasA = p0 + 8 < pe;
        if (hasA) {
#pragma unroll
            for (int q = 0; q < 4; ++q) A[q] = __ldg(rec + p0 + 8 + q);
        }
        process(Bq);
        if (!hasA) break;
    }
}

// Header of one row block with its first four packed records, fetched one
// block ahead so the dependent bptr -> record loads leave the critical path.
struct BlkPre {
    int pb, pe;
    float4 A[4];
};

__device__ __forceinline__ void blk_prefetch(BlkPre& P, bool valid, int k, const int* __restrict__ bptr,
                                             const float4* __restrict__ rec) {
    if (valid) {
        P.pb = __ldg(bptr + k);
        P.pe = __ldg(bptr + k + 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) P.A[q] = __ldg(rec + P.pb + q);
    } else {
        P.pb = P.pe = 0;
    }
}

// union_loop_packed with the first group already in registers (P.A)
template <int TPT, int R, typename Gather>
__device__ __forceinline__ void union_loop_pre(const BlkPre& P, const float4* __restrict__ rec,
                                               CV<float, TPT> (&acc)[R], Gather gather) {
    const int pb = P.pb, pe = P.pe;
    if (pb >= pe) return;
    float4 A[4], Bq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) A[q] = P.A[q];
    auto process = [&](const float4 (&E)[4]) {
        CV<float, TPT> y[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) y[q] = gather(__float_as_int(E[q].x));
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            cfma<float, TPT>(acc[0], E[q].y, y[q]);
            if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], E[q].z, y[q]);
            if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], E[q].w, y[q]);
        }
    };
    for (int p0 = pb;; p0 += 8) {
        const bool hasB = p0 + 4 < pe;
        if (hasB) {
#pragma unroll
            for (int q = 0; q < 4; ++q) Bq[q] = __ldg(rec + p0 + 4 + q);
        }
        process(A);
        if (!hasB) break;
        const bool hasA = p0 + 8 < pe;
        if (hasA) {
#pragma unroll
            for (int q = 0; q < 4; ++q) A[q] = __ldg(rec + p0 + 8 + q);
        }
        process(Bq);
        if (!hasA) break;
    }
}

template <typename Real, int TPT, int R, typename Gather>
__device__ __forceinline__ void union_any(int pb, int pe, const int* __restrict__ bcol,
                                          const Real* __restrict__ bcoef, CV<Real, TPT> (&acc)[R], Gather gather) {
    if constexpr (sizeof(Real) == 4 && R <= 3) {
        union_loop_packed<TPT, R>(pb, pe, reinterpret_cast<const float4*>(bcoef), acc, gather);
    } else {
        union_loop<Real, TPT, R, UnionGroup<R>::G>(pb, pe, bcol, bcoef, acc, gather);
    }
}

// Row-blocked SpMM: w = H q_j for all trajectories of the chunk, R rows per
// block.  kWrite: also alpha_j[b] = <q_j, w>_b; !kWrite: ||H q_j||_b only.
// With rjm (kWrite, j >= 2) the kernel writes w = H q_j - beta_{j-1} q_{j-1}
// instead and alpha_j = <q_j, w> (the ordering of Paige's stable variant):
// q_{j-1} is one streaming read per row next to the latency-bound gathers,
// and the axpy that follows reads two slabs instead of three.  The term is
// folded into the accumulator's start value, -(beta_{j-1} sc_{j-1} / sc_j)
// r_{j-1}, so it holds no registers across the gather loop.
template <typename Real, int TPT, int R, bool kBilinear, bool kWrite, int NT = kBThreads>
__global__ void __launch_bounds__(NT) k_spmm_blk(int n, int B, int TC, int bpc, int nb, int j,
                                                       const int* __restrict__ bptr, const int* __restrict__ bcol,
                                                       const Real* __restrict__ bcoef, const Real* __restrict__ d,
                                                       const Real* __restrict__ rj, const Real* __restrict__ rjm,
                                                       Real* __restrict__ w, BatchedScalars S, int cy0, int nch) {
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    const int chunk = blockIdx.y + cy0;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + tr * TPT;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    double sc[TPT], ar[TPT], ai[TPT];
    Real fm[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        sc[t] = S.sc[(size_t)j * B + b0 + t];
        ar[t] = 0.0;
        ai[t] = 0.0;
        fm[t] = 0;
        if (rjm) {
            // sc_j = 0 only after a breakdown, where beta_{j-1} = 0 as well
            const size_t km = (size_t)(j - 1) * B + b0 + t;
            fm[t] = sc[t] != 0.0 ? (Real)(S.beta[km] * S.sc[km] / sc[t]) : Real(0);
        }
    }
    constexpr bool kPk = sizeof(Real) == 4 && R <= 3;
    const float4* rec = reinterpret_cast<const float4*>(bcoef);
    BlkPre P;
    if constexpr (kPk) blk_prefetch(P, k0 + rl < k1, k0 + rl, bptr, rec);
    for (int k = k0 + rl; k < k1; k += RPC) {
        const int row0 = k * R;
        BlkPre cur;
        if constexpr (kPk) {
            cur = P;
            blk_prefetch(P, k + RPC < k1, k + RPC, bptr, rec);
        }
        // the block's own rows and diagonal are loaded first and used only
        // after the union loop, so their latency hides under the gathers
        CV<Real, TPT> acc[R], xo[R];
        Real dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = min(row0 + i, n - 1);
            const size_t base = (size_t)row * B + b0;
            xo[i] = ldv<Real, TPT, true>(rj, base);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                dd[i][t] = row0 + i < n ? __ldg(d + base + t) : Real(0);
                acc[i].v[2 * t] = 0;
                acc[i].v[2 * t + 1] = 0;
            }
            if (rjm) {
                const CV<Real, TPT> xm = ldv_cs<Real, TPT>(rjm, base);
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    acc[i].v[2 * t] = -fm[t] * xm.v[2 * t];
                    acc[i].v[2 * t + 1] = -fm[t] * xm.v[2 * t + 1];
                }
            }
        }
        auto gather = [&](int c) { return ldv<Real, TPT, true>(rj, (size_t)c * B + b0); };
        if constexpr (kPk) union_loop_pre<TPT, R>(cur, rec, acc, gather);
        else union_any<Real, TPT, R>(__ldg(bptr + k), __ldg(bptr + k + 1), bcol, bcoef, acc, gather);
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                acc[i].v[2 * t] = fma(dd[i][t], xo[i].v[2 * t], acc[i].v[2 * t]);
                acc[i].v[2 * t + 1] = fma(dd[i][t], xo[i].v[2 * t + 1], acc[i].v[2 * t + 1]);
            }
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            if (row >= n) break;
            const size_t base = (size_t)row * B + b0;
            if (kWrite) {
                const CV<Real, TPT>& x = xo[i];
                CV<Real, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    o.v[2 * t] = (Real)(sc[t] * (double)acc[i].v[2 * t]);
                    o.v[2 * t + 1] = (Real)(sc[t] * (double)acc[i].v[2 * t + 1]);
                    const double xr = x.v[2 * t], xi = x.v[2 * t + 1], ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                    if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                    else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                }
                stv<Real, TPT>(w, base, o);
            } else {
#pragma unroll
                for (int t = 0; t < TPT; ++t)
                    ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] + (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
            }
        }
    }
    __shared__ double2 red[kMaxTC];
    __shared__ double2 rscratch[NT * 2];
    if (chunk_reduce_s<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk, rscratch)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double s = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s * s;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s * s;
            } else {
                S.nav[b] = sqrt(v.x) * s;
            }
        }
    }
}

// K per-trajectory real sums of one block: summed over the block's row lanes
// in shared memory (one quantity at a time through `sm`, blockDim.x * TPT
// doubles), stored as partial[chunk][block][K][TC]; one ticket per chunk, and
// the last block adds the blocks' partials in a fixed order (deterministic).
// Returns true in that block, with the totals in red_out[q * TC + t].
template <int K, int TPT>
__device__ __forceinline__ bool chunk_reduce_multi(const double (&v)[K][TPT], int TC, double* partial,
                                                   unsigned int* ticket, double* red_out, int chunk, double* sm) {
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    double* mypart = partial + ((size_t)chunk * gridDim.x + blockIdx.x) * K * TC;
#pragma unroll
    for (int q = 0; q < K; ++q) {
#pragma unroll
        for (int t = 0; t < TPT; ++t) sm[rl * TC + tr * TPT + t] = v[q][t];
        __syncthreads();
        if (threadIdx.x < TC) {
            double s = 0.0;
            for (int r = 0; r < RPC; ++r) s += sm[r * TC + threadIdx.x];
            mypart[q * TC + threadIdx.x] = s;
        }
        __syncthreads();
    }
    const bool last = last_block_ticket(ticket + chunk, gridDim.x);
    if (last) {
        const int per = blockDim.x / TC;
        const int tl = threadIdx.x % TC, part = threadIdx.x / TC;
        const double* base = partial + (size_t)chunk * gridDim.x * K * TC;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            double s = 0.0;
            for (unsigned int g = part; g < gridDim.x; g += per) s += __ldcg(base + ((size_t)g * K + q) * TC + tl);
            sm[part * TC + tl] = s;
            __syncthreads();
            if (threadIdx.x < TC) {
                double a = 0.0;
                for (int p = 0; p < per; ++p) a += sm[p * TC + threadIdx.x];
                red_out[q * TC + threadIdx.x] = a;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) ticket[chunk] = 0;
        __syncthreads();
    }
    return last;
}

// One Lanczos iteration in one launch without the axpy pass (staged = 8).
// Instead of the residual, iteration j - 1 leaves p_j = H q_{j-1} -
// beta_{j-2} q_{j-2} in HBM together with alpha_{j-1} = <q_{j-1}, p_j> and
// beta_{j-1} = ||p_j - alpha_{j-1} q_{j-1}||, the latter from three sums of
// the same pass (||p_j||^2 - 2 Re(conj(alpha) <q, p_j>) + |alpha|^2 ||q||^2,
// all FP64 over the stored values).  Iteration j gathers only p_j:
//   q_j     = (p_j - alpha_{j-1} q_{j-1}) / beta_{j-1}                 (stored, unit norm)
//   H q_j   = (H p_j - alpha_{j-1} (p_j + beta_{j-2} q_{j-2})) / beta_{j-1}
//             (H q_{j-1} = p_j + beta_{j-2} q_{j-2} by the recurrence)
//   p_{j+1} = H q_j - beta_{j-1} q_{j-1}                                 (stored)
// and sums <q_j, p_{j+1}> (the alpha form), the Hermitian <q_j, p_{j+1}>,
// ||p_{j+1}||^2 and ||q_j||^2 for alpha_j and beta_j: the ordering of
// Paige's variant (lanczosClass.cu:405-526 in exact arithmetic).  Per
// site-trajectory it moves p_j, q_{j-1}, q_{j-2}, the diagonal, q_j and
// p_{j+1} (44 B in complex64) where the SpMM + axpy pair moves 52 B, in one
// launch instead of two.  kMode 0 (j = 1): gathers psi = r_1 (q_1 = sc_1 r_1)
// and writes p_2 only; kMode 2 (j = m + 1): writes q_{m+1} and gives
// ||H q_{m+1}|| (nav) instead of p_{m+2}.  The slabs q_j, j >= 2, are stored
// normalised (sc_j = 1).  Gathers go through L1 over row blocks of R rows as
// in k_spmm_blk; the per-row arithmetic after the gather runs in FP64.
template <typename Real, int TPT, int R, bool kBilinear, int kMode, int NT>
__global__ void __launch_bounds__(NT) k_lanczos_p(int n, int B, int TC, int bpc, int nb, int j,
                                                  const int* __restrict__ bptr, const int* __restrict__ bcol,
                                                  const Real* __restrict__ bcoef, const Real* __restrict__ d,
                                                  const Real* __restrict__ pin, const Real* __restrict__ qm1,
                                                  const Real* __restrict__ qm2, Real* __restrict__ qout,
                                                  Real* __restrict__ pout, BatchedScalars S, int nch) {
    constexpr bool kFirst = kMode == 0, kLast = kMode == 2;
    constexpr int K = kLast ? 1 : (kBilinear ? 6 : 4);
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    const int chunk = blockIdx.y;
    const int b0 = chunk * TC + tr * TPT;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    // per-trajectory coefficients of this iteration, in shared memory (read
    // once per row after the gathers, so they hold no registers across them):
    // [0] alpha_r, [1] alpha_i, [2] 1/beta_{j-1}, [3] beta_{j-1}, [4] sc_{j-1}
    // (sc_1 for j = 1), [5], [6] alpha_{j-1} beta_{j-2} sc_{j-2} (the q_{j-2}
    // term of H q_j)
    __shared__ double cf[7][kMaxTC];
    for (int t = threadIdx.x; t < TC; t += blockDim.x) {
        const int b = chunk * TC + t;
        double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if constexpr (kFirst) {
            v[4] = S.sc[(size_t)B + b];
        } else {
            const size_t km = (size_t)(j - 1) * B + b;
            v[0] = S.alpha[2 * km];
            v[1] = S.alpha[2 * km + 1];
            v[3] = S.beta[km];
            v[2] = v[3] > 0.0 ? 1.0 / v[3] : 0.0;
            v[4] = S.sc[km];
            if (j >= 3) {
                const size_t k2 = (size_t)(j - 2) * B + b;
                v[5] = v[0] * S.beta[k2] * S.sc[k2];
                v[6] = v[1] * S.beta[k2] * S.sc[k2];
            }
        }
#pragma unroll
        for (int q = 0; q < 7; ++q) cf[q][t] = v[q];
    }
    __syncthreads();
    double sum[K][TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t)
#pragma unroll
        for (int q = 0; q < K; ++q) sum[q][t] = 0.0;
    constexpr bool kPk = sizeof(Real) == 4 && R <= 3;
    const float4* rec = reinterpret_cast<const float4*>(bcoef);
    BlkPre P;
    if constexpr (kPk) blk_prefetch(P, k0 + rl < k1, k0 + rl, bptr, rec);
    for (int k = k0 + rl; k < k1; k += RPC) {
        const int row0 = k * R;
        BlkPre cur;
        if constexpr (kPk) {
            cur = P;
            blk_prefetch(P, k + RPC < k1, k + RPC, bptr, rec);
        }
        // the diagonal is loaded before the gathers; the rows of q_{j-1} and
        // q_{j-2} are only prefetched into L1 then (no registers held across
        // the gather loop) and read after it together with the block's own
        // rows of the gathered vector, which its neighbours' gathers have
        // just brought into L1
        CV<Real, TPT> acc[R];
        Real dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = min(row0 + i, n - 1);
            const size_t base = (size_t)row * B + b0;
            if constexpr (!kFirst) {
                asm volatile("prefetch.global.L1 [%0];" ::"l"(qm1 + 2 * base));
                if (qm2) asm volatile("prefetch.global.L1 [%0];" ::"l"(qm2 + 2 * base));
            }
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                dd[i][t] = row0 + i < n ? __ldg(d + base + t) : Real(0);
                acc[i].v[2 * t] = 0;
                acc[i].v[2 * t + 1] = 0;
            }
        }
        auto gather = [&](int c) { return ldv<Real, TPT, true>(pin, (size_t)c * B + b0); };
        if constexpr (kPk) union_loop_pre<TPT, R>(cur, rec, acc, gather);
        else union_any<Real, TPT, R>(__ldg(bptr + k), __ldg(bptr + k + 1), bcol, bcoef, acc, gather);
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            if (row >= n) break;
            const size_t base = (size_t)row * B + b0;
            const CV<Real, TPT> po = ldv<Real, TPT, true>(pin, base);
            CV<Real, TPT> x1, x2;
#pragma unroll
            for (int v = 0; v < 2 * TPT; ++v) x1.v[v] = x2.v[v] = 0;
            if constexpr (!kFirst) {
                x1 = ldv<Real, TPT, true>(qm1, base);
                if (qm2) x2 = ldv_cs<Real, TPT>(qm2, base);
            }
            CV<Real, TPT> oq, op;
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                const int tt = tr * TPT + t;
                const double a_r = cf[0][tt], a_i = cf[1][tt], ib = cf[2][tt], b1 = cf[3][tt], s1 = cf[4][tt];
                const double c2r = cf[5][tt], c2i = cf[6][tt];
                const double pr = po.v[2 * t], pi = po.v[2 * t + 1];
                // H p at this row: gathered off-diagonal part plus the diagonal
                const double hr = (double)fma(dd[i][t], po.v[2 * t], acc[i].v[2 * t]);
                const double hi = (double)fma(dd[i][t], po.v[2 * t + 1], acc[i].v[2 * t + 1]);
                double qr, qi, ur, ui;   // q_j and the vector whose products are summed
                if constexpr (kFirst) {
                    qr = s1 * pr;
                    qi = s1 * pi;
                    ur = s1 * hr;     // p_2 = H q_1
                    ui = s1 * hi;
                } else {
                    const double y1r = s1 * x1.v[2 * t], y1i = s1 * x1.v[2 * t + 1];
                    const double y2r = x2.v[2 * t], y2i = x2.v[2 * t + 1];
                    qr = (pr - (a_r * y1r - a_i * y1i)) * ib;
                    qi = (pi - (a_r * y1i + a_i * y1r)) * ib;
                    // H q_j = (H p - alpha p - alpha beta_{j-2} sc_{j-2} r_{j-2}) / beta_{j-1}
                    const double gr = (hr - (a_r * pr - a_i * pi) - (c2r * y2r - c2i * y2i)) * ib;
                    const double gi = (hi - (a_r * pi + a_i * pr) - (c2r * y2i + c2i * y2r)) * ib;
                    if constexpr (kLast) {
                        ur = gr;
                        ui = gi;
                    } else {
                        ur = gr - b1 * y1r;   // p_{j+1} = H q_j - beta_{j-1} q_{j-1}
                        ui = gi - b1 * y1i;
                    }
                }
                oq.v[2 * t] = (Real)qr;
                oq.v[2 * t + 1] = (Real)qi;
                op.v[2 * t] = (Real)ur;
                op.v[2 * t + 1] = (Real)ui;
                // the sums use the stored (rounded) values that the next iteration reads
                const double sqr = kFirst ? qr : (double)oq.v[2 * t], sqi = kFirst ? qi : (double)oq.v[2 * t + 1];
                const double spr = kLast ? ur : (double)op.v[2 * t], spi = kLast ? ui : (double)op.v[2 * t + 1];
                if constexpr (kLast) {
                    sum[0][t] += spr * spr + spi * spi;
                } else {
                    if (kBilinear) {
                        sum[0][t] += sqr * spr - sqi * spi;
                        sum[1][t] += sqr * spi + sqi * spr;
                    } else {
                        sum[0][t] += sqr * spr + sqi * spi;
                        sum[1][t] += sqr * spi - sqi * spr;
                    }
                    if constexpr (kBilinear) {
                        sum[K - 2][t] += sqr * spr + sqi * spi;
                        sum[K - 1][t] += sqr * spi - sqi * spr;
                    }
                    sum[2][t] += spr * spr + spi * spi;
                    sum[3][t] += sqr * sqr + sqi * sqi;
                }
            }
            if constexpr (!kFirst) stv<Real, TPT>(qout, base, oq);
            if constexpr (!kLast) stv<Real, TPT>(pout, base, op);
        }
    }
    __shared__ double red[K * kMaxTC];
    __shared__ double rsm[NT * TPT > kMaxTC * 8 ? NT * TPT : kMaxTC * 8];
    if (chunk_reduce_multi<K, TPT>(sum, TC, S.partial, S.tickets + (kLast ? 2 : 0) * nch, red, chunk, rsm)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            if constexpr (kLast) {
                S.nav[b] = sqrt(red[threadIdx.x]);
            } else {
                const double ar = red[threadIdx.x], ai = red[TC + threadIdx.x];
                const double hr = kBilinear ? red[(K - 2) * TC + threadIdx.x] : ar;
                const double hi = kBilinear ? red[(K - 1) * TC + threadIdx.x] : ai;
                const double np = red[2 * TC + threadIdx.x], nq = red[3 * TC + threadIdx.x];
                const double b2 = np - 2.0 * (ar * hr + ai * hi) + (ar * ar + ai * ai) * nq;
                double bt = sqrt(fmax(b2, 0.0));
                if (!isfinite(b2)) atomicCAS(S.status, 0, DQ_ERR_NAN);
                // lucky breakdown: invariant Krylov space, continue with q_{j+1} = 0
                const size_t kj = (size_t)j * B + b;
                const double scale = sqrt(ar * ar + ai * ai) + (j > 1 ? S.beta[(size_t)(j - 1) * B + b] : 0.0);
                if (bt <= kBreakdownRel * scale) bt = 0.0;
                S.alpha[2 * kj] = ar;
                S.alpha[2 * kj + 1] = ai;
                S.beta[kj] = bt;
                S.sc[(size_t)(j + 1) * B + b] = bt > 0.0 ? 1.0 : 0.0;
            }
        }
    }
}

// Row-blocked SpMM whose gathers are asynchronous copies into shared memory
// (staged = 9; complex64, packed records, R <= 3, TC = 64, 2 trajectories per
// lane, 512-thread CTAs).  In k_spmm_blk every gathered row waits in the
// registers of the warp that asked for it, so the registers bound the gathers
// in flight (four per warp).  Here lane l of the warp that owns a row block
// issues cp.async.ca (16 bytes, through L1) of its two trajectories of each
// gathered row into its own slot of a per-warp ring of kCpaStages groups of
// four records, commits one group at a time and keeps kCpaStages - 1 groups in
// flight (12 rows per warp); it reads each group back from its own slots
// after cp.async.wait_group, so no lane waits for another and no barrier is
// involved.  The block's records are staged once per block in a per-warp
// shared buffer (at most kCpaMaxRec; dq_set_tiling refuses larger blocks) and
// read by broadcast.  Everything after the gathers (the minus beta q_{j-1}
// start value, the diagonal, alpha or the norm) is k_spmm_blk's.
constexpr int kCpaStages = 4;
constexpr int kCpaMaxRec = 128;
constexpr int kCpaWarps = 16;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

inline size_t cpa_smem_bytes() {
    return (size_t)kCpaWarps * ((size_t)kCpaStages * 4 * 32 * sizeof(float4) + (size_t)kCpaMaxRec * sizeof(float4));
}

template <int R, bool kBilinear, bool kWrite>
__global__ void __launch_bounds__(512, 1) k_spmm_cpa(int n, int B, int bpc, int nb, int j,
                                                    const int* __restrict__ bptr, const float4* __restrict__ rec,
                                                    const float* __restrict__ d, const float* __restrict__ rj,
                                                    const float* __restrict__ rjm, float* __restrict__ w,
                                                    BatchedScalars S, int nch) {
    constexpr int TPT = 2, TC = 64;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float4* ring = reinterpret_cast<float4*>(smem_raw) + (size_t)warp * kCpaStages * 4 * 32;
    float4* recs = reinterpret_cast<float4*>(smem_raw) + (size_t)kCpaWarps * kCpaStages * 4 * 32 +
                   (size_t)warp * kCpaMaxRec;
    const int chunk = blockIdx.y;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + lane * TPT;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    double sc[TPT], ar[TPT], ai[TPT];
    float fm[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        sc[t] = S.sc[(size_t)j * B + b0 + t];
        ar[t] = 0.0;
        ai[t] = 0.0;
        fm[t] = 0.f;
        if (rjm) {
            const size_t km = (size_t)(j - 1) * B + b0 + t;
            fm[t] = sc[t] != 0.0 ? (float)(S.beta[km] * S.sc[km] / sc[t]) : 0.f;
        }
    }
    const float* lane_src = rj + 2 * (size_t)b0;   // this lane's two trajectories of row 0
    for (int k = k0 + warp; k < k1; k += kCpaWarps) {
        const int row0 = k * R;
        const int pb = __ldg(bptr + k), pe = __ldg(bptr + k + 1);
        const int nrec = pe - pb;   // a multiple of 4, at most kCpaMaxRec
        __syncwarp();   // every lane is done with the previous block's records
        for (int e = lane; e < nrec; e += 32) recs[e] = __ldg(rec + pb + e);
        // the block's own rows, diagonal and q_{j-1}, used after the gathers
        CV<float, TPT> acc[R], xo[R];
        float dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = min(row0 + i, n - 1);
            const size_t base = (size_t)row * B + b0;
            xo[i] = ldv<float, TPT, true>(rj, base);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                dd[i][t] = row0 + i < n ? __ldg(d + base + t) : 0.f;
                acc[i].v[2 * t] = 0.f;
                acc[i].v[2 * t + 1] = 0.f;
            }
            if (rjm) {
                const CV<float, TPT> xm = ldv_cs<float, TPT>(rjm, base);
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    acc[i].v[2 * t] = -fm[t] * xm.v[2 * t];
                    acc[i].v[2 * t + 1] = -fm[t] * xm.v[2 * t + 1];
                }
            }
        }
        __syncwarp();   // the records are in the buffer
        const int ng = nrec >> 2;
        auto issue = [&](int g) {
            float4* slot = ring + (size_t)(g % kCpaStages) * 4 * 32 + lane;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int c = __float_as_int(recs[4 * g + q].x);
                cp_async16(slot + q * 32, lane_src + 2 * (size_t)c * B);
            }
        };
#pragma unroll
        for (int g = 0; g < kCpaStages - 1; ++g) {
            if (g < ng) issue(g);
            cp_async_commit();
        }
        for (int g = 0; g < ng; ++g) {
            if (g + kCpaStages - 1 < ng) issue(g + kCpaStages - 1);
            cp_async_commit();
            cp_async_wait<kCpaStages - 1>();   // group g has landed in this lane's slots
            const float4* slot = ring + (size_t)(g % kCpaStages) * 4 * 32 + lane;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 yv = slot[q * 32];
                CV<float, TPT> y;
                y.v[0] = yv.x; y.v[1] = yv.y; y.v[2] = yv.z; y.v[3] = yv.w;
                const float4 r = recs[4 * g + q];
                cfma<float, TPT>(acc[0], r.y, y);
                if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], r.z, y);
                if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], r.w, y);
            }
        }
        cp_async_wait<0>();
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                acc[i].v[2 * t] = fmaf(dd[i][t], xo[i].v[2 * t], acc[i].v[2 * t]);
                acc[i].v[2 * t + 1] = fmaf(dd[i][t], xo[i].v[2 * t + 1], acc[i].v[2 * t + 1]);
            }
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            if (row >= n) break;
            const size_t base = (size_t)row * B + b0;
            if (kWrite) {
                const CV<float, TPT>& x = xo[i];
                CV<float, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    o.v[2 * t] = (float)(sc[t] * (double)acc[i].v[2 * t]);
                    o.v[2 * t + 1] = (float)(sc[t] * (double)acc[i].v[2 * t + 1]);
                    const double xr = x.v[2 * t], xi = x.v[2 * t + 1], ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                    if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                    else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                }
                stv<float, TPT>(w, base, o);
            } else {
#pragma unroll
                for (int t = 0; t < TPT; ++t)
                    ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] + (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
            }
        }
    }
    __syncthreads();   // the ring becomes the reduction scratch
    __shared__ double2 red[kMaxTC];
    double2* rscratch = reinterpret_cast<double2*>(smem_raw);
    if (chunk_reduce_s<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk, rscratch)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double s = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s * s;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s * s;
            } else {
                S.nav[b] = sqrt(v.x) * s;
            }
        }
    }
}

// Row-blocked SpMM with eight gathers in flight per warp (staged = 10;
// complex64, packed records, R <= 3, TC = 64, 2 trajectories per lane, one
// 512-thread CTA per SM).  Each warp owns whole row blocks (k0 + warp,
// k0 + warp + 16, ...), so the 16 warps of a CTA walk one sliding window of
// rows together and every record of a block is warp-uniform.  The records
// arrive 32 at a time (one coalesced 16-byte load per lane, the next batch or
// the next block's first one in flight while the current one is used) into a
// per-warp shared buffer; a group of eight gathers is issued from the eight
// columns read there by broadcast, and the coefficients are read again only
// after the gathers, so the registers a warp holds across its gather wait are
// the eight gathered values and its accumulators.  That doubles the gathers
// in flight per warp of k_spmm_blk (four) at the same occupancy.  Everything
// after the gathers (the minus beta q_{j-1} start value, the diagonal, alpha
// or the norm) is k_spmm_blk's.
constexpr int kWgWarps = 16;

template <int R, bool kBilinear, bool kWrite, bool kAxpy = false>
__global__ void __launch_bounds__(512, 1) k_spmm_wg(int n, int B, int bpc, int nb, int j,
                                                   const int* __restrict__ bptr, const float4* __restrict__ rec,
                                                   const float* __restrict__ d, const float* __restrict__ rj,
                                                   const float* __restrict__ rjm, float* __restrict__ w,
                                                   BatchedScalars S, int cy0, int nch, float* __restrict__ rjp = nullptr) {
    constexpr int TPT = 2, TC = 64, G = 8;
    __shared__ float4 rbuf[kWgWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int chunk = blockIdx.y + cy0;
    // kAxpy: the chunk's alpha generation before this block can arrive at the
    // alpha ticket, so the increment by the ticket's last block is always seen
    unsigned int* const gen = S.tickets + 7 * (size_t)nch + chunk;
    unsigned int gen0 = 0;
    if (kAxpy && threadIdx.x == 0) gen0 = ld_acquire_u32(gen);
    if (!kAxpy && chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + lane * TPT;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    double sc[TPT], ar[TPT], ai[TPT];
    float fm[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        sc[t] = S.sc[(size_t)j * B + b0 + t];
        ar[t] = 0.0;
        ai[t] = 0.0;
        fm[t] = 0.f;
        if (rjm) {
            const size_t km = (size_t)(j - 1) * B + b0 + t;
            fm[t] = sc[t] != 0.0 ? (float)(S.beta[km] * S.sc[km] / sc[t]) : 0.f;
        }
    }
    const float* lane_src = rj + 2 * (size_t)b0;   // this lane's two trajectories of row 0
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4* const buf = rbuf[warp];
    int k = k0 + warp;
    int pb = 0, pe = 0;
    if (k < k1) {
        pb = __ldg(bptr + k);
        pe = __ldg(bptr + k + 1);
    }
    float4 nxt = (k < k1 && lane < pe - pb) ? __ldg(rec + pb + lane) : zero4;
    while (k < k1) {
        const int kn = k + kWgWarps;
        int pbn = 0, pen = 0;
        if (kn < k1) {
            pbn = __ldg(bptr + kn);
            pen = __ldg(bptr + kn + 1);
        }
        const int row0 = k * R;
        // the block's own rows and diagonal are loaded first and used only
        // after the gathers, so their latency hides under them
        CV<float, TPT> acc[R], xo[R];
        float dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const size_t base = (size_t)min(row0 + i, n - 1) * B + b0;
            xo[i] = ldv<float, TPT, true>(rj, base);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                dd[i][t] = row0 + i < n ? __ldg(d + base + t) : 0.f;
                acc[i].v[2 * t] = 0.f;
                acc[i].v[2 * t + 1] = 0.f;
            }
            if (rjm) {
                const CV<float, TPT> xm = ldv_cs<float, TPT>(rjm, base);
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    acc[i].v[2 * t] = -fm[t] * xm.v[2 * t];
                    acc[i].v[2 * t + 1] = -fm[t] * xm.v[2 * t + 1];
                }
            }
        }
        for (int e0 = pb; e0 < pe; e0 += 32) {
            __syncwarp();   // every lane is done with the previous batch
            buf[lane] = nxt;
            __syncwarp();
            if (e0 + 32 < pe) nxt = (e0 + 32 + lane < pe) ? __ldg(rec + e0 + 32 + lane) : zero4;
            else nxt = (kn < k1 && lane < pen - pbn) ? __ldg(rec + pbn + lane) : zero4;
            const int cnt = min(32, pe - e0);   // a multiple of 4
            for (int e = 0; e < cnt; e += G) {
                const bool two = e + 4 < cnt;   // warp-uniform: the group's second half exists
                CV<float, TPT> y[G];
#pragma unroll
                for (int q = 0; q < G; ++q) {
                    if (q < 4 || two) {
                        const int c = __float_as_int(buf[e + q].x);
                        const float4 v = __ldg(reinterpret_cast<const float4*>(lane_src + 2 * (size_t)c * B));
                        y[q].v[0] = v.x; y[q].v[1] = v.y; y[q].v[2] = v.z; y[q].v[3] = v.w;
                    }
                }
#pragma unroll
                for (int q = 0; q < G; ++q) {
                    if (q < 4 || two) {
                        const float4 r = buf[e + q];
                        cfma<float, TPT>(acc[0], r.y, y[q]);
                        if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], r.z, y[q]);
                        if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], r.w, y[q]);
                    }
                }
            }
        }
        if (pe <= pb) nxt = (kn < k1 && lane < pen - pbn) ? __ldg(rec + pbn + lane) : zero4;
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                acc[i].v[2 * t] = fmaf(dd[i][t], xo[i].v[2 * t], acc[i].v[2 * t]);
                acc[i].v[2 * t + 1] = fmaf(dd[i][t], xo[i].v[2 * t + 1], acc[i].v[2 * t + 1]);
            }
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            if (row >= n) break;
            const size_t base = (size_t)row * B + b0;
            if (kWrite) {
                const CV<float, TPT>& x = xo[i];
                CV<float, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    o.v[2 * t] = (float)(sc[t] * (double)acc[i].v[2 * t]);
                    o.v[2 * t + 1] = (float)(sc[t] * (double)acc[i].v[2 * t + 1]);
                    const double xr = x.v[2 * t], xi = x.v[2 * t + 1], ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                    if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                    else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                }
                stv<float, TPT>(w, base, o);
            } else {
#pragma unroll
                for (int t = 0; t < TPT; ++t)
                    ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] + (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
            }
        }
        k = kn;
        pb = pbn;
        pe = pen;
    }
    __shared__ double2 red[kMaxTC];
    __shared__ double2 rscratch[512 * 2];
    const bool last = chunk_reduce_s<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk,
                                          rscratch);
    if (last) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double s = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s * s;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s * s;
            } else {
                S.nav[b] = sqrt(v.x) * s;
            }
        }
    }
    if constexpr (kAxpy) {
        // The residual r_{j+1} = w - alpha_j q_j of this block's rows, in the
        // same launch: every block of the chunk waits (bounded) for the alpha
        // ticket's last block to publish alpha_j, then reads w, which it has
        // just written, and q_j while both are still in L2.  The launch is
        // cooperative, so all blocks are resident and the wait ends.
        __shared__ int s_ok;
        __syncthreads();   // the last block's alpha stores are done
        if (threadIdx.x == 0) {
            int ok = 1;
            if (last) {
                __threadfence();
                atomicAdd(gen, 1u);
            } else {
                // a negative budget is the forced-timeout test mode: wait
                // |budget| cycles for a generation that never comes
                const long long budget = g_dq_wait_cycles;
                const long long lim = budget < 0 ? -budget : budget;
                const long long t0 = clock64();
                ok = 0;
                while (clock64() - t0 < lim) {
                    if (budget > 0 && ld_acquire_u32(gen) != gen0) {
                        ok = 1;
                        break;
                    }
                    __nanosleep(64);
                }
                if (!ok) atomicCAS(S.status, 0, DQ_ERR_TIMEOUT);
            }
            s_ok = ok;
        }
        __syncthreads();
        const bool ok = s_ok != 0;
        double ajr[TPT], aji[TPT], nn[TPT], zero[TPT];
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            const size_t kk = (size_t)j * B + b0 + t;
            ajr[t] = __ldcg(&S.alpha[2 * kk]) * S.sc[kk];
            aji[t] = __ldcg(&S.alpha[2 * kk + 1]) * S.sc[kk];
            nn[t] = 0.0;
            zero[t] = 0.0;
        }
        // after a timeout the block adds nothing but still takes its ticket,
        // so the reduction stays consistent (the status reports the failure)
        // four rows per warp per trip: eight independent loads in flight per lane
        constexpr int kAx = 4;
        const int rend = ok ? min(n, k1 * R) : 0;
        for (int row = k0 * R + warp; row < rend; row += kAx * kWgWarps) {
            float4 u[kAx], x[kAx];
#pragma unroll
            for (int h = 0; h < kAx; ++h) {
                const int rr = row + h * kWgWarps;
                const size_t base = (size_t)(rr < rend ? rr : row) * B + b0;
                u[h] = __ldcg(reinterpret_cast<const float4*>(w + 2 * base));
                x[h] = __ldg(reinterpret_cast<const float4*>(rj + 2 * base));
            }
#pragma unroll
            for (int h = 0; h < kAx; ++h) {
                const int rr = row + h * kWgWarps;
                if (rr >= rend) break;
                const float uv[4] = {u[h].x, u[h].y, u[h].z, u[h].w}, xv[4] = {x[h].x, x[h].y, x[h].z, x[h].w};
                float ov[4];
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    const double xr = xv[2 * t], xi = xv[2 * t + 1];
                    ov[2 * t] = (float)((double)uv[2 * t] - (ajr[t] * xr - aji[t] * xi));
                    ov[2 * t + 1] = (float)((double)uv[2 * t + 1] - (ajr[t] * xi + aji[t] * xr));
                    nn[t] += (double)ov[2 * t] * ov[2 * t] + (double)ov[2 * t + 1] * ov[2 * t + 1];
                }
                *reinterpret_cast<float4*>(rjp + 2 * ((size_t)rr * B + b0)) = make_float4(ov[0], ov[1], ov[2], ov[3]);
            }
        }
        if (chunk_reduce_s<TPT>(nn, zero, TC, S.partial, S.tickets + 1 * nch, red, chunk, rscratch)) {
            if (threadIdx.x < TC) {
                const int b = chunk * TC + threadIdx.x;
                double bt = sqrt(red[threadIdx.x].x);
                if (!isfinite(bt)) atomicCAS(S.status, 0, DQ_ERR_NAN);
                // lucky breakdown as in k_axpy_beta
                const size_t kj = (size_t)j * B + b;
                const double a0 = __ldcg(&S.alpha[2 * kj]), a1 = __ldcg(&S.alpha[2 * kj + 1]);
                const double scale = sqrt(a0 * a0 + a1 * a1) + (j > 1 ? S.beta[(size_t)(j - 1) * B + b] : 0.0);
                if (bt <= kBreakdownRel * scale) bt = 0.0;
                S.beta[kj] = bt;
                S.sc[(size_t)(j + 1) * B + b] = bt > 0.0 ? 1.0 / bt : 0.0;
            }
        }
    }
}

// Lean row-blocked SpMM (staged = 12; complex64, packed records, R <= 3, 2
// trajectories per lane) for 32 warps per SM: NT = 1024 threads in one CTA
// per SM or NT = 512 in two, at most 64 registers a thread.  k_spmm_blk holds
// about 124 registers (the block's own rows and diagonal, two record groups,
// the next block's header, alpha sums and scalars across the gather loop), so
// only 16 warps fit per SM and each warp's FMA and store work between its
// gather waits is exposed.  Here a thread holds only the accumulators, the
// group of four records and their four gathered rows: the records are loaded
// where they are used (consecutive records share L1 lines), the own rows,
// diagonal and q_{j-1} rows are prefetched into L1 at the block's start and
// read after the gathers (minus beta q_{j-1} is added after the couplings),
// the chunk's scalars are staged once in shared memory and read per block,
// and the FP64 alpha sums of each thread live in shared memory.
template <int R, bool kBilinear, bool kWrite, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_spmm_lean(int n, int B, int TC, int bpc, int nb, int j,
                                                            const int* __restrict__ bptr,
                                                            const float4* __restrict__ rec,
                                                            const float* __restrict__ d, const float* __restrict__ rj,
                                                            const float* __restrict__ rjm, float* __restrict__ w,
                                                            BatchedScalars S, int cy0, int nch) {
    constexpr int TPT = 2;
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = NT / TPR;
    const int chunk = blockIdx.y + cy0;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + tr * TPT;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    // per-thread FP64 alpha (or norm) sums, then the reduction's scratch
    __shared__ double2 sums[NT * TPT];
    __shared__ double2 red[kMaxTC];
    // the chunk's sc_j and beta_{j-1} sc_{j-1} / sc_j, read per block from here
    __shared__ double sc_s[kMaxTC];
    __shared__ float fm_s[kMaxTC];
#pragma unroll
    for (int t = 0; t < TPT; ++t) sums[threadIdx.x * TPT + t] = make_double2(0.0, 0.0);
    if (threadIdx.x < TC) {
        const int b = chunk * TC + threadIdx.x;
        const double scb = S.sc[(size_t)j * B + b];
        float f = 0.f;
        if (rjm) {
            // sc_j = 0 only after a breakdown, where beta_{j-1} = 0 as well
            const size_t km = (size_t)(j - 1) * B + b;
            f = scb != 0.0 ? (float)(S.beta[km] * S.sc[km] / scb) : 0.f;
        }
        sc_s[threadIdx.x] = scb;
        fm_s[threadIdx.x] = f;
    }
    __syncthreads();
    const int tl = tr * TPT;   // this thread's first trajectory within the chunk
    const float* src = rj + 2 * (size_t)b0;
    for (int k = k0 + rl; k < k1; k += RPC) {
        const int row0 = k * R;
        const int pb = __ldg(bptr + k), pe = __ldg(bptr + k + 1);
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const size_t base = (size_t)min(row0 + i, n - 1) * B + b0;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(rj + 2 * base));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(d + base));
            if (rjm) asm volatile("prefetch.global.L1 [%0];" ::"l"(rjm + 2 * base));
        }
        CV<float, TPT> acc[R];
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int v = 0; v < 2 * TPT; ++v) acc[i].v[v] = 0.f;
        for (int e = pb; e < pe; e += 4) {   // a multiple of 4 records per block
            float4 r[4];
            CV<float, TPT> y[4];
            // the record line two groups ahead, within the block (the gathers'
            // addresses depend on the records)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(rec + min(e + 8, pe - 1)));
#pragma unroll
            for (int u = 0; u < 4; ++u) r[u] = __ldg(rec + e + u);
#pragma unroll
            for (int u = 0; u < 4; ++u) y[u] = ldv<float, TPT, true>(src, (size_t)__float_as_int(r[u].x) * B);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                cfma<float, TPT>(acc[0], r[u].y, y[u]);
                if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], r[u].z, y[u]);
                if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], r[u].w, y[u]);
            }
        }
        // minus beta_{j-1} q_{j-1} and the diagonal, then w and the sums
        double sc[TPT];
        float fm[TPT];
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            sc[t] = sc_s[tl + t];
            fm[t] = fm_s[tl + t];
        }
        double ar[TPT], ai[TPT];
#pragma unroll
        for (int t = 0; t < TPT; ++t) { ar[t] = 0.0; ai[t] = 0.0; }
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            if (row >= n) break;
            const size_t base = (size_t)row * B + b0;
            const CV<float, TPT> x = ldv<float, TPT, true>(rj, base);
            if (rjm) {
                const CV<float, TPT> xm = ldv<float, TPT, true>(rjm, base);
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    acc[i].v[2 * t] = fmaf(-fm[t], xm.v[2 * t], acc[i].v[2 * t]);
                    acc[i].v[2 * t + 1] = fmaf(-fm[t], xm.v[2 * t + 1], acc[i].v[2 * t + 1]);
                }
            }
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                const float dv = __ldg(d + base + t);
                acc[i].v[2 * t] = fmaf(dv, x.v[2 * t], acc[i].v[2 * t]);
                acc[i].v[2 * t + 1] = fmaf(dv, x.v[2 * t + 1], acc[i].v[2 * t + 1]);
            }
            if (kWrite) {
                CV<float, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    o.v[2 * t] = (float)(sc[t] * (double)acc[i].v[2 * t]);
                    o.v[2 * t + 1] = (float)(sc[t] * (double)acc[i].v[2 * t + 1]);
                    const double xr = x.v[2 * t], xi = x.v[2 * t + 1], ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                    if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                    else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                }
                stv<float, TPT>(w, base, o);
            } else {
#pragma unroll
                for (int t = 0; t < TPT; ++t)
                    ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] + (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
            }
        }
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            double2& sm = sums[threadIdx.x * TPT + t];
            sm.x += ar[t];
            sm.y += ai[t];
        }
    }
    double ar[TPT], ai[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        ar[t] = sums[threadIdx.x * TPT + t].x;
        ai[t] = sums[threadIdx.x * TPT + t].y;
    }
    __syncthreads();   // the sums become the reduction's scratch
    if (chunk_reduce_s<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk, sums)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double s = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s * s;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s * s;
            } else {
                S.nav[b] = sqrt(v.x) * s;
            }
        }
    }
}

// Warp-per-block SpMM (staged = 3; complex64, packed records, R <= 3).  All
// 32 lanes of a warp work on one block of R rows for TC = 32 TPT
// trajectories, so the block's column-union records are one warp-uniform
// stream: the warp fetches 32 records at a time with one coalesced 16-byte
// load per lane (the next batch, or the next block's first one, in flight
// while the current batch is used) and keeps them in a per-warp shared
// buffer that every lane reads back by broadcast.  The next block's header
// is fetched one block ahead, its own rows and diagonal at its start, so no
// index load sits on the gathers' dependency chain.
template <int TPT, int R, bool kBilinear, bool kWrite>
__global__ void __launch_bounds__(kBThreads) k_spmm_warp(int n, int B, int bpc, int nb, int j,
                                                        const int* __restrict__ bptr,
                                                        const float4* __restrict__ rec,
                                                        const float* __restrict__ d, const float* __restrict__ rj,
                                                        float* __restrict__ w, BatchedScalars S, int cy0, int nch) {
    constexpr int TC = 32 * TPT;
    constexpr int kWarps = kBThreads / 32;
    __shared__ float4 rbuf[kWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int chunk = blockIdx.y + cy0;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + lane * TPT;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    double sc[TPT], ar[TPT], ai[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        sc[t] = S.sc[(size_t)j * B + b0 + t];
        ar[t] = 0.0;
        ai[t] = 0.0;
    }
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    int k = k0 + warp;
    int pb = 0, pe = 0;
    if (k < k1) {
        pb = __ldg(bptr + k);
        pe = __ldg(bptr + k + 1);
    }
    float4 nxt = (k < k1 && lane < pe - pb) ? __ldg(rec + pb + lane) : zero4;
    while (k < k1) {
        const int kn = k + kWarps;
        int pbn = 0, pen = 0;
        if (kn < k1) {
            pbn = __ldg(bptr + kn);
            pen = __ldg(bptr + kn + 1);
        }
        const int row0 = k * R;
        CV<float, TPT> acc[R], xo[R];
        float dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const size_t base = (size_t)min(row0 + i, n - 1) * B + b0;
            xo[i] = ldv<float, TPT, true>(rj, base);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                dd[i][t] = row0 + i < n ? __ldg(d + base + t) : 0.f;
                acc[i].v[2 * t] = 0.f;
                acc[i].v[2 * t + 1] = 0.f;
            }
        }
        for (int e0 = pb; e0 < pe; e0 += 32) {
            __syncwarp();
            rbuf[warp][lane] = nxt;
            __syncwarp();
            if (e0 + 32 < pe) nxt = (e0 + 32 + lane < pe) ? __ldg(rec + e0 + 32 + lane) : zero4;
            else nxt = (kn < k1 && lane < pen - pbn) ? __ldg(rec + pbn + lane) : zero4;
            const int cnt = min(32, pe - e0);   // a multiple of 4
            for (int e = 0; e < cnt; e += 4) {
                float4 r[4];
                CV<float, TPT> y[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) r[q] = rbuf[warp][e + q];
#pragma unroll
                for (int q = 0; q < 4; ++q) y[q] = ldv<float, TPT, true>(rj, (size_t)__float_as_int(r[q].x) * B + b0);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    cfma<float, TPT>(acc[0], r[q].y, y[q]);
                    if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], r[q].z, y[q]);
                    if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], r[q].w, y[q]);
                }
            }
        }
        if (pe <= pb) nxt = (kn < k1 && lane < pen - pbn) ? __ldg(rec + pbn + lane) : zero4;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            if (row >= n) break;
            const size_t base = (size_t)row * B + b0;
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                acc[i].v[2 * t] = fmaf(dd[i][t], xo[i].v[2 * t], acc[i].v[2 * t]);
                acc[i].v[2 * t + 1] = fmaf(dd[i][t], xo[i].v[2 * t + 1], acc[i].v[2 * t + 1]);
            }
            if (kWrite) {
                CV<float, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    o.v[2 * t] = (float)(sc[t] * (double)acc[i].v[2 * t]);
                    o.v[2 * t + 1] = (float)(sc[t] * (double)acc[i].v[2 * t + 1]);
                    const double xr = xo[i].v[2 * t], xi = xo[i].v[2 * t + 1];
                    const double ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                    if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                    else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                }
                stv<float, TPT>(w, base, o);
            } else {
#pragma unroll
                for (int t = 0; t < TPT; ++t)
                    ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] + (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
            }
        }
        k = kn;
        pb = pbn;
        pe = pen;
    }
    __shared__ double2 red[kMaxTC];
    if (chunk_reduce<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double s2 = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s2 * s2;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s2 * s2;
            } else {
                S.nav[b] = sqrt(v.x) * s2;
            }
        }
    }
}

// SpMM over a TMA-fed shared-memory ring (staged = 6, LT = 2; staged = 7,
// LT = 4; complex64, packed records, R <= 3, TC = 32 trajectories, LT per
// lane; one 512-thread CTA per SM).  The CTA owns rows [r0, r1) of one chunk.  Ring block b holds rows
// y0 + b SR .. (y0 = r0 - halo, SR = 16 R rows: one block of R rows per
// warp per step); the ring has NB = 2hb + D + 1 blocks, so while step s
// gathers from blocks s .. s + 2hb the boxes of the next D blocks are in
// flight, and block s + NB is issued into block s's place once step s is
// done.  Warp w owns row block (r0 + s SR)/R + w: its records arrive 32 at a
// time (one coalesced 16-byte load per lane, the next batch in flight) into
// a per-warp buffer; the warp's lanes form 32 / (32 / LT) groups of 32 / LT
// lanes, group g takes records g, g + groups, ... of every batch for the same
// 32 trajectories, and shuffles add the groups.  With LT = 4 each record's
// coefficients serve twice the FMAs of LT = 2 for the same record traffic and
// slot arithmetic.  Every gather is a 16-byte shared load (two with LT = 4);
// no global load sits on the gathers' dependency chain.  Each mbarrier wait
// is bounded.
constexpr int kRingThreads = 512;

template <int R, bool kBilinear, bool kWrite, int LT = 2>
__global__ void __launch_bounds__(kRingThreads, 1) k_spmm_ring(int n, int B, int rows_per_cta, int hb, int D, int j,
                                                              const int* __restrict__ bptr,
                                                              const float4* __restrict__ rec,
                                                              const float* __restrict__ d, float* __restrict__ w,
                                                              BatchedScalars S, int nch,
                                                              const __grid_constant__ CUtensorMap tmap) {
    constexpr int TPT = LT, TC = 32;
    constexpr int GL = TC / TPT;   // lanes per record group
    constexpr int NG = 32 / GL;    // record groups per warp
    constexpr int QN = 8 / NG;     // records per group per pass (8 records per warp pass)
    constexpr int kWarps = kRingThreads / 32;
    constexpr int SR = kWarps * R;
    constexpr size_t row_reals = TC * 2;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* const smem_raw = align_smem128(smem_dyn);
    __shared__ __align__(8) uint64_t bars[32];
    __shared__ __align__(8) uint64_t never_bar;   // a barrier no copy completes (the timeout test hook)
    __shared__ float4 rbuf[kWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int half = lane / GL, hl = lane % GL;   // record group, lane within it
    const int NB = 2 * hb + D + 1;
    const int W = NB * SR;
    const int halo = hb * SR;
    const int chunk = blockIdx.y;
    if (chunk_converged(S, chunk)) return;
    // trajectories of this lane within the chunk: 2 hl, 2 hl + 1 (and, with
    // LT = 4, 16 + 2 hl, 17 + 2 hl), so each group's 16-byte shared loads
    // cover 128 contiguous bytes of a ring row (no bank conflicts)
    auto tj = [&](int t) { return (t < 2) ? 2 * hl + t : 16 + 2 * hl + (t - 2); };
    const int cb = chunk * TC;
    // one lane's values from a row of 32 interleaved complex64 (shared or global)
    auto ld_lane = [&](const float* rowp) {
        CV<float, TPT> v;
        const float4 a4 = *reinterpret_cast<const float4*>(rowp + 4 * hl);
        v.v[0] = a4.x; v.v[1] = a4.y; v.v[2] = a4.z; v.v[3] = a4.w;
        if constexpr (TPT == 4) {
            const float4 b4 = *reinterpret_cast<const float4*>(rowp + 32 + 4 * hl);
            v.v[4] = b4.x; v.v[5] = b4.y; v.v[6] = b4.z; v.v[7] = b4.w;
        }
        return v;
    };
    const int r0 = blockIdx.x * rows_per_cta;
    const int r1 = min(n, r0 + rows_per_cta);
    const int nsteps = r1 > r0 ? (r1 - r0 + SR - 1) / SR : 0;
    const int nbox = nsteps > 0 ? nsteps + 2 * hb : 0;
    const int y0 = r0 - halo;
    const int xc = chunk * TC * 2;
    float* ring = reinterpret_cast<float*>(smem_raw);
    const uint32_t box_bytes = (uint32_t)(SR * row_reals * sizeof(float));
    auto issue = [&](int b) {
        uint64_t* bar = &bars[b % NB];
        mbar_arrive_expect_tx(bar, box_bytes);
        tma_load_2d(ring + (size_t)(b % NB) * SR * row_reals, &tmap, bar, xc, y0 + b * SR);
    };
    if (threadIdx.x == 0) {
        for (int q = 0; q < NB; ++q) mbar_init(&bars[q], 1);
        mbar_init(&never_bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int b = 0; b < min(NB, nbox); ++b) issue(b);
    int issued = min(NB, nbox) - 1;
    double sc[TPT], ar[TPT], ai[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        sc[t] = S.sc[(size_t)j * B + cb + tj(t)];
        ar[t] = 0.0;
        ai[t] = 0.0;
    }
    // records past a block's end read as its first row with zero
    // coefficients, so every slot of a batch is a valid gather
    auto pad = [](int blk) { return make_float4(__int_as_float(blk * R), 0.f, 0.f, 0.f); };
    // this warp's block of step 0, its header and first record batch
    int k = r0 / R + warp;
    int pb = 0, pe = 0;
    if (nsteps > 0 && k * R < r1) {
        pb = __ldg(bptr + k);
        pe = __ldg(bptr + k + 1);
    }
    float4 nxt = lane < pe - pb ? __ldg(rec + pb + lane) : pad(k);
    for (int s = 0; s < nsteps; ++s) {
        const int row0 = k * R;
        const bool has_blk = row0 < r1;
        // next step's block header
        const int kn = k + kWarps;
        const bool has_next = s + 1 < nsteps && kn * R < r1;
        int pbn = 0, pen = 0;
        if (has_next) {
            pbn = __ldg(bptr + kn);
            pen = __ldg(bptr + kn + 1);
        }
        CV<float, TPT> acc[R], xo[R];
        float dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const size_t bse = (size_t)min(row0 + i, n - 1) * B + cb;
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                dd[i][t] = (has_blk && row0 + i < r1) ? __ldg(d + bse + tj(t)) : 0.f;
                acc[i].v[2 * t] = 0.f;
                acc[i].v[2 * t + 1] = 0.f;
            }
        }
        // rows of step s: ring blocks s .. s + 2hb (step 0 waits for all of
        // them, later steps for the one block that is new)
        const int bl = s + 2 * hb;
        int failed = -1;
        const long long budget = g_dq_wait_cycles;
        if (budget < 0 && s == 0) {
            // test hook: wait (|budget| cycles) for a barrier that nothing
            // completes, so the wait runs out and the timeout path below runs
            if (!mbar_wait_bounded(&never_bar, 0u, -budget)) failed = 0;
        }
        for (int q = (s == 0 ? 0 : bl); q <= bl; ++q)
            if (failed < 0 && !mbar_wait_bounded(&bars[q % NB], (uint32_t)((q / NB) & 1), budget < 0 ? kWaitCycles : budget))
                failed = q;
        if (__syncthreads_or(failed >= 0)) {
            if (threadIdx.x == 0) {
                atomicCAS(S.status, 0, DQ_ERR_TIMEOUT);
                // let every copy still in flight land (bounded) before leaving:
                // from the box this thread gave up on, or past the ones it saw land
                for (int q = (failed >= 0 ? failed : bl + 1); q <= issued; ++q)
                    mbar_wait_bounded(&bars[q % NB], (uint32_t)((q / NB) & 1));
            }
            return;
        }
        const int base = y0 + s * SR;
        const int q0 = (s % NB) * SR;
        auto slot = [&](int c) {
            int t = c - base + q0;
            t -= (t >= W) ? W : 0;
            return ring + (size_t)t * row_reals;
        };
        if (has_blk) {
            for (int e0 = pb; e0 < pe; e0 += 32) {
                __syncwarp();
                rbuf[warp][lane] = nxt;
                __syncwarp();
                if (e0 + 32 < pe) nxt = (e0 + 32 + lane < pe) ? __ldg(rec + e0 + 32 + lane) : pad(k);
                else nxt = (has_next && lane < pen - pbn) ? __ldg(rec + pbn + lane) : pad(kn);
                const int cnt = min(32, pe - e0);   // a multiple of 4
                // this group's records: e + NG q (slots past cnt are padding;
                // e + NG (QN - 1) <= 31 since e <= 24 + NG - 1)
                for (int e = half; e < cnt; e += 8) {
                    float4 r[QN];
                    CV<float, TPT> y[QN];
#pragma unroll
                    for (int q = 0; q < QN; ++q) r[q] = rbuf[warp][e + NG * q];
#pragma unroll
                    for (int q = 0; q < QN; ++q) y[q] = ld_lane(slot(__float_as_int(r[q].x)));
#pragma unroll
                    for (int q = 0; q < QN; ++q) {
                        cfma<float, TPT>(acc[0], r[q].y, y[q]);
                        if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], r[q].z, y[q]);
                        if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], r[q].w, y[q]);
                    }
                }
            }
        }
        if (pe <= pb) nxt = (has_next && lane < pen - pbn) ? __ldg(rec + pbn + lane) : pad(kn);
        // the groups add up; group 0 finishes the block
#pragma unroll
        for (int off = GL; off < 32; off <<= 1)
#pragma unroll
            for (int i = 0; i < R; ++i)
#pragma unroll
                for (int v = 0; v < 2 * TPT; ++v) acc[i].v[v] += __shfl_xor_sync(0xffffffffu, acc[i].v[v], off);
        if (has_blk && half == 0) {
            float far[TPT], fai[TPT];   // this block's alpha terms, one conversion per block
#pragma unroll
            for (int t = 0; t < TPT; ++t) { far[t] = 0.f; fai[t] = 0.f; }
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const int row = row0 + i;
                if (row >= r1) break;
                xo[i] = ld_lane(slot(row));
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    acc[i].v[2 * t] = fmaf(dd[i][t], xo[i].v[2 * t], acc[i].v[2 * t]);
                    acc[i].v[2 * t + 1] = fmaf(dd[i][t], xo[i].v[2 * t + 1], acc[i].v[2 * t + 1]);
                }
                if (kWrite) {
                    CV<float, TPT> o;
#pragma unroll
                    for (int t = 0; t < TPT; ++t) {
                        o.v[2 * t] = (float)sc[t] * acc[i].v[2 * t];
                        o.v[2 * t + 1] = (float)sc[t] * acc[i].v[2 * t + 1];
                        const float xr = xo[i].v[2 * t], xi = xo[i].v[2 * t + 1];
                        const float ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                        if (kBilinear) { far[t] += xr * ur - xi * ui; fai[t] += xr * ui + xi * ur; }
                        else { far[t] += xr * ur + xi * ui; fai[t] += xr * ui - xi * ur; }
                    }
                    float* wr = w + 2 * ((size_t)row * B + cb);
                    *reinterpret_cast<float4*>(wr + 4 * hl) = make_float4(o.v[0], o.v[1], o.v[2], o.v[3]);
                    if constexpr (TPT == 4)
                        *reinterpret_cast<float4*>(wr + 32 + 4 * hl) = make_float4(o.v[4], o.v[5], o.v[6], o.v[7]);
                } else {
#pragma unroll
                    for (int t = 0; t < TPT; ++t)
                        far[t] += acc[i].v[2 * t] * acc[i].v[2 * t] + acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
                }
            }
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                ar[t] += (double)far[t];
                ai[t] += (double)fai[t];
            }
        }
        __syncthreads();   // step s done: block s's place can take block s + NB
        if (threadIdx.x == 0 && s + NB < nbox) {
            issue(s + NB);
            issued = s + NB;
        }
        k = kn;
        pb = pbn;
        pe = pen;
    }
    __shared__ double2 red[kMaxTC];
    double2* scratch = reinterpret_cast<double2*>(smem_raw);   // the ring is free now
    if (chunk_reduce_s<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk, scratch)) {
        if (threadIdx.x < TC) {
            // red[i] belongs to trajectory tj(i % TPT) of lane i / TPT
            const int li = threadIdx.x / TPT, ti = threadIdx.x % TPT;
            const int b = chunk * TC + ((ti < 2) ? 2 * li + ti : 16 + 2 * li + (ti - 2));
            const double s2 = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s2 * s2;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s2 * s2;
            } else {
                S.nav[b] = sqrt(v.x) * s2;
            }
        }
    }
}

// Row-blocked SpMM with the gathered trajectory rows staged in shared
// memory.  The CTA owns rows [r0, r1) of one trajectory chunk and walks them
// in steps of SR rows; a ring of W = wmask+1 rows holds [a-halo, a+SR+halo)
// for the current step a, where halo >= the matrix bandwidth.  Thread 0
// issues the next step's SR new rows as one 2-D TMA box before the current
// step computes, so the copy overlaps the gathers (the ring holds two
// windows: W >= 2 halo + 2 SR).  Rows outside [0, n) arrive as zeros.
template <typename Real, int TPT, int R, bool kBilinear, bool kWrite>
__global__ void __launch_bounds__(kBThreads) k_spmm_win(int n, int B, int TC, int rows_per_cta, int halo, int wmask,
                                                       int j, const int* __restrict__ bptr,
                                                       const int* __restrict__ bcol, const Real* __restrict__ bcoef,
                                                       const Real* __restrict__ d, Real* __restrict__ w,
                                                       BatchedScalars S, int cy0, int nch,
                                                       const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* const smem_raw = align_smem128(smem_dyn);
    Real* win = reinterpret_cast<Real*>(smem_raw);   // [W][TC] complex
    __shared__ __align__(8) uint64_t bars[2];
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int BPS = blockDim.x / TPR;   // row blocks per step
    const int SR = BPS * R;             // rows per step
    const int tl = tr * TPT;
    const int chunk = blockIdx.y + cy0;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + tl;
    const int r0 = blockIdx.x * rows_per_cta;
    const int r1 = min(n, r0 + rows_per_cta);
    const int nsteps = r1 > r0 ? (r1 - r0 + SR - 1) / SR : 0;
    const int xc = chunk * TC * 2;
    const uint32_t box_bytes = (uint32_t)(SR * TC * 2 * sizeof(Real));
    auto slot = [&](int row) { return win + (size_t)(row & wmask) * TC * 2; };
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && nsteps > 0) {
        const int nbox = (2 * halo + SR) / SR;
        mbar_arrive_expect_tx(&bars[0], box_bytes * nbox);
        for (int q = 0; q < nbox; ++q) {
            const int y = r0 - halo + q * SR;
            tma_load_2d(slot(y), &tmap, &bars[0], xc, y);
        }
    }
    double sc[TPT], ar[TPT], ai[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        sc[t] = S.sc[(size_t)j * B + b0 + t];
        ar[t] = 0.0;
        ai[t] = 0.0;
    }
    int issued = 0;   // highest step whose load was issued
    constexpr bool kPk = sizeof(Real) == 4 && R <= 3;
    const float4* rec = reinterpret_cast<const float4*>(bcoef);
    BlkPre P;
    if constexpr (kPk) blk_prefetch(P, r0 + rl * R < r1, r0 / R + rl, bptr, rec);
    for (int s = 0; s < nsteps; ++s) {
        const int a = r0 + s * SR;
        BlkPre cur;
        if constexpr (kPk) {
            // this thread's block of the next step: rows a + SR + rl R
            cur = P;
            blk_prefetch(P, a + SR + rl * R < r1, (a + SR) / R + rl, bptr, rec);
        }
        __syncthreads();   // step s-1 done: the rows the next load overwrites are free
        if (threadIdx.x == 0 && s + 1 < nsteps) {
            const int y = a + SR + halo;
            mbar_arrive_expect_tx(&bars[(s + 1) & 1], box_bytes);
            tma_load_2d(slot(y), &tmap, &bars[(s + 1) & 1], xc, y);
        }
        if (s + 1 < nsteps) issued = s + 1;
        const bool ok = mbar_wait_bounded(&bars[s & 1], (uint32_t)((s >> 1) & 1), wait_budget());
        if (__syncthreads_or(!ok)) {
            // a copy never completed: flag it, give the copies in flight (this
            // step's and the next one's) a bounded chance to land, and leave
            // without reducing
            if (threadIdx.x == 0) {
                atomicCAS(S.status, 0, DQ_ERR_TIMEOUT);
                mbar_wait_bounded(&bars[s & 1], (uint32_t)((s >> 1) & 1));
                if (issued > s) mbar_wait_bounded(&bars[issued & 1], (uint32_t)((issued >> 1) & 1));
            }
            return;
        }
        const int k = a / R + rl;
        const int row0 = k * R;
        if (row0 < r1) {
            // diagonal loads issued first, applied after the union loop
            CV<Real, TPT> acc[R];
            Real dd[R][TPT];
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const int row = row0 + i;
                const size_t base = (size_t)min(row, n - 1) * B + b0;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    dd[i][t] = row < n ? __ldg(d + base + t) : Real(0);
                    acc[i].v[2 * t] = 0;
                    acc[i].v[2 * t + 1] = 0;
                }
            }
            auto gather = [&](int c) { return ldv<Real, TPT, false>(slot(c), tl); };
            if constexpr (kPk) union_loop_pre<TPT, R>(cur, rec, acc, gather);
            else union_any<Real, TPT, R>(__ldg(bptr + k), __ldg(bptr + k + 1), bcol, bcoef, acc, gather);
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const CV<Real, TPT> x = ldv<Real, TPT, false>(slot(row0 + i), tl);
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    acc[i].v[2 * t] = fma(dd[i][t], x.v[2 * t], acc[i].v[2 * t]);
                    acc[i].v[2 * t + 1] = fma(dd[i][t], x.v[2 * t + 1], acc[i].v[2 * t + 1]);
                }
            }
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const int row = row0 + i;
                if (row >= r1) break;
                const size_t base = (size_t)row * B + b0;
                if (kWrite) {
                    const CV<Real, TPT> x = ldv<Real, TPT, false>(slot(row), tl);
                    CV<Real, TPT> o;
#pragma unroll
                    for (int t = 0; t < TPT; ++t) {
                        o.v[2 * t] = (Real)(sc[t] * (double)acc[i].v[2 * t]);
                        o.v[2 * t + 1] = (Real)(sc[t] * (double)acc[i].v[2 * t + 1]);
                        const double xr = x.v[2 * t], xi = x.v[2 * t + 1], ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                        if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                        else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                    }
                    stv<Real, TPT>(w, base, o);
                } else {
#pragma unroll
                    for (int t = 0; t < TPT; ++t)
                        ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] + (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
                }
            }
        }
    }
    __shared__ double2 red[kMaxTC];
    if (chunk_reduce<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * nch, red, chunk)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double s2 = S.sc[(size_t)j * B + b];
            const double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s2 * s2;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s2 * s2;
            } else {
                S.nav[b] = sqrt(v.x) * s2;
            }
        }
    }
}

// One whole Lanczos iteration in one kernel (staged = 2).  Produces
//   r_j = cw w - (alpha_{j-1} sc_{j-1}) r_{j-1} - (beta_{j-2} sc_{j-2}) r_{j-2}
// (cw = 1 when w holds sc_{j-1} H r_{j-1}, sc_{j-1} when it holds H r_{j-1})
// from TMA-streamed boxes of w, r_{j-1} and r_{j-2} straight into a
// shared-memory ring, writes r_j for the CTA's own rows, and gathers
// H r_j from the ring: w_out = H r_j (unscaled) and <r_j, H r_j>, or, for the
// last iteration (kLast), only ||H r_j||.  One pass of the chunk reductions
// gives beta_{j-1} = ||r_j||, sc_j, alpha_j (or nav).
//
// The CTA owns rows [r0, r1) of one trajectory chunk.  Production blocks of
// SR rows start at y0 = r0 - halo (halo = hb SR >= the matrix bandwidth);
// SpMM step s (rows r0 + s SR ..) needs production blocks s .. s + 2hb, so the
// ring holds at least 2hb + 1 blocks and block p = s + 2hb is produced right
// before step s.  Input boxes run D production blocks ahead in D stages (one
// mbarrier each, every wait bounded).  Halo rows are produced by both
// neighbouring CTAs (identical values); each row is written and reduced by
// its owner only.  Rows outside [0, n) arrive as zeros.
struct FusedMaps {
    CUtensorMap w, r1, r2;
};

template <typename Real, int TPT, int R, bool kBilinear, bool kLast>
__global__ void __launch_bounds__(kBThreads) k_lanczos_fused(int n, int B, int TC, int rows_per_cta, int hb, int D,
                                                            int j, int w_scaled,
                                                            const int* __restrict__ bptr,
                                                            const int* __restrict__ bcol,
                                                            const Real* __restrict__ bcoef,
                                                            const Real* __restrict__ d, Real* __restrict__ r_out,
                                                            Real* __restrict__ w_out, BatchedScalars S, int nch,
                                                            const __grid_constant__ FusedMaps maps) {
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* const smem_raw = align_smem128(smem_dyn);
    __shared__ __align__(8) uint64_t bars[4];
    __shared__ double cf[kMaxTC][5];   // cw, Re/Im(alpha sc), beta sc, per trajectory of the chunk
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int BPS = blockDim.x / TPR;
    const int SR = BPS * R;
    const int halo = hb * SR;
    const int NB = 2 * hb + 1;                       // ring blocks
    const int W = NB * SR;                           // ring rows
    const int tl = tr * TPT;
    const int chunk = blockIdx.y;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + tl;
    const int r0 = blockIdx.x * rows_per_cta;
    const int r1 = min(n, r0 + rows_per_cta);
    const int nsteps = r1 > r0 ? (r1 - r0 + SR - 1) / SR : 0;
    const int NP = nsteps > 0 ? nsteps + 2 * hb : 0;  // production blocks
    const int y0 = r0 - halo;
    const int xc = chunk * TC * 2;
    const bool has2 = j > 2;                          // r_{j-2} exists
    const int nbox = has2 ? 3 : 2;
    const size_t row_reals = (size_t)TC * 2;
    // ring [W][TC] (production block p in ring block p mod NB), then D stages
    // of 3 boxes [SR][TC], each box 128-byte aligned
    Real* ring = reinterpret_cast<Real*>(smem_raw);
    const size_t box_reals = (size_t)SR * row_reals;
    const uint32_t box_bytes = (uint32_t)(box_reals * sizeof(Real));
    const size_t stage_off = ((size_t)W * row_reals * sizeof(Real) + 127) & ~(size_t)127;
    const size_t bstride = (((size_t)box_bytes + 127) & ~(size_t)127) / sizeof(Real);
    Real* stage = reinterpret_cast<Real*>(smem_raw + stage_off);
    auto issue = [&](int p) {
        const int st = p % D;
        uint64_t* bar = &bars[st];
        Real* dst = stage + (size_t)st * 3 * bstride;
        const int y = y0 + p * SR;
        mbar_arrive_expect_tx(bar, box_bytes * nbox);
        tma_load_2d(dst, &maps.w, bar, xc, y);
        tma_load_2d(dst + bstride, &maps.r1, bar, xc, y);
        if (has2) tma_load_2d(dst + 2 * bstride, &maps.r2, bar, xc, y);
    };
    if (threadIdx.x == 0) {
        for (int q = 0; q < D; ++q) mbar_init(&bars[q], 1);
        fence_barrier_init();
    }
    for (int t = threadIdx.x; t < TC; t += blockDim.x) {
        const int b = chunk * TC + t;
        const size_t k1 = (size_t)(j - 1) * B + b;
        const double s1 = S.sc[k1];
        cf[t][0] = w_scaled ? 1.0 : s1;
        cf[t][1] = S.alpha[2 * k1] * s1;
        cf[t][2] = S.alpha[2 * k1 + 1] * s1;
        cf[t][3] = has2 ? S.beta[(size_t)(j - 2) * B + b] * S.sc[(size_t)(j - 2) * B + b] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int p = 0; p < min(D, NP); ++p) issue(p);
    double cw[TPT], car[TPT], cai[TPT], cb[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        cw[t] = cf[tl + t][0];
        car[t] = cf[tl + t][1];
        cai[t] = cf[tl + t][2];
        cb[t] = cf[tl + t][3];
    }
    double nn[TPT], ar[TPT], ai[TPT], zero[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { nn[t] = 0.0; ar[t] = 0.0; ai[t] = 0.0; zero[t] = 0.0; }
    int issued = min(D, NP) - 1;
    constexpr bool kPk = sizeof(Real) == 4 && R <= 3;
    const float4* rec = reinterpret_cast<const float4*>(bcoef);
    for (int p = 0; p < NP; ++p) {
        const int st = p % D;
        // this step's block header, first records and diagonal are fetched
        // before the production phase, which hides their latency
        const int s = p - 2 * hb;
        const int k = (r0 + s * SR) / R + rl;
        const int row0 = k * R;
        const bool has_blk = s >= 0 && row0 < r1;
        BlkPre P;
        if constexpr (kPk) blk_prefetch(P, has_blk, k, bptr, rec);
        Real dd[R][TPT];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int row = row0 + i;
            const size_t base = (size_t)min(max(row, 0), n - 1) * B + b0;
#pragma unroll
            for (int t = 0; t < TPT; ++t) dd[i][t] = (has_blk && row < r1) ? __ldg(d + base + t) : Real(0);
        }
        const bool ok = mbar_wait_bounded(&bars[st], (uint32_t)((p / D) & 1), wait_budget());
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicCAS(S.status, 0, DQ_ERR_TIMEOUT);
                // box p itself may still be in flight: drain p .. issued
                for (int q = p; q <= issued; ++q) mbar_wait_bounded(&bars[q % D], (uint32_t)((q / D) & 1));
            }
            return;
        }
        // ---- produce r_j for rows y0 + p SR + rl R + i ----
        {
            const Real* sw = stage + (size_t)st * 3 * bstride;
            const Real* s1 = sw + bstride;
            const Real* s2 = sw + 2 * bstride;
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const int lr = rl * R + i;                // row within the block
                const int row = y0 + p * SR + lr;
                const size_t off = (size_t)lr * row_reals + tl * 2;
                const CV<Real, TPT> u = ldv<Real, TPT, false>(sw + off, 0);
                const CV<Real, TPT> x1 = ldv<Real, TPT, false>(s1 + off, 0);
                CV<Real, TPT> x2;
                if (has2) x2 = ldv<Real, TPT, false>(s2 + off, 0);
                CV<Real, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    const double xr = x1.v[2 * t], xi = x1.v[2 * t + 1];
                    double rr = cw[t] * (double)u.v[2 * t] - (car[t] * xr - cai[t] * xi);
                    double ri = cw[t] * (double)u.v[2 * t + 1] - (car[t] * xi + cai[t] * xr);
                    if (has2) {
                        rr -= cb[t] * (double)x2.v[2 * t];
                        ri -= cb[t] * (double)x2.v[2 * t + 1];
                    }
                    o.v[2 * t] = (Real)rr;
                    o.v[2 * t + 1] = (Real)ri;
                }
                stv<Real, TPT>(ring + (size_t)((p % NB) * SR + lr) * row_reals + tl * 2, 0, o);
                if (row >= r0 && row < r1) {
                    stv<Real, TPT>(r_out, (size_t)row * B + b0, o);
#pragma unroll
                    for (int t = 0; t < TPT; ++t)
                        nn[t] += (double)o.v[2 * t] * o.v[2 * t] + (double)o.v[2 * t + 1] * o.v[2 * t + 1];
                }
            }
        }
        __syncthreads();   // block p is in the ring; its stage is free
        if (threadIdx.x == 0 && p + D < NP) {
            issue(p + D);
            issued = p + D;
        }
        if (has_blk) {
            // ---- SpMM step s: rows row0 .. row0 + R of step s ----
            {
                CV<Real, TPT> acc[R];
#pragma unroll
                for (int i = 0; i < R; ++i)
#pragma unroll
                    for (int t = 0; t < TPT; ++t) {
                        acc[i].v[2 * t] = 0;
                        acc[i].v[2 * t + 1] = 0;
                    }
                // rows of step s lie in ring blocks s .. s + 2hb: row c sits at
                // c - base + q (mod W), base = y0 + s SR, q = (s mod NB) SR
                const int base = y0 + s * SR;
                const int q = (s % NB) * SR;
                auto slot = [&](int c) {
                    int t = c - base + q;
                    t -= (t >= W) ? W : 0;
                    return ring + (size_t)t * row_reals + tl * 2;
                };
                auto gather = [&](int c) { return ldv<Real, TPT, false>(slot(c), 0); };
                if constexpr (kPk) {
                    union_loop_pre<TPT, R>(P, rec, acc, gather);
                } else {
                    union_any<Real, TPT, R>(__ldg(bptr + k), __ldg(bptr + k + 1), bcol, bcoef, acc, gather);
                }
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    const int row = row0 + i;
                    if (row >= r1) break;
                    const CV<Real, TPT> x = ldv<Real, TPT, false>(slot(row), 0);
#pragma unroll
                    for (int t = 0; t < TPT; ++t) {
                        acc[i].v[2 * t] = fma(dd[i][t], x.v[2 * t], acc[i].v[2 * t]);
                        acc[i].v[2 * t + 1] = fma(dd[i][t], x.v[2 * t + 1], acc[i].v[2 * t + 1]);
                    }
                    if constexpr (kLast) {
#pragma unroll
                        for (int t = 0; t < TPT; ++t)
                            ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] +
                                     (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
                    } else {
                        stv<Real, TPT>(w_out, (size_t)row * B + b0, acc[i]);
#pragma unroll
                        for (int t = 0; t < TPT; ++t) {
                            const double xr = x.v[2 * t], xi = x.v[2 * t + 1];
                            const double ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                            if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                            else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                        }
                    }
                }
            }
        }
        __syncthreads();   // step s done: the next production may overwrite block s
    }
    // beta_{j-1} = ||r_j||, sc_j; then alpha_j = sc_j^2 <r_j, H r_j> (or nav).
    // The ring is free now (the loop ended on a barrier): it is the scratch.
    __shared__ double2 red[kMaxTC];
    double2* scratch = reinterpret_cast<double2*>(smem_raw);
    if (chunk_reduce_s<TPT>(nn, zero, TC, S.partial, S.tickets + 5 * nch, red, chunk, scratch)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            double bt = sqrt(red[threadIdx.x].x);
            if (!isfinite(bt)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            const size_t km = (size_t)(j - 1) * B + b;
            const double scale = sqrt(S.alpha[2 * km] * S.alpha[2 * km] + S.alpha[2 * km + 1] * S.alpha[2 * km + 1]) +
                                 (j > 2 ? S.beta[(size_t)(j - 2) * B + b] : 0.0);
            if (bt <= kBreakdownRel * scale) bt = 0.0;
            S.beta[km] = bt;
            S.sc[(size_t)j * B + b] = bt > 0.0 ? 1.0 / bt : 0.0;
        }
    }
    double* part2 = S.partial + (size_t)gridDim.y * gridDim.x * TC * 2;
    if (chunk_reduce_s<TPT>(ar, ai, TC, part2, S.tickets + 6 * nch, red, chunk, scratch)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double sj = __ldcg(&S.sc[(size_t)j * B + b]);
            const double2 v = red[threadIdx.x];
            if constexpr (kLast) {
                S.nav[b] = sqrt(v.x) * sj;
            } else {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * sj * sj;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * sj * sj;
            }
        }
    }
}

// Fused iteration with warp-owned row blocks (staged = 4; complex64,
// packed records, R <= 3, TC = 32 TPT; one 512-thread CTA per SM).  Same
// production ring and TMA stages as k_lanczos_fused, but the SpMM phase gives
// each of the 16 warps RB whole blocks of R rows per step (SR = 16 RB R
// rows), so a block's records are a
// warp-uniform stream read 32 at a time into a per-warp shared buffer (the
// next batch, or the next block's first one, in flight while the current
// batch is used) and every gather is a broadcast-free 16-byte shared load
// from the ring.  Lane l handles trajectories chunk TC + l TPT throughout.
constexpr int kFwThreads = 512;

template <int TPT, int R, bool kBilinear, bool kLast>
__global__ void __launch_bounds__(kFwThreads, 1) k_lanczos_fw(int n, int B, int rows_per_cta, int hb, int D, int RB, int j,
                                                         int w_scaled, const int* __restrict__ bptr,
                                                         const float4* __restrict__ rec,
                                                         const float* __restrict__ d, float* __restrict__ r_out,
                                                         float* __restrict__ w_out, BatchedScalars S, int nch,
                                                         const __grid_constant__ FusedMaps maps) {
    constexpr int TC = 32 * TPT;
    constexpr int kWarps = kFwThreads / 32;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* const smem_raw = align_smem128(smem_dyn);
    __shared__ __align__(8) uint64_t bars[4];
    __shared__ float4 rbuf[kWarps][32];
    __shared__ double cf[TC][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int SR = kWarps * RB * R;
    const int halo = hb * SR;
    const int NB = 2 * hb + 1;
    const int W = NB * SR;
    const int tl = lane * TPT;
    const int chunk = blockIdx.y;
    if (chunk_converged(S, chunk)) return;
    const int b0 = chunk * TC + tl;
    const int r0 = blockIdx.x * rows_per_cta;
    const int r1 = min(n, r0 + rows_per_cta);
    const int nsteps = r1 > r0 ? (r1 - r0 + SR - 1) / SR : 0;
    const int NP = nsteps > 0 ? nsteps + 2 * hb : 0;
    const int y0 = r0 - halo;
    const int xc = chunk * TC * 2;
    const bool has2 = j > 2;
    const int nbox = has2 ? 3 : 2;
    constexpr size_t row_reals = (size_t)TC * 2;
    float* ring = reinterpret_cast<float*>(smem_raw);
    const size_t box_reals = (size_t)SR * row_reals;
    const uint32_t box_bytes = (uint32_t)(box_reals * sizeof(float));
    const size_t stage_off = ((size_t)W * row_reals * sizeof(float) + 127) & ~(size_t)127;
    const size_t bstride = (((size_t)box_bytes + 127) & ~(size_t)127) / sizeof(float);
    float* stage = reinterpret_cast<float*>(smem_raw + stage_off);
    auto issue = [&](int p) {
        const int st = p % D;
        uint64_t* bar = &bars[st];
        float* dst = stage + (size_t)st * 3 * bstride;
        const int y = y0 + p * SR;
        mbar_arrive_expect_tx(bar, box_bytes * nbox);
        tma_load_2d(dst, &maps.w, bar, xc, y);
        tma_load_2d(dst + bstride, &maps.r1, bar, xc, y);
        if (has2) tma_load_2d(dst + 2 * bstride, &maps.r2, bar, xc, y);
    };
    if (threadIdx.x == 0) {
        for (int q = 0; q < D; ++q) mbar_init(&bars[q], 1);
        fence_barrier_init();
    }
    for (int t = threadIdx.x; t < TC; t += blockDim.x) {
        const int b = chunk * TC + t;
        const size_t k1 = (size_t)(j - 1) * B + b;
        const double s1 = S.sc[k1];
        cf[t][0] = w_scaled ? 1.0 : s1;
        cf[t][1] = S.alpha[2 * k1] * s1;
        cf[t][2] = S.alpha[2 * k1 + 1] * s1;
        cf[t][3] = has2 ? S.beta[(size_t)(j - 2) * B + b] * S.sc[(size_t)(j - 2) * B + b] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int p = 0; p < min(D, NP); ++p) issue(p);
    double cw[TPT], car[TPT], cai[TPT], cb[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        cw[t] = cf[tl + t][0];
        car[t] = cf[tl + t][1];
        cai[t] = cf[tl + t][2];
        cb[t] = cf[tl + t][3];
    }
    double nn[TPT], ar[TPT], ai[TPT], zero[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { nn[t] = 0.0; ar[t] = 0.0; ai[t] = 0.0; zero[t] = 0.0; }
    int issued = min(D, NP) - 1;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int p = 0; p < NP; ++p) {
        const int st = p % D;
        // this warp's first block of step s: header and first record batch
        // are fetched before the production phase, which hides them
        const int s = p - 2 * hb;
        const int kfirst = (r0 + s * SR) / R + warp * RB;
        int k = kfirst, pb = 0, pe = 0;
        float4 nxt = zero4;
        if (s >= 0 && k * R < r1) {
            pb = __ldg(bptr + k);
            pe = __ldg(bptr + k + 1);
            nxt = lane < pe - pb ? __ldg(rec + pb + lane) : zero4;
        }
        const bool ok = mbar_wait_bounded(&bars[st], (uint32_t)((p / D) & 1), wait_budget());
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicCAS(S.status, 0, DQ_ERR_TIMEOUT);
                // box p itself may still be in flight: drain p .. issued
                for (int q = p; q <= issued; ++q) mbar_wait_bounded(&bars[q % D], (uint32_t)((q / D) & 1));
            }
            return;
        }
        // ---- produce r_j: warp w writes rows lr = w, w + 8, ... of block p ----
        {
            const float* sw = stage + (size_t)st * 3 * bstride;
            const float* s1 = sw + bstride;
            const float* s2 = sw + 2 * bstride;
            float* blk = ring + (size_t)((p % NB) * SR) * row_reals;
            for (int lr = warp; lr < SR; lr += kWarps) {
                const int row = y0 + p * SR + lr;
                const size_t off = (size_t)lr * row_reals + tl * 2;
                const CV<float, TPT> u = ldv<float, TPT, false>(sw + off, 0);
                const CV<float, TPT> x1 = ldv<float, TPT, false>(s1 + off, 0);
                CV<float, TPT> x2;
                if (has2) x2 = ldv<float, TPT, false>(s2 + off, 0);
                CV<float, TPT> o;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    const double xr = x1.v[2 * t], xi = x1.v[2 * t + 1];
                    double rr = cw[t] * (double)u.v[2 * t] - (car[t] * xr - cai[t] * xi);
                    double ri = cw[t] * (double)u.v[2 * t + 1] - (car[t] * xi + cai[t] * xr);
                    if (has2) {
                        rr -= cb[t] * (double)x2.v[2 * t];
                        ri -= cb[t] * (double)x2.v[2 * t + 1];
                    }
                    o.v[2 * t] = (float)rr;
                    o.v[2 * t + 1] = (float)ri;
                }
                stv<float, TPT>(blk + off, 0, o);
                if (row >= r0 && row < r1) {
                    stv<float, TPT>(r_out, (size_t)row * B + b0, o);
#pragma unroll
                    for (int t = 0; t < TPT; ++t)
                        nn[t] += (double)o.v[2 * t] * o.v[2 * t] + (double)o.v[2 * t + 1] * o.v[2 * t + 1];
                }
            }
        }
        __syncthreads();   // block p is in the ring; its stage is free
        if (threadIdx.x == 0 && p + D < NP) {
            issue(p + D);
            issued = p + D;
        }
        if (s >= 0) {
            // ---- SpMM step s: this warp's RB blocks ----
            const int base = y0 + s * SR;
            const int q0 = (s % NB) * SR;
            auto slot = [&](int c) {
                int t = c - base + q0;
                t -= (t >= W) ? W : 0;
                return ring + (size_t)t * row_reals + tl * 2;
            };
            for (int ib = 0; ib < RB; ++ib, ++k) {
                const int row0 = k * R;
                if (row0 >= r1) break;
                // next block's header (its first batch is fetched during this block's last batch)
                const int kn = k + 1;
                const bool has_next = ib + 1 < RB && kn * R < r1;
                int pbn = 0, pen = 0;
                if (has_next) {
                    pbn = __ldg(bptr + kn);
                    pen = __ldg(bptr + kn + 1);
                }
                CV<float, TPT> acc[R];
                float dd[R][TPT];
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    const size_t bse = (size_t)min(row0 + i, n - 1) * B + b0;
#pragma unroll
                    for (int t = 0; t < TPT; ++t) {
                        dd[i][t] = row0 + i < r1 ? __ldg(d + bse + t) : 0.f;
                        acc[i].v[2 * t] = 0.f;
                        acc[i].v[2 * t + 1] = 0.f;
                    }
                }
                for (int e0 = pb; e0 < pe; e0 += 32) {
                    __syncwarp();
                    rbuf[warp][lane] = nxt;
                    __syncwarp();
                    if (e0 + 32 < pe) nxt = (e0 + 32 + lane < pe) ? __ldg(rec + e0 + 32 + lane) : zero4;
                    else nxt = (has_next && lane < pen - pbn) ? __ldg(rec + pbn + lane) : zero4;
                    const int cnt = min(32, pe - e0);   // a multiple of 4
                    for (int e = 0; e < cnt; e += 4) {
                        float4 r[4];
                        CV<float, TPT> y[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) r[q] = rbuf[warp][e + q];
#pragma unroll
                        for (int q = 0; q < 4; ++q) y[q] = ldv<float, TPT, false>(slot(__float_as_int(r[q].x)), 0);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            cfma<float, TPT>(acc[0], r[q].y, y[q]);
                            if constexpr (R > 1) cfma<float, TPT>(acc[R > 1 ? 1 : 0], r[q].z, y[q]);
                            if constexpr (R > 2) cfma<float, TPT>(acc[R > 2 ? 2 : 0], r[q].w, y[q]);
                        }
                    }
                }
                if (pe <= pb) nxt = (has_next && lane < pen - pbn) ? __ldg(rec + pbn + lane) : zero4;
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    const int row = row0 + i;
                    if (row >= r1) break;
                    const CV<float, TPT> x = ldv<float, TPT, false>(slot(row), 0);
#pragma unroll
                    for (int t = 0; t < TPT; ++t) {
                        acc[i].v[2 * t] = fmaf(dd[i][t], x.v[2 * t], acc[i].v[2 * t]);
                        acc[i].v[2 * t + 1] = fmaf(dd[i][t], x.v[2 * t + 1], acc[i].v[2 * t + 1]);
                    }
                    if constexpr (kLast) {
#pragma unroll
                        for (int t = 0; t < TPT; ++t)
                            ar[t] += (double)acc[i].v[2 * t] * acc[i].v[2 * t] +
                                     (double)acc[i].v[2 * t + 1] * acc[i].v[2 * t + 1];
                    } else {
                        stv<float, TPT>(w_out, (size_t)row * B + b0, acc[i]);
#pragma unroll
                        for (int t = 0; t < TPT; ++t) {
                            const double xr = x.v[2 * t], xi = x.v[2 * t + 1];
                            const double ur = acc[i].v[2 * t], ui = acc[i].v[2 * t + 1];
                            if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                            else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
                        }
                    }
                }
                pb = pbn;
                pe = pen;
            }
        }
        __syncthreads();   // step s done: the next production may overwrite block s
    }
    __shared__ double2 red[kMaxTC];
    double2* scratch = reinterpret_cast<double2*>(smem_raw);
    if (chunk_reduce_s<TPT>(nn, zero, TC, S.partial, S.tickets + 5 * nch, red, chunk, scratch)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            double bt = sqrt(red[threadIdx.x].x);
            if (!isfinite(bt)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            const size_t km = (size_t)(j - 1) * B + b;
            const double scale = sqrt(S.alpha[2 * km] * S.alpha[2 * km] + S.alpha[2 * km + 1] * S.alpha[2 * km + 1]) +
                                 (j > 2 ? S.beta[(size_t)(j - 2) * B + b] : 0.0);
            if (bt <= kBreakdownRel * scale) bt = 0.0;
            S.beta[km] = bt;
            S.sc[(size_t)j * B + b] = bt > 0.0 ? 1.0 / bt : 0.0;
        }
    }
    double* part2 = S.partial + (size_t)gridDim.y * gridDim.x * TC * 2;
    if (chunk_reduce_s<TPT>(ar, ai, TC, part2, S.tickets + 6 * nch, red, chunk, scratch)) {
        if (threadIdx.x < TC) {
            const int b = chunk * TC + threadIdx.x;
            const double sj = __ldcg(&S.sc[(size_t)j * B + b]);
            const double2 v = red[threadIdx.x];
            if constexpr (kLast) {
                S.nav[b] = sqrt(v.x) * sj;
            } else {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * sj * sj;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * sj * sj;
            }
        }
    }
}

// r_{j+1} = w - alpha_j q_j - beta_{j-1} q_{j-1};  beta_j = ||r_{j+1}||.
// rjm == nullptr: the SpMM already subtracted beta_{j-1} q_{j-1} from w.
template <typename Real, int TPT>
__global__ void __launch_bounds__(kBThreads) k_axpy_beta(int n, int B, int TC, int rpc, int j,
                                                        const Real* __restrict__ w, const Real* __restrict__ rj,
                                                        const Real* __restrict__ rjm, Real* __restrict__ rjp,
                                                        BatchedScalars S, int cy0, int nch) {
    const Tile<TPT> T(TC, rpc, n, cy0);
    if (chunk_converged(S, T.chunk)) return;
    const bool prev = j > 1 && rjm != nullptr;
    double ajr[TPT], aji[TPT], bm[TPT], nn[TPT], zero[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        const size_t k = (size_t)j * B + T.b0 + t;
        ajr[t] = S.alpha[2 * k] * S.sc[k];
        aji[t] = S.alpha[2 * k + 1] * S.sc[k];
        bm[t] = prev ? S.beta[(size_t)(j - 1) * B + T.b0 + t] * S.sc[(size_t)(j - 1) * B + T.b0 + t] : 0.0;
        nn[t] = 0.0;
        zero[t] = 0.0;
    }
    // two rows per trip so six independent loads are in flight per thread
    for (int row = T.r0 + T.rl; row < T.r1; row += 2 * T.RPC) {
        const int row2 = row + T.RPC;
        const bool has2 = row2 < T.r1;
        const size_t base = (size_t)row * B + T.b0;
        const size_t base2 = (size_t)(has2 ? row2 : row) * B + T.b0;
        CV<Real, TPT> u[2], x[2], xm[2];
        u[0] = ldv_cs<Real, TPT>(w, base);
        x[0] = ldv<Real, TPT, false>(rj, base);
        u[1] = ldv_cs<Real, TPT>(w, base2);
        x[1] = ldv<Real, TPT, false>(rj, base2);
        if (prev) {
            xm[0] = ldv_cs<Real, TPT>(rjm, base);
            xm[1] = ldv_cs<Real, TPT>(rjm, base2);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 1 && !has2) break;
            CV<Real, TPT> o;
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                const double xr = x[h].v[2 * t], xi = x[h].v[2 * t + 1];
                double rr = (double)u[h].v[2 * t] - (ajr[t] * xr - aji[t] * xi);
                double ri = (double)u[h].v[2 * t + 1] - (ajr[t] * xi + aji[t] * xr);
                if (prev) {
                    rr -= bm[t] * (double)xm[h].v[2 * t];
                    ri -= bm[t] * (double)xm[h].v[2 * t + 1];
                }
                o.v[2 * t] = (Real)rr;
                o.v[2 * t + 1] = (Real)ri;
                nn[t] += (double)o.v[2 * t] * o.v[2 * t] + (double)o.v[2 * t + 1] * o.v[2 * t + 1];
            }
            stv<Real, TPT>(rjp, h ? base2 : base, o);
        }
    }
    __shared__ double2 red[kMaxTC];
    if (chunk_reduce<TPT>(nn, zero, TC, S.partial, S.tickets + 1 * nch, red, T.chunk, T.bx)) {
        if (threadIdx.x < TC) {
            const int b = T.chunk * TC + threadIdx.x;
            double bt = sqrt(red[threadIdx.x].x);
            if (!isfinite(bt)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            // lucky breakdown: invariant Krylov space, continue with q_{j+1} = 0
            const size_t kj = (size_t)j * B + b;
            const double scale = sqrt(S.alpha[2 * kj] * S.alpha[2 * kj] + S.alpha[2 * kj + 1] * S.alpha[2 * kj + 1]) +
                                 (j > 1 ? S.beta[(size_t)(j - 1) * B + b] : 0.0);
            if (bt <= kBreakdownRel * scale) bt = 0.0;
            S.beta[kj] = bt;
            S.sc[(size_t)(j + 1) * B + b] = bt > 0.0 ? 1.0 / bt : 0.0;
        }
    }
}

// Full reorthogonalisation (Hermitian dot, cfg.reorth; classical
// Gram-Schmidt once, FP64 sums): after the axpy of iteration j, h_k =
// <q_k, r_{j+1}> for k = 1..j (k_reorth_dots_b), then r_{j+1} -= sum_k h_k q_k
// and beta_j, sc_{j+1} from its norm (k_reorth_apply_b).
// All h_k = <q_k, r_{j+1}>, k = 1..j, of full reorthogonalisation in one
// launch (classical Gram-Schmidt in blocks of kReorthKB): blockIdx.z picks
// the block of k, blockIdx.y the trajectory chunk, and each CTA reads r_{j+1}
// and that block's q_k over its row range once, so an iteration reads
// j + ceil(j / kReorthKB) slabs instead of the 2 j of one launch per k.
// FP64 sums, one ticket per (k block, chunk); the last CTA of each writes
// h_k into the combine-weight array (unused until the Padé step).
constexpr int kReorthKB = 8;
// ticket words per trajectory: regions 0..7 of the iteration kernels (one
// ticket per chunk each), the population ticket at 8 B, and from 9 B one
// region per block of k of the reorthogonalisation dots
constexpr int kReorthTicket = 9;
constexpr size_t kTicketWords = kReorthTicket + (kMaxL + kReorthKB - 1) / kReorthKB;

template <typename Real>
__global__ void __launch_bounds__(kBThreads, 2) k_reorth_dots_b(int n, int B, int TC, int rpc, int j,
                                                               const Real* __restrict__ slabs, size_t slab_stride,
                                                               BatchedScalars S, unsigned int* tickets, int cy0,
                                                               int nch) {
    // one trajectory per lane whatever the tiling (fewer live sums per
    // thread, so two CTAs fit per SM), two rows per trip so that 18
    // independent loads are in flight per thread
    constexpr int KQ = 2 * kReorthKB;   // complex h_k as two real sums each
    const int chunk = blockIdx.y + cy0, kb = blockIdx.z;
    const int k_first = 1 + kb * kReorthKB;
    const int tr = threadIdx.x % TC, rl = threadIdx.x / TC;
    const int RPC = blockDim.x / TC;
    const int b = chunk * TC + tr;
    const int r0 = blockIdx.x * rpc, r1 = min(n, r0 + rpc);
    if (chunk_converged(S, chunk)) return;
    const Real* r = slabs + 2 * slab_stride * (j + 1);
    double h[KQ][1];
    double sck[kReorthKB];
#pragma unroll
    for (int q = 0; q < kReorthKB; ++q) {
        const int k = k_first + q;
        sck[q] = k <= j ? S.sc[(size_t)k * B + b] : 0.0;
        h[2 * q][0] = h[2 * q + 1][0] = 0.0;
    }
    for (int row = r0 + rl; row < r1; row += 2 * RPC) {
        const int row2 = row + RPC;
        const bool two = row2 < r1;
        const size_t base = (size_t)row * B + b, base2 = (size_t)(two ? row2 : row) * B + b;
        const CV<Real, 1> v = ldv<Real, 1, false>(r, base);
        const CV<Real, 1> v2 = ldv<Real, 1, false>(r, base2);
        CV<Real, 1> x[kReorthKB], x2[kReorthKB];
#pragma unroll
        for (int q = 0; q < kReorthKB; ++q) {
            const int k = min(k_first + q, j);   // past j: a valid slab, weight 0
            x[q] = ldv<Real, 1, false>(slabs + 2 * slab_stride * k, base);
            x2[q] = ldv<Real, 1, false>(slabs + 2 * slab_stride * k, base2);
        }
        const double w2 = two ? 1.0 : 0.0;
#pragma unroll
        for (int q = 0; q < kReorthKB; ++q) {
            const double qr = sck[q] * x[q].v[0], qi = sck[q] * x[q].v[1];
            const double pr = sck[q] * w2 * x2[q].v[0], pi = sck[q] * w2 * x2[q].v[1];
            h[2 * q][0] += qr * v.v[0] + qi * v.v[1] + (pr * v2.v[0] + pi * v2.v[1]);   // conj(q) v
            h[2 * q + 1][0] += qr * v.v[1] - qi * v.v[0] + (pr * v2.v[1] - pi * v2.v[0]);
        }
    }
    __shared__ double red[KQ * kMaxTC];
    __shared__ double rsm[kBThreads];
    // each k block has its own tickets (one per chunk) and partial region
    double* part = S.partial + (size_t)kb * nch * gridDim.x * KQ * TC;
    if (chunk_reduce_multi<KQ, 1>(h, TC, part, tickets + (size_t)kb * nch, red, chunk, rsm)) {
        if (threadIdx.x < TC) {
            const int bb = chunk * TC + threadIdx.x;
            for (int q = 0; q < kReorthKB; ++q) {
                const int k = k_first + q;
                if (k > j) break;
                const size_t kbb = (size_t)k * B + bb;
                S.yt[2 * kbb] = red[(2 * q) * TC + threadIdx.x];
                S.yt[2 * kbb + 1] = red[(2 * q + 1) * TC + threadIdx.x];
            }
        }
    }
}

template <typename Real, int TPT>
__global__ void __launch_bounds__(kBThreads) k_reorth_apply_b(int n, int B, int TC, int rpc, int j, Real* slabs,
                                                             size_t slab_stride, BatchedScalars S, int cy0, int nch) {
    const Tile<TPT> T(TC, rpc, n, cy0);
    if (chunk_converged(S, T.chunk)) return;
    Real* r = slabs + 2 * slab_stride * (j + 1);
    // sc_k h_k of the CTA's trajectories, staged once instead of re-read per row
    __shared__ double2 hs[kMaxL][kMaxTC];
    for (int e = threadIdx.x; e < j * TC; e += blockDim.x) {
        const int k = 1 + e / TC, t = e % TC;
        const size_t kb = (size_t)k * B + T.chunk * TC + t;
        hs[k][t] = make_double2(S.yt[2 * kb] * S.sc[kb], S.yt[2 * kb + 1] * S.sc[kb]);
    }
    __syncthreads();
    double nn[TPT], zero[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { nn[t] = 0.0; zero[t] = 0.0; }
    for (int row = T.r0 + T.rl; row < T.r1; row += T.RPC) {
        const size_t base = (size_t)row * B + T.b0;
        const CV<Real, TPT> v0 = ldv<Real, TPT, false>(r, base);
        double vr[TPT], vi[TPT];
#pragma unroll
        for (int t = 0; t < TPT; ++t) { vr[t] = v0.v[2 * t]; vi[t] = v0.v[2 * t + 1]; }
        // eight q_k rows in flight at a time (the loads of a block are independent)
        for (int k0 = 1; k0 <= j; k0 += kReorthKB) {
            CV<Real, TPT> x[kReorthKB];
#pragma unroll
            for (int q = 0; q < kReorthKB; ++q)
                x[q] = ldv<Real, TPT, false>(slabs + 2 * slab_stride * min(k0 + q, j), base);
#pragma unroll
            for (int q = 0; q < kReorthKB; ++q) {
                const int k = k0 + q;
                if (k > j) break;
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    const double2 hk = hs[k][T.tr * TPT + t];
                    const double hr = hk.x, hi = hk.y;
                    vr[t] -= hr * x[q].v[2 * t] - hi * x[q].v[2 * t + 1];
                    vi[t] -= hr * x[q].v[2 * t + 1] + hi * x[q].v[2 * t];
                }
            }
        }
        CV<Real, TPT> o;
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            o.v[2 * t] = (Real)vr[t];
            o.v[2 * t + 1] = (Real)vi[t];
            nn[t] += (double)o.v[2 * t] * o.v[2 * t] + (double)o.v[2 * t + 1] * o.v[2 * t + 1];
        }
        stv<Real, TPT>(r, base, o);
    }
    __shared__ double2 red[kMaxTC];
    if (chunk_reduce<TPT>(nn, zero, TC, S.partial, S.tickets + 1 * nch, red, T.chunk)) {
        if (threadIdx.x < TC) {
            const int b = T.chunk * TC + threadIdx.x;
            double bt = sqrt(red[threadIdx.x].x);
            if (!isfinite(bt)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            const size_t kj = (size_t)j * B + b;
            const double scale = sqrt(S.alpha[2 * kj] * S.alpha[2 * kj] + S.alpha[2 * kj + 1] * S.alpha[2 * kj + 1]) +
                                 (j > 1 ? S.beta[(size_t)(j - 1) * B + b] : 0.0);
            if (bt <= kBreakdownRel * scale) bt = 0.0;
            S.beta[kj] = bt;
            S.sc[(size_t)(j + 1) * B + b] = bt > 0.0 ? 1.0 / bt : 0.0;
        }
    }
}

// ---- adaptive Krylov dimension (cfg.m_min > 0) -------------------------------
__global__ void k_adapt_reset(int B, int chunks, int mmax, BatchedScalars S) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
        S.mtraj[b] = 0;
        if (b < chunks) {
            S.cdone[b] = 0;
            S.mchunk[b] = mmax;
        }
    }
}

// One CTA per undecided trajectory after iteration j: EXPOKIT's first error
// term beta_j |E(j-1, j)| of exp(tau Tbar_j); the trajectory keeps dimension
// j when it meets the tolerance.
__global__ void k_mcheck_b(int j, int B, int TC, double tau_im, int norm_mode, double tol, BatchedScalars S) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ cd al[kMaxL], be[kMaxL];
    const int b = blockIdx.x;
    if (S.mtraj[b] != 0 || S.cdone[b / TC]) return;
    for (int i = threadIdx.x; i <= j + 1; i += blockDim.x) {
        const size_t k = (size_t)i * B + b;
        al[i] = (i >= 1 && i <= j) ? cmk(S.alpha[2 * k], S.alpha[2 * k + 1]) : cmk(0, 0);
        be[i] = (i >= 1 && i <= j) ? cmk(S.beta[k], 0.0) : cmk(0, 0);
    }
    __syncthreads();
    const PadeOut o = pade_exp_tbar(j, al, be, cmk(0.0, tau_im), norm_mode, nullptr, smem);
    if (threadIdx.x == 0 && o.s >= 0 && fabs(be[j].x) * sqrt(cabs2(o.e_m1_m)) <= tol) S.mtraj[b] = j;
}

// Per chunk: all trajectories decided -> its remaining iterations are skipped;
// the largest decided dimension bounds the combine.  final: undecided
// trajectories take the largest dimension.
__global__ void k_chunk_flags(int TC, int mmax, int final_pass, BatchedScalars S) {
    __shared__ int s_all, s_max;
    if (threadIdx.x == 0) { s_all = 1; s_max = 0; }
    __syncthreads();
    const int c = blockIdx.x;
    for (int t = threadIdx.x; t < TC; t += blockDim.x) {
        int mb = S.mtraj[c * TC + t];
        if (mb == 0 && final_pass) {
            mb = mmax;
            S.mtraj[c * TC + t] = mb;
        }
        if (mb == 0) atomicAnd(&s_all, 0);
        atomicMax(&s_max, mb);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_all) {
            S.cdone[c] = 1;
            S.mchunk[c] = s_max;
        }
    }
}

// one CTA per trajectory: exp(tau Tbar), combine weights, error estimate
__global__ void k_pade_b(int mmax, int B, double tau_im, int norm_mode, BatchedScalars S, double* erracc) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ cd al[kMaxL], be[kMaxL], y[kMaxM];
    const int b = blockIdx.x;
    // adaptive dimension: this trajectory's choice; weights past it are zero
    const int m = S.mtraj ? S.mtraj[b] : mmax;
    for (int j = threadIdx.x; j <= m + 1; j += blockDim.x) {
        const size_t k = (size_t)j * B + b;
        al[j] = (j >= 1 && j <= m) ? cmk(S.alpha[2 * k], S.alpha[2 * k + 1]) : cmk(0, 0);
        be[j] = (j >= 1 && j <= m) ? cmk(S.beta[k], 0.0) : cmk(0, 0);
    }
    __syncthreads();
    PadeOut o = pade_exp_tbar(m, al, be, cmk(0.0, tau_im), norm_mode, y, smem);
    if (o.s < 0) {
        if (threadIdx.x == 0) atomicCAS(S.status, 0, o.s == -1 ? DQ_ERR_SCALING : DQ_ERR_SINGULAR);
        return;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < mmax; j += blockDim.x) {
        const size_t k = (size_t)(j + 1) * B + b;
        const cd v = j < m ? cscale(y[j], S.sc[k]) : cmk(0.0, 0.0);
        S.yt[2 * k] = v.x;
        S.yt[2 * k + 1] = v.y;
    }
    if (threadIdx.x == 0) {
        // with the adaptive dimension only err1 (||H q_{m+1}|| belongs to the largest m)
        if (S.mtraj) erracc[b] += fmax(fabs(be[m].x) * sqrt(cabs2(o.e_m1_m)), 1.110223e-16);
        else erracc[b] += expokit_error(be[m].x, S.nav[b], o.e_m1_m, o.e_m1_mp1);
    }
}

// psi = sum_j yt_j r_j written over slab 1; ||psi||^2 and <psi0|psi> per
// trajectory; correlation point step+1 per chunk (propStep.cu:31-44,
// systemClass.cu:1771-1829, spectraClass.cu:510-571)
template <typename Real, int TPT>
__global__ void __launch_bounds__(kBThreads) k_combine_b(int n, int B, int TC, int rpc, int m,
                                                        Real* __restrict__ slabs, size_t slab_stride,
                                                        const cd* __restrict__ psi0, BatchedScalars S) {
    const Tile<TPT> T(TC, rpc, n);
    const int ch = T.chunk;
    const int step = *S.step;
    __shared__ double2 yts[kMaxM * kMaxTC];
    for (int e = threadIdx.x; e < m * TC; e += blockDim.x) {
        const int j = 1 + e / TC, b = ch * TC + e % TC;
        const size_t k = (size_t)j * B + b;
        yts[e] = make_double2(S.yt[2 * k], S.yt[2 * k + 1]);
    }
    __syncthreads();
    const int tl = T.b0 - ch * TC;   // trajectory lane within the chunk
    double nn[TPT], cr[TPT], ci[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { nn[t] = 0.0; cr[t] = 0.0; ci[t] = 0.0; }
    Real* r1 = slabs + 2 * slab_stride;
    if (S.mchunk) m = S.mchunk[ch];   // adaptive: the chunk's largest Krylov dimension
    for (int row = T.r0 + T.rl; row < T.r1; row += T.RPC) {
        const size_t base = (size_t)row * B + T.b0;
        double accr[TPT], acci[TPT];
#pragma unroll
        for (int t = 0; t < TPT; ++t) { accr[t] = 0.0; acci[t] = 0.0; }
        // eight slabs per trip: eight independent loads in flight per thread
        int j = 1;
        for (; j + 7 <= m; j += 8) {
            CV<Real, TPT> x[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) x[q] = ldv<Real, TPT, false>(slabs + 2 * slab_stride * (j + q), base);
#pragma unroll
            for (int q = 0; q < 8; ++q)
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    const double2 yv = yts[(j + q - 1) * TC + tl + t];
                    accr[t] += yv.x * x[q].v[2 * t] - yv.y * x[q].v[2 * t + 1];
                    acci[t] += yv.x * x[q].v[2 * t + 1] + yv.y * x[q].v[2 * t];
                }
        }
        for (; j + 3 <= m; j += 4) {
            CV<Real, TPT> x[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) x[q] = ldv<Real, TPT, false>(slabs + 2 * slab_stride * (j + q), base);
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int t = 0; t < TPT; ++t) {
                    const double2 yv = yts[(j + q - 1) * TC + tl + t];
                    accr[t] += yv.x * x[q].v[2 * t] - yv.y * x[q].v[2 * t + 1];
                    acci[t] += yv.x * x[q].v[2 * t + 1] + yv.y * x[q].v[2 * t];
                }
        }
        for (; j <= m; ++j) {
            const CV<Real, TPT> x = ldv<Real, TPT, false>(slabs + 2 * slab_stride * j, base);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                const double2 yv = yts[(j - 1) * TC + tl + t];
                accr[t] += yv.x * x.v[2 * t] - yv.y * x.v[2 * t + 1];
                acci[t] += yv.x * x.v[2 * t + 1] + yv.y * x.v[2 * t];
            }
        }
        CV<Real, TPT> o;
        const cd p0 = psi0[row];
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            o.v[2 * t] = (Real)accr[t];
            o.v[2 * t + 1] = (Real)acci[t];
            const double vr = o.v[2 * t], vi = o.v[2 * t + 1];
            nn[t] += vr * vr + vi * vi;
            cr[t] += p0.x * vr + p0.y * vi;   // conj(psi0) * psi
            ci[t] += p0.x * vi - p0.y * vr;
        }
        stv<Real, TPT>(r1, base, o);
    }
    __shared__ double2 red[kMaxTC];
    double zero[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) zero[t] = 0.0;
    if (chunk_reduce<TPT>(nn, zero, TC, S.partial, S.tickets + 3 * gridDim.y, red, T.chunk, T.bx)) {
        if (threadIdx.x < TC) {
            const int b = ch * TC + threadIdx.x;
            const double n2 = red[threadIdx.x].x;
            S.norm2[b] = n2;
            S.sc[B + b] = 1.0 / sqrt(n2);   // sc[1][b]: next step's q_1 = psi / ||psi||
            if (!(n2 > 0.0) || !isfinite(n2)) atomicCAS(S.status, 0, DQ_ERR_NAN);
        }
    }
    __syncthreads();
    // correlation of the normalised state: the last block of the second
    // ticket runs after every block of the chunk passed the first one, so the
    // chunk's norms are published by then
    double* part2 = S.partial + (size_t)gridDim.y * gridDim.x * TC * 2;
    if (chunk_reduce<TPT>(cr, ci, TC, part2, S.tickets + 4 * gridDim.y, red, T.chunk, T.bx)) {
        if (threadIdx.x == 0) {
            double sr = 0.0, si = 0.0;
            for (int t = 0; t < TC; ++t) {
                const int b = ch * TC + t;
                const double s1 = 1.0 / sqrt(__ldcg(&S.norm2[b]));
                sr += red[t].x * s1;
                si += red[t].y * s1;
            }
            double* cp = S.corr + ((size_t)(step + 1) * gridDim.y + ch) * 2;
            cp[0] = sr;
            cp[1] = si;
        }
    }
}

// populations: one warp per row, all trajectories, fixed order; advances the
// step counter in its last block
template <typename Real>
__global__ void k_pop_b(int n, int B, int pop_every, const Real* __restrict__ r1, double* __restrict__ pops,
                        BatchedScalars S, unsigned int* ticket) {
    const int step = *S.step;
    const bool due = ((step + 1) % pop_every) == 0;
    if (due) {
        double* row_out = pops + (size_t)((step + 1) / pop_every) * n;
        const int lane = threadIdx.x & 31;
        const int wpb = blockDim.x >> 5;
        for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < n; row += gridDim.x * wpb) {
            double s = 0.0;
            for (int b = lane; b < B; b += 32) {
                const size_t x = (size_t)row * B + b;
                const double vr = r1[2 * x], vi = r1[2 * x + 1];
                s += (vr * vr + vi * vi) / S.norm2[b];
            }
            s = warp_sum(s);
            if (lane == 0) row_out[row] += s;
        }
    }
    if (last_block_ticket(ticket, gridDim.x)) {
        if (threadIdx.x == 0) {
            *ticket = 0;
            *S.step = step + 1;
        }
    }
}

// ipr[step + 1] += sum_b 1 / sum_i (|r1_ib|^2 / ||r1_b||^2)^2 (systemClass.cu:2219-2257):
// one thread per trajectory sums a strided share of the rows (coalesced over
// trajectories); the last block adds the row-group partials in a fixed order.
template <typename Real>
__global__ void k_ipr_b(int n, int B, const Real* __restrict__ r1, BatchedScalars S, double* partial,
                        unsigned int* ticket, double* ipr) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    if (b < B) {
        const double inv = 1.0 / S.norm2[b];
        double s = 0.0;
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t x = (size_t)row * B + b;
            const double vr = r1[2 * x], vi = r1[2 * x + 1];
            const double a = (vr * vr + vi * vi) * inv;
            s += a * a;
        }
        partial[(size_t)blockIdx.x * B + b] = s;
    }
    if (last_block_ticket(ticket, gridDim.x * gridDim.y)) {
        __shared__ double scratch[32];
        double acc = 0.0;
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x) {
            double q = 0.0;
            for (unsigned int g = 0; g < gridDim.x; ++g) q += __ldcg(&partial[(size_t)g * B + bb]);
            acc += 1.0 / q;
        }
        acc = block_sum(acc, scratch);
        if (threadIdx.x == 0) {
            ipr[*S.step + 1] += acc;
            *ticket = 0;
        }
    }
}

// ipr[0] += B / sum_i |psi0_i|^4
__global__ void k_ipr_init_b(int n, int B, const cd* __restrict__ psi0, double* ipr) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = cabs2(psi0[i]);
        s += a * a;
    }
    s = block_sum(s, scratch);
    if (threadIdx.x == 0) ipr[0] += (double)B / s;
}

// initial record: pops[0] += B |psi0|^2, corr[0] = B <psi0|psi0> (B with a
// separate correlation bra: the reference stores M(0) = 1, spectraClass.cu:296)
__global__ void k_init_obs_b(int n, int B, const cd* __restrict__ psi0, double* pops, BatchedScalars S,
                             int chunks, int unit0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        pops[i] += (double)B * cabs2(psi0[i]);
    if (blockIdx.x == 0) {
        __shared__ double scratch[32];
        double s = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) s += cabs2(psi0[i]);
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) {
            for (int ch = 0; ch < chunks; ++ch) {
                S.corr[2 * ch] = (ch == 0) ? (double)B * (unit0 ? 1.0 : s) : 0.0;
                S.corr[2 * ch + 1] = 0.0;
            }
        }
    }
}

__global__ void k_set_norms_b(int n, int B, const cd* __restrict__ psi0, BatchedScalars S) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += cabs2(psi0[i]);
    s = block_sum(s, scratch);
    __shared__ double tot;
    if (threadIdx.x == 0) tot = s;
    __syncthreads();
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        S.norm2[b] = tot;
        S.sc[B + b] = 1.0 / sqrt(tot);
    }
    if (threadIdx.x == 0) { *S.step = 0; *S.status = 0; }
}

template <typename Real>
__global__ void k_get_states_b(int n, int B, const Real* __restrict__ r1, const BatchedScalars S, cd* __restrict__ out) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        for (int b = threadIdx.x; b < B; b += blockDim.x) {
            const size_t x = (size_t)i * B + b;
            const double s = 1.0 / sqrt(S.norm2[b]);
            out[(size_t)b * n + i] = cmk(r1[2 * x] * s, r1[2 * x + 1] * s);
        }
    }
}

// correlation sums over chunks -> d_corr (called by the getters)
__global__ void k_corr_collect(int np, int chunks, const double* __restrict__ corr_chunks, cd* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        double sr = 0.0, si = 0.0;
        for (int ch = 0; ch < chunks; ++ch) {
            sr += corr_chunks[((size_t)k * chunks + ch) * 2];
            si += corr_chunks[((size_t)k * chunks + ch) * 2 + 1];
        }
        out[k] = cmk(sr, si);
    }
}

// ---------------------------------------------------------------------------
#define DQ_CU(call)                                                     \
    do {                                                                \
        dq_status _s = check_cuda(c, (call), #call);                    \
        if (_s != DQ_OK) return _s;                                     \
    } while (0)

static void drop_graph(BatchedState* bs) {
    if (bs->exec) cudaGraphExecDestroy(bs->exec);
    if (bs->graph) cudaGraphDestroy(bs->graph);
    bs->exec = nullptr;
    bs->graph = nullptr;
}

static int r_index(int R) { return R == 1 ? 0 : R == 2 ? 1 : R == 3 ? 2 : R == 4 ? 3 : R == 8 ? 4 : -1; }

static void free_fmt(BlockFmt& f) {
    cudaFree(f.bptr); cudaFree(f.bcol); cudaFree(f.bcoef);
    f = BlockFmt();
}

static inline float __int_as_float_host(int v) {
    float f;
    std::memcpy(&f, &v, sizeof f);
    return f;
}

// Packed column-union records on the device (complex64, R <= 3, rows with
// non-decreasing columns): thread k merges the sorted column lists of block
// k's rows, summing each row's duplicate columns in CSR order in FP64 before
// the conversion, exactly as the host builder does, and pads the block to a
// multiple of 4 records with zero coefficients on its first row.  With
// pptr == nullptr it only counts (counts[k]); otherwise it writes the block's
// records from rec[pptr[k]].
template <int R>
__global__ void k_fmt_packed(int n, int nb, const int* __restrict__ rowptr, const int* __restrict__ col,
                             const double* __restrict__ val, const int* __restrict__ pptr, int* __restrict__ counts,
                             float4* __restrict__ rec) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const int r0 = k * R;
    int p[R], e[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const bool has = r0 + i < n;
        p[i] = has ? rowptr[r0 + i] : 0;
        e[i] = has ? rowptr[r0 + i + 1] : 0;
    }
    float4* out = pptr ? rec + pptr[k] : nullptr;
    int cnt = 0;
    for (;;) {
        int cmin = INT_MAX;
#pragma unroll
        for (int i = 0; i < R; ++i)
            if (p[i] < e[i]) cmin = min(cmin, col[p[i]]);
        if (cmin == INT_MAX) break;
        double cf[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < R; ++i)
            while (p[i] < e[i] && col[p[i]] == cmin) cf[i] += val[p[i]++];
        if (out) out[cnt] = make_float4(__int_as_float(cmin), (float)cf[0], (float)cf[1], (float)cf[2]);
        ++cnt;
    }
    while (cnt % 4) {
        if (out) out[cnt] = make_float4(__int_as_float(r0), 0.f, 0.f, 0.f);
        ++cnt;
    }
    if (!out) counts[k] = cnt;
}

static dq_status build_fmt_packed_device(dq_ctx* c, int R, BlockFmt& f) {
    const int n = c->n, nb = (n + R - 1) / R;
    int* counts = nullptr;
    DQ_CU(cudaMalloc(&counts, sizeof(int) * (size_t)nb));
    const int thr = 256, grid = (nb + thr - 1) / thr;
    auto launch = [&](const int* pptr, float4* rec) {
        switch (R) {
            case 1: k_fmt_packed<1><<<grid, thr, 0, c->stream>>>(n, nb, c->d_rowptr, c->d_col, c->d_val, pptr, counts, rec); break;
            case 2: k_fmt_packed<2><<<grid, thr, 0, c->stream>>>(n, nb, c->d_rowptr, c->d_col, c->d_val, pptr, counts, rec); break;
            default: k_fmt_packed<3><<<grid, thr, 0, c->stream>>>(n, nb, c->d_rowptr, c->d_col, c->d_val, pptr, counts, rec); break;
        }
    };
    launch(nullptr, nullptr);
    std::vector<int> pptr(nb + 1, 0);
    cudaError_t e = cudaMemcpyAsync(pptr.data() + 1, counts, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(counts);
    DQ_CU(e);
    for (int k = 0; k < nb; ++k) {
        f.max_block = std::max(f.max_block, pptr[k + 1]);
        pptr[k + 1] += pptr[k];
    }
    f.packed = true;
    f.nunion = (size_t)pptr[nb];
    DQ_CU(cudaMalloc(&f.bptr, sizeof(int) * (nb + 1)));
    DQ_CU(cudaMemcpyAsync(f.bptr, pptr.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, c->stream));
    DQ_CU(cudaMalloc(&f.bcoef, sizeof(float4) * std::max<size_t>(f.nunion, 1)));
    if (f.nunion) launch(f.bptr, reinterpret_cast<float4*>(f.bcoef));
    DQ_CU(cudaMalloc(&f.bcol, sizeof(int)));
    // pptr (host) must outlive the upload that reads it
    DQ_CU(cudaStreamSynchronize(c->stream));
    return DQ_OK;
}

// Builds the row-blocked column-union form of the (scaled) off-diagonal CSR.
static dq_status build_fmt(dq_ctx* c, int R, BlockFmt& f) {
    BatchedState* bs = c->bat;
    const int n = c->n, nb = (n + R - 1) / R;
    if (bs->mixed && R <= 3 && c->rows_sorted && c->nnz_off > 0) {
        bs->bw = c->bw;
        f.R = R;
        f.nb = nb;
        return build_fmt_packed_device(c, R, f);
    }
    std::vector<int> bptr(nb + 1, 0), bcol;
    std::vector<double> coef;
    std::vector<int> cols;
    bcol.reserve((size_t)c->nnz_off + nb);
    coef.reserve(((size_t)c->nnz_off + nb) * R);
    for (int k = 0; k < nb; ++k) {
        const int r0 = k * R, r1 = std::min(n, r0 + R);
        cols.clear();
        for (int r = r0; r < r1; ++r)
            for (int p = c->rowptr[r]; p < c->rowptr[r + 1]; ++p) cols.push_back(c->col[p]);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        const size_t base = bcol.size();
        bcol.insert(bcol.end(), cols.begin(), cols.end());
        coef.resize(bcol.size() * R, 0.0);
        for (int r = r0; r < r1; ++r)
            for (int p = c->rowptr[r]; p < c->rowptr[r + 1]; ++p) {
                const size_t u = base + (std::lower_bound(cols.begin(), cols.end(), c->col[p]) - cols.begin());
                coef[u * R + (r - r0)] += c->val[p];
            }
        bptr[k + 1] = (int)bcol.size();
    }
    int bw = 0;
    for (int r = 0; r < n; ++r)
        for (int p = c->rowptr[r]; p < c->rowptr[r + 1]; ++p) bw = std::max(bw, std::abs(c->col[p] - r));
    bs->bw = bw;
    f.R = R;
    f.nb = nb;
    if (bs->mixed && R <= 3) {
        // 16-byte records {col, c0, c1, c2}; every block padded to a multiple of
        // 4 records with zero coefficients on its own first row, so the kernel
        // loop needs neither clamps nor guards
        std::vector<float4> rec;
        std::vector<int> pptr(nb + 1, 0);
        for (int k = 0; k < nb; ++k) {
            const int u0 = bptr[k], u1 = bptr[k + 1];
            for (int u = u0; u < u1; ++u) {
                float4 r;
                r.x = __int_as_float_host(bcol[u]);
                r.y = (float)coef[(size_t)u * R];
                r.z = R > 1 ? (float)coef[(size_t)u * R + 1] : 0.f;
                r.w = R > 2 ? (float)coef[(size_t)u * R + 2] : 0.f;
                rec.push_back(r);
            }
            while ((rec.size() - (size_t)pptr[k]) % 4) {
                float4 r;
                r.x = __int_as_float_host(k * R);
                r.y = r.z = r.w = 0.f;
                rec.push_back(r);
            }
            pptr[k + 1] = (int)rec.size();
        }
        f.packed = true;
        f.nunion = rec.size();
        for (int k = 0; k < nb; ++k) f.max_block = std::max(f.max_block, pptr[k + 1] - pptr[k]);
        DQ_CU(cudaMalloc(&f.bptr, sizeof(int) * (nb + 1)));
        DQ_CU(cudaMemcpy(f.bptr, pptr.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice));
        DQ_CU(cudaMalloc(&f.bcoef, sizeof(float4) * std::max<size_t>(rec.size(), 1)));
        if (!rec.empty()) DQ_CU(cudaMemcpy(f.bcoef, rec.data(), sizeof(float4) * rec.size(), cudaMemcpyHostToDevice));
        DQ_CU(cudaMalloc(&f.bcol, sizeof(int)));
        return DQ_OK;
    }
    if (R == 3) return DQ_ERR_ARG;   // three rows per block only in the packed (complex64) form
    f.nunion = bcol.size();
    const size_t nu = std::max<size_t>(f.nunion, 1);
    DQ_CU(cudaMalloc(&f.bptr, sizeof(int) * (nb + 1)));
    DQ_CU(cudaMalloc(&f.bcol, sizeof(int) * nu));
    DQ_CU(cudaMemcpy(f.bptr, bptr.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice));
    if (f.nunion) DQ_CU(cudaMemcpy(f.bcol, bcol.data(), sizeof(int) * f.nunion, cudaMemcpyHostToDevice));
    if (bs->mixed) {
        std::vector<float> cf(coef.begin(), coef.end());
        DQ_CU(cudaMalloc(&f.bcoef, sizeof(float) * nu * R));
        if (f.nunion) DQ_CU(cudaMemcpy(f.bcoef, cf.data(), sizeof(float) * f.nunion * R, cudaMemcpyHostToDevice));
    } else {
        DQ_CU(cudaMalloc(&f.bcoef, sizeof(double) * nu * R));
        if (f.nunion) DQ_CU(cudaMemcpy(f.bcoef, coef.data(), sizeof(double) * f.nunion * R, cudaMemcpyHostToDevice));
    }
    return DQ_OK;
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2-D tensor map over one slab-shaped buffer (n rows of 2B reals), boxes of
// sr rows x 2tc reals.
static dq_status encode_slab_map(dq_ctx* c, void* base, int tc, int sr, CUtensorMap* map) {
    BatchedState* bs = c->bat;
    auto enc = tensor_map_encoder();
    if (!enc) {
        c->err = "cuTensorMapEncodeTiled unavailable";
        return DQ_ERR_CUDA;
    }
    const size_t rsz = bs->mixed ? sizeof(float) : sizeof(double);
    cuuint64_t dims[2] = {(cuuint64_t)(2 * bs->B), (cuuint64_t)c->n};
    cuuint64_t strides[1] = {(cuuint64_t)(2 * bs->B * rsz)};
    cuuint32_t box[2] = {(cuuint32_t)(2 * tc), (cuuint32_t)sr};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, bs->mixed ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        c->err = "cuTensorMapEncodeTiled failed";
        return DQ_ERR_CUDA;
    }
    return DQ_OK;
}

// One tensor map per slab (window SpMM).
static dq_status build_tmaps(dq_ctx* c, int tc, int sr) {
    BatchedState* bs = c->bat;
    const int m = c->cfg.m;
    const size_t rsz = bs->mixed ? sizeof(float) : sizeof(double);
    bs->tmaps.assign(m + 2, CUtensorMap{});
    for (int j = 0; j <= m + 1; ++j) {
        dq_status st = encode_slab_map(c, (char*)bs->slabs + (size_t)j * c->n * bs->B * 2 * rsz, tc, sr, &bs->tmaps[j]);
        if (st) return st;
    }
    return DQ_OK;
}

// Fused iteration: maps of slabs 0..m (w and the residuals it reads) and of wB.
static dq_status build_fmaps(dq_ctx* c, int tc, int sr) {
    BatchedState* bs = c->bat;
    const int m = c->cfg.m;
    const size_t rsz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)c->n * bs->B * 2 * rsz;
    if (!bs->wB) DQ_CU(cudaMalloc(&bs->wB, slab));
    bs->fmaps.assign(m + 2, CUtensorMap{});
    for (int j = 0; j <= m; ++j) {
        dq_status st = encode_slab_map(c, (char*)bs->slabs + (size_t)j * slab, tc, sr, &bs->fmaps[j]);
        if (st) return st;
    }
    return encode_slab_map(c, bs->wB, tc, sr, &bs->fmaps[m + 1]);
}

template <typename Real, int TPT, int R>
static cudaError_t win_attr(int bytes) {
    cudaError_t e = cudaSuccess;
    e = raise_smem_limit(k_spmm_win<Real, TPT, R, false, true>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_spmm_win<Real, TPT, R, true, true>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_spmm_win<Real, TPT, R, false, false>, bytes);
    return e;
}

template <typename Real, int TPT>
static cudaError_t win_attr_r(int R, int bytes) {
    switch (R) {
        case 1: return win_attr<Real, TPT, 1>(bytes);
        case 2: return win_attr<Real, TPT, 2>(bytes);
        case 3: return sizeof(Real) == 4 ? win_attr<Real, TPT, 3>(bytes) : cudaErrorInvalidValue;
        case 4: return win_attr<Real, TPT, 4>(bytes);
        default: return win_attr<Real, TPT, 8>(bytes);
    }
}

constexpr size_t kWinSmemMax = 200 * 1024;

// dynamic shared memory limit of every ring SpMM instance for R rows per block
template <int LT, int R>
static cudaError_t ring_attr_r(int bytes) {
    cudaError_t e = raise_smem_limit(k_spmm_ring<R, true, true, LT>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_spmm_ring<R, true, false, LT>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_spmm_ring<R, false, true, LT>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_spmm_ring<R, false, false, LT>, bytes);
    return e;
}

template <int LT>
static cudaError_t ring_attr(int R, int bytes) {
    return R == 1 ? ring_attr_r<LT, 1>(bytes) : R == 2 ? ring_attr_r<LT, 2>(bytes) : ring_attr_r<LT, 3>(bytes);
}

template <typename Real, int TPT, int R>
static cudaError_t fused_attr(int bytes) {
    cudaError_t e = raise_smem_limit(k_lanczos_fused<Real, TPT, R, false, false>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_lanczos_fused<Real, TPT, R, true, false>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_lanczos_fused<Real, TPT, R, false, true>, bytes);
    if (e == cudaSuccess)
        e = raise_smem_limit(k_lanczos_fused<Real, TPT, R, true, true>, bytes);
    return e;
}

template <typename Real, int TPT>
static cudaError_t fused_attr_r(int R, int bytes) {
    switch (R) {
        case 1: return fused_attr<Real, TPT, 1>(bytes);
        case 2: return fused_attr<Real, TPT, 2>(bytes);
        case 3: return sizeof(Real) == 4 ? fused_attr<Real, TPT, 3>(bytes) : cudaErrorInvalidValue;
        case 4: return fused_attr<Real, TPT, 4>(bytes);
        default: return fused_attr<Real, TPT, 8>(bytes);
    }
}

template <int TPT, int R>
static cudaError_t fw_attr(int bytes) {
    cudaError_t e = cudaSuccess;
    for (int v = 0; v < 4 && e == cudaSuccess; ++v) {
        const void* f = v == 0 ? (const void*)k_lanczos_fw<TPT, R, false, false>
                      : v == 1 ? (const void*)k_lanczos_fw<TPT, R, true, false>
                      : v == 2 ? (const void*)k_lanczos_fw<TPT, R, false, true>
                               : (const void*)k_lanczos_fw<TPT, R, true, true>;
        e = raise_smem_limit(f, bytes);
    }
    return e;
}

template <int TPT>
static cudaError_t fw_attr_r(int R, int bytes) {
    switch (R) {
        case 1: return fw_attr<TPT, 1>(bytes);
        case 2: return fw_attr<TPT, 2>(bytes);
        default: return fw_attr<TPT, 3>(bytes);
    }
}

// Shared memory of the fused iteration: ring of (2hb+1) SR rows, D stages of
// three 128-byte-aligned boxes of SR rows.
static size_t fused_smem(int tc, int sr, int hb, int D, size_t rsz) {
    const size_t row = (size_t)tc * 2 * rsz;
    const size_t ring = (((size_t)(2 * hb + 1) * sr * row) + 127) & ~(size_t)127;
    const size_t box = ((size_t)sr * row + 127) & ~(size_t)127;
    return ring + (size_t)D * 3 * box;
}

// Tiling: TC trajectories per chunk, TPT per thread, ~ctas_per_sm CTAs per
// SM, R rows per SpMM block, staged: TMA shared-memory window SpMM.
template <int R>
static cudaError_t cpa_attr(int bytes) {
    cudaError_t e = raise_smem_limit(k_spmm_cpa<R, false, true>, bytes);
    if (e == cudaSuccess) e = raise_smem_limit(k_spmm_cpa<R, true, true>, bytes);
    if (e == cudaSuccess) e = raise_smem_limit(k_spmm_cpa<R, false, false>, bytes);
    if (e == cudaSuccess) e = raise_smem_limit(k_spmm_cpa<R, true, false>, bytes);
    return e;
}

// The L1-gather forms in 512-thread CTAs (k_spmm_blk of staged 5, k_lanczos_p
// of staged 8) keep their gather window in L1: ask for the largest L1 share of
// the SM's unified L1/shared memory (their own shared memory is a few KB).
template <typename Real, int TPT, int R>
static void prefer_l1_r() {
    const int carve = cudaSharedmemCarveoutMaxL1;
    auto set = [&](const void* f) { cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carve); };
    set((const void*)k_spmm_blk<Real, TPT, R, false, true, 512>);
    set((const void*)k_spmm_blk<Real, TPT, R, true, true, 512>);
    set((const void*)k_spmm_blk<Real, TPT, R, false, false, 512>);
    set((const void*)k_spmm_blk<Real, TPT, R, true, false, 512>);
    set((const void*)k_lanczos_p<Real, TPT, R, false, 0, 512>);
    set((const void*)k_lanczos_p<Real, TPT, R, false, 1, 512>);
    set((const void*)k_lanczos_p<Real, TPT, R, false, 2, 512>);
    set((const void*)k_lanczos_p<Real, TPT, R, true, 0, 512>);
    set((const void*)k_lanczos_p<Real, TPT, R, true, 1, 512>);
    set((const void*)k_lanczos_p<Real, TPT, R, true, 2, 512>);
    cudaGetLastError();   // a hint: a refusal changes nothing
}

template <int R>
static void prefer_l1_lean() {
    const int carve = cudaSharedmemCarveoutMaxL1;
    auto set = [&](const void* f) { cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carve); };
    set((const void*)k_spmm_lean<R, false, true, 1024>);
    set((const void*)k_spmm_lean<R, true, true, 1024>);
    set((const void*)k_spmm_lean<R, false, false, 1024>);
    set((const void*)k_spmm_lean<R, true, false, 1024>);
    set((const void*)k_spmm_lean<R, false, true, 512>);
    set((const void*)k_spmm_lean<R, true, true, 512>);
    set((const void*)k_spmm_lean<R, false, false, 512>);
    set((const void*)k_spmm_lean<R, true, false, 512>);
    cudaGetLastError();   // a hint: a refusal changes nothing
}

template <int R>
static void prefer_l1_wg() {
    const int carve = cudaSharedmemCarveoutMaxL1;
    auto set = [&](const void* f) { cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carve); };
    set((const void*)k_spmm_wg<R, false, true>);
    set((const void*)k_spmm_wg<R, true, true>);
    set((const void*)k_spmm_wg<R, false, false>);
    set((const void*)k_spmm_wg<R, true, false>);
    set((const void*)k_spmm_wg<R, false, true, true>);
    set((const void*)k_spmm_wg<R, true, true, true>);
    cudaGetLastError();   // a hint: a refusal changes nothing
}

template <typename Real, int TPT>
static void prefer_l1(int R) {
    switch (R) {
        case 1: prefer_l1_r<Real, TPT, 1>(); break;
        case 2: prefer_l1_r<Real, TPT, 2>(); break;
        case 3: if constexpr (sizeof(Real) == 4) prefer_l1_r<Real, TPT, 3>(); break;
        case 4: prefer_l1_r<Real, TPT, 4>(); break;
        default: prefer_l1_r<Real, TPT, 8>(); break;
    }
}

dq_status batched_set_tiling(dq_ctx* c, int tc, int tpt, int ctas_per_sm, int R, int staged, int groups) {
    BatchedState* bs = c->bat;
    const int B = bs->B, n = c->n;
    if (tpt != 1 && tpt != 2) return DQ_ERR_ARG;
    if (!bs->mixed && tpt != 1) return DQ_ERR_ARG;
    if (tc < tpt || tc > kMaxTC || (tc & (tc - 1)) || B % tc || tc / tpt > kBThreads) return DQ_ERR_ARG;
    if (ctas_per_sm < 1 || ctas_per_sm > 16) return DQ_ERR_ARG;
    if (staged < 0 || staged > 12) return DQ_ERR_ARG;
    // reorthogonalisation runs between the axpy and the next SpMM: not in the fused forms
    if ((c->cfg.reorth || c->cfg.m_min > 0) && (staged == 2 || staged == 4 || staged == 8 || staged == 11))
        return DQ_ERR_ARG;
    // p-form iteration: one launch per iteration over all chunks
    if (staged == 8 && (groups != 1 || c->cfg.m < 2)) return DQ_ERR_ARG;
    // asynchronous-copy gathers: complex64 packed records, one warp per 64-trajectory block, one CTA per SM
    if (staged == 9 && (!bs->mixed || R > 3 || tc != 64 || tpt != 2 || ctas_per_sm != 1 || groups != 1))
        return DQ_ERR_ARG;
    // eight gathers in flight per warp (11: and the axpy in the same cooperative launch):
    // the same restrictions, chunk groups allowed
    if ((staged == 10 || staged == 11) && (!bs->mixed || R > 3 || tc != 64 || tpt != 2 || ctas_per_sm != 1))
        return DQ_ERR_ARG;
    // lean SpMM for 32 warps per SM: one 1024-thread CTA or two 512-thread CTAs per SM
    if (staged == 12 && (!bs->mixed || R > 3 || tpt != 2 || ctas_per_sm > 2)) return DQ_ERR_ARG;
    // ring SpMM: complex64 packed records, 32 trajectories per chunk, 2 per lane in the other
    // kernels (the ring itself takes 2 per lane with staged 6, 4 with staged 7), one CTA per SM
    const bool ring = staged == 6 || staged == 7;
    if (ring && (!bs->mixed || R > 3 || tc != 32 || tpt != 2 || ctas_per_sm != 1 || groups != 1))
        return DQ_ERR_ARG;
    if ((staged == 5 || staged == 8) && tc / tpt > 512) return DQ_ERR_ARG;
    // warp-per-block forms: complex64 packed records, one warp spans the chunk
    if ((staged == 3 || staged == 4) && (!bs->mixed || R > 3 || tc != 32 * tpt)) return DQ_ERR_ARG;
    const int ri = r_index(R);
    if (ri < 0) return DQ_ERR_ARG;
    const int chunks = B / tc;
    if (groups < 1 || chunks % groups) return DQ_ERR_ARG;
    const int cpg = chunks / groups;   // chunks per launch of the per-iteration kernels
    const int TPR = tc / tpt, RPC = kBThreads / TPR;
    const int RPC_spmm = (staged == 12 ? (ctas_per_sm == 1 ? 1024 : 512) : staged == 5 || staged >= 8 ? 512 : kBThreads) / TPR;   // row blocks in flight per SpMM CTA
    // bandwidth-bound per-row kernels (noise, axpy, combine) always run wide:
    // one wave of kStreamCtasPerSm CTAs per SM while every thread still walks
    // several rows, twice as many CTAs when that wave would leave each thread
    // fewer than 4 rows (small systems are latency-bound, not bandwidth-bound)
    int stream_per_sm = kStreamCtasPerSm;
    {
        const int g4 = std::max(1, (bs->sms * kStreamCtasPerSm) / cpg);
        if ((n + g4 - 1) / g4 < 4 * RPC) stream_per_sm = 2 * kStreamCtasPerSm;
    }
    int gx = std::max(1, (bs->sms * stream_per_sm) / cpg);
    int rpc = (n + gx - 1) / gx;
    rpc = ((rpc + RPC - 1) / RPC) * RPC;
    gx = (n + rpc - 1) / rpc;
    const int nb = (n + R - 1) / R;
    int gxs = std::max(1, (bs->sms * ctas_per_sm) / cpg);
    int bpc = (nb + gxs - 1) / gxs;
    bpc = ((bpc + RPC_spmm - 1) / RPC_spmm) * RPC_spmm;
    gxs = (nb + bpc - 1) / bpc;
    if (gx > kMaxCtasPerChunk || (size_t)gx * B * 2 > bs->partial_cap) return DQ_ERR_ARG;
    if (gxs > kMaxCtasPerChunk || (size_t)gxs * B * 2 > bs->partial_cap) return DQ_ERR_ARG;
    if (!bs->fmt[ri].bptr) {
        dq_status st = build_fmt(c, R, bs->fmt[ri]);
        if (st) return st;
    }
    if (staged == 9) {
        if (bs->fmt[ri].max_block > kCpaMaxRec) return DQ_ERR_ARG;
        cudaError_t e = cudaSuccess;
        const int bytes = (int)cpa_smem_bytes();
        switch (R) {
            case 1: e = cpa_attr<1>(bytes); break;
            case 2: e = cpa_attr<2>(bytes); break;
            default: e = cpa_attr<3>(bytes); break;
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            return DQ_ERR_ARG;
        }
    }
    if (staged == 8) {
        // six sums per trajectory per CTA in the partials; p_j ping-pongs between slab 0 and wB
        if ((size_t)gxs * B * 6 > bs->partial_cap) return DQ_ERR_ARG;
        if (!bs->wB) {
            const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
            DQ_CU(cudaMalloc(&bs->wB, (size_t)n * B * 2 * real_sz));
        }
    }
    int halo = 0, wmask = 0, rpc_win = 0, gxw = 0;
    size_t smem = 0;
    int f_sr = 0, f_hb = 0, f_D = 0, f_rpc = 0, f_gx = 0, f_rb = 1;
    size_t f_smem = 0;
    if (staged == 4) {
        // fused iteration with warp-owned blocks: the largest RB (blocks per
        // warp per step) and deepest staging that fit ctas_per_sm CTAs per SM
        // one 512-thread CTA per SM; the reduction scratch (2 x 512 double2)
        // lives in the dynamic region
        if (groups != 1 || c->cfg.m < 2 || ctas_per_sm != 1) return DQ_ERR_ARG;
        constexpr size_t kStatic = 13 * 1024;   // record buffers, coefficients, reduction slots, reserve
        for (int rb = 16 / R; rb >= 1 && !f_D; --rb) {
            const int SR = (kFwThreads / 32) * rb * R;
            if (SR > 256) continue;
            const int hb = (bs->bw + SR - 1) / SR;
            for (int D = 4; D >= 2; --D) {
                const size_t sm = std::max<size_t>(fused_smem(tc, SR, hb, D, sizeof(float)), 16384) + kSmemAlignPad;
                if (sm + kStatic <= 227 * 1024) {
                    f_D = D; f_smem = sm; f_sr = SR; f_hb = hb; f_rb = rb;
                    break;
                }
            }
        }
        if (!f_D) return DQ_ERR_ARG;
        f_gx = std::max(1, (bs->sms * ctas_per_sm) / chunks);
        f_rpc = (n + f_gx - 1) / f_gx;
        f_rpc = ((f_rpc + f_sr - 1) / f_sr) * f_sr;
        f_gx = (n + f_rpc - 1) / f_rpc;
        if (f_gx > kMaxCtasPerChunk || (size_t)f_gx * B * 2 > bs->partial_cap) return DQ_ERR_ARG;
        cudaError_t e = tpt == 2 ? fw_attr_r<2>(R, (int)f_smem) : fw_attr_r<1>(R, (int)f_smem);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return DQ_ERR_ARG;
        }
        dq_status st = build_fmaps(c, tc, f_sr);
        if (st) return st;
    }
    if (ring) {
        // ring SpMM: SR = 16 R rows per step; the deepest prefetch (D boxes)
        // whose ring fits one CTA per SM; the ring doubles as the reduction
        // scratch (512 / (32 / LT) x 32 double2)
        const int SR = (kRingThreads / 32) * R;
        const int hb = (bs->bw + SR - 1) / SR;
        constexpr size_t kStatic = 11 * 1024;   // record buffers, barriers, reduction slots, reserve
        const size_t min_sm = staged == 7 ? 32768 : 16384;
        for (int D = 4; D >= 1; --D) {
            const int NB = 2 * hb + D + 1;
            const size_t sm = std::max<size_t>((size_t)NB * SR * 32 * 2 * sizeof(float), min_sm) + kSmemAlignPad;
            if (NB <= 32 && sm + kStatic <= 227 * 1024) {
                f_D = D; f_smem = sm; f_sr = SR; f_hb = hb;
                break;
            }
        }
        if (!f_D) return DQ_ERR_ARG;
        f_gx = std::max(1, bs->sms / chunks);
        f_rpc = (n + f_gx - 1) / f_gx;
        f_rpc = ((f_rpc + SR - 1) / SR) * SR;
        f_gx = (n + f_rpc - 1) / f_rpc;
        if (f_gx > kMaxCtasPerChunk || (size_t)f_gx * B * 2 > bs->partial_cap) return DQ_ERR_ARG;
        cudaError_t e = staged == 7 ? ring_attr<4>(R, (int)f_smem) : ring_attr<2>(R, (int)f_smem);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return DQ_ERR_ARG;
        }
        dq_status st = build_tmaps(c, tc, SR);
        if (st) return st;
    }
    if (staged == 2) {
        // fused iteration: one launch covers every chunk, no trajectory groups
        const size_t rsz = bs->mixed ? sizeof(float) : sizeof(double);
        const int SR = RPC * R;
        if (groups != 1 || c->cfg.m < 2 || SR > 256 || 2 * tc > 256 || (tc * 2 * rsz) % 16) return DQ_ERR_ARG;
        f_sr = SR;
        f_hb = (bs->bw + SR - 1) / SR;
        // static shared memory (coefficient table, reduction slots, barriers)
        // plus the 1 KB the SM reserves per CTA; the per-SM pool is 228 KB
        constexpr size_t kStatic = 6 * 1024;
        f_D = 0;
        for (int D = 4; D >= 2; --D) {
            const size_t sm = fused_smem(tc, SR, f_hb, D, rsz) + kSmemAlignPad;
            if (sm <= kWinSmemMax && (size_t)ctas_per_sm * (sm + kStatic) <= 228 * 1024) {
                f_D = D;
                f_smem = sm;
                break;
            }
        }
        if (!f_D) return DQ_ERR_ARG;
        f_gx = std::max(1, (bs->sms * ctas_per_sm) / chunks);
        f_rpc = (n + f_gx - 1) / f_gx;
        f_rpc = ((f_rpc + SR - 1) / SR) * SR;
        f_gx = (n + f_rpc - 1) / f_rpc;
        if (f_gx > kMaxCtasPerChunk || (size_t)f_gx * B * 2 > bs->partial_cap) return DQ_ERR_ARG;
        cudaError_t e = bs->mixed ? (tpt == 2 ? fused_attr_r<float, 2>(R, (int)f_smem)
                                              : fused_attr_r<float, 1>(R, (int)f_smem))
                                  : fused_attr_r<double, 1>(R, (int)f_smem);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return DQ_ERR_ARG;
        }
        dq_status st = build_fmaps(c, tc, SR);
        if (st) return st;
    }
    if (staged == 1) {
        const size_t rsz = bs->mixed ? sizeof(float) : sizeof(double);
        const int SR = RPC * R;
        // boxes of SR rows tile the power-of-two ring without wrapping
        if (SR > 256 || (SR & (SR - 1)) || 2 * tc > 256 || tc * 2 * rsz < 16) return DQ_ERR_ARG;
        halo = ((bs->bw + SR - 1) / SR) * SR;
        int W = 1;
        while (W < 2 * halo + 2 * SR) W <<= 1;
        smem = (size_t)W * tc * 2 * rsz + kSmemAlignPad;
        if (smem > kWinSmemMax) return DQ_ERR_ARG;
        wmask = W - 1;
        const int fit = std::max(1, (int)((228 * 1024) / (smem + 12 * 1024)));
        gxw = std::max(1, (bs->sms * std::min(ctas_per_sm, fit)) / cpg);
        rpc_win = (n + gxw - 1) / gxw;
        rpc_win = ((rpc_win + SR - 1) / SR) * SR;
        gxw = (n + rpc_win - 1) / rpc_win;
        if (gxw > kMaxCtasPerChunk || (size_t)gxw * B * 2 > bs->partial_cap) return DQ_ERR_ARG;
        cudaError_t e = bs->mixed ? (tpt == 2 ? win_attr_r<float, 2>(R, (int)smem) : win_attr_r<float, 1>(R, (int)smem))
                                  : win_attr_r<double, 1>(R, (int)smem);
        if (e != cudaSuccess) return DQ_ERR_ARG;
        dq_status st = build_tmaps(c, tc, SR);
        if (st) return st;
    }
    if (staged == 5 || staged == 8) {
        if (!bs->mixed) prefer_l1<double, 1>(R);
        else if (tpt == 2) prefer_l1<float, 2>(R);
        else prefer_l1<float, 1>(R);
    }
    if (staged == 10 || staged == 11) {
        switch (R) {
            case 1: prefer_l1_wg<1>(); break;
            case 2: prefer_l1_wg<2>(); break;
            default: prefer_l1_wg<3>(); break;
        }
    }
    if (staged == 12) {
        switch (R) {
            case 1: prefer_l1_lean<1>(); break;
            case 2: prefer_l1_lean<2>(); break;
            default: prefer_l1_lean<3>(); break;
        }
    }
    if (staged == 11) {
        // the cooperative launch needs every block of a chunk group resident at once
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spmm_wg<3, false, true, true>, 512, 0) !=
                cudaSuccess ||
            occ < 1 || (size_t)gxs * cpg > (size_t)occ * bs->sms) {
            cudaGetLastError();
            return DQ_ERR_ARG;
        }
    }
    bs->TC = tc;
    bs->TPT = tpt;
    bs->chunks = chunks;
    bs->gx = gx;
    bs->rpc = rpc;
    bs->ctas_per_sm = ctas_per_sm;
    bs->R = R;
    bs->gxs = gxs;
    bs->bpc = bpc;
    bs->staged = staged;
    bs->groups = groups;
    bs->halo = halo;
    bs->wmask = wmask;
    bs->rpc_win = rpc_win;
    bs->gxw = gxw;
    bs->win_smem = smem;
    bs->f_sr = f_sr;
    bs->f_hb = f_hb;
    bs->f_D = f_D;
    bs->f_rpc = f_rpc;
    bs->f_gx = f_gx;
    bs->f_smem = f_smem;
    bs->f_rb = f_rb;
    drop_graph(bs);
    return DQ_OK;
}

// The couplings changed: drop every block format and rebuild the one the
// current tiling uses (falling back to the unstaged SpMM when the new
// matrix's bandwidth no longer fits the staged window).
dq_status batched_invalidate_blocks(dq_ctx* c) {
    BatchedState* bs = c->bat;
    if (!bs) return DQ_OK;
    for (auto& f : bs->fmt) free_fmt(f);
    drop_graph(bs);
    if (!bs->TC) return DQ_OK;
    dq_status st = batched_set_tiling(c, bs->TC, bs->TPT, bs->ctas_per_sm, bs->R, bs->staged, bs->groups);
    if (st && bs->staged) st = batched_set_tiling(c, bs->TC, bs->TPT, bs->ctas_per_sm, bs->R, 0, bs->groups);
    if (st) c->err = "batched: could not rebuild the coupling blocks";
    return st;
}

// Gives dst (a second workspace of the same B and precision) the tiling of
// c->bat.  The block formats are shared (dst does not own them); the staged
// SpMM's tensor maps are built on dst's own slabs.
dq_status batched_mirror_tiling(dq_ctx* c, BatchedState* dst) {
    BatchedState* src = c->bat;
    if (!src || !dst || dst->B != src->B || dst->mixed != src->mixed) return DQ_ERR_STATE;
    drop_graph(dst);
    if (!dst->fmt_borrowed)
        for (auto& f : dst->fmt) free_fmt(f);
    for (int k = 0; k < 5; ++k) dst->fmt[k] = src->fmt[k];
    dst->fmt_borrowed = true;
    dst->TC = src->TC; dst->TPT = src->TPT; dst->chunks = src->chunks; dst->gx = src->gx; dst->rpc = src->rpc;
    dst->ctas_per_sm = src->ctas_per_sm; dst->R = src->R; dst->gxs = src->gxs; dst->bpc = src->bpc;
    dst->staged = src->staged; dst->groups = src->groups; dst->halo = src->halo; dst->wmask = src->wmask;
    dst->rpc_win = src->rpc_win; dst->gxw = src->gxw; dst->bw = src->bw; dst->win_smem = src->win_smem;
    dst->f_sr = src->f_sr; dst->f_hb = src->f_hb; dst->f_D = src->f_D; dst->f_rpc = src->f_rpc;
    dst->f_gx = src->f_gx; dst->f_smem = src->f_smem; dst->f_rb = src->f_rb;
    dst->tmaps.clear();
    dst->fmaps.clear();
    if (src->staged == 2 || src->staged == 4) {
        c->bat = dst;
        dq_status st = build_fmaps(c, src->TC, src->f_sr);
        c->bat = src;
        if (st) return st;
    }
    if (src->staged == 8 && !dst->wB) {
        const size_t real_sz = dst->mixed ? sizeof(float) : sizeof(double);
        DQ_CU(cudaMalloc(&dst->wB, (size_t)c->n * dst->B * 2 * real_sz));
    }
    if (src->staged == 1 || src->staged == 6 || src->staged == 7) {
        const int SR = src->staged >= 6 ? src->f_sr : (kBThreads / (src->TC / src->TPT)) * src->R;
        c->bat = dst;
        dq_status st = build_tmaps(c, src->TC, SR);
        c->bat = src;
        if (st) return st;
    }
    return DQ_OK;
}

// Allocates and initialises one workspace of B trajectories and attaches it
// to c->bat (the caller restores c->bat when the workspace is a second one).
static dq_status alloc_ws_into(dq_ctx* c, BatchedState* bs, int B, bool mixed, bool default_tiling = true) {
    const int n = c->n, m = c->cfg.m;
    c->bat = bs;
    bs->B = B;
    bs->mixed = mixed;
    cudaDeviceGetAttribute(&bs->sms, cudaDevAttrMultiProcessorCount, c->cfg.device);
    if (B % 2 && bs->mixed) {
        c->err = "batched: n_traj must be even for the mixed path";
        return DQ_ERR_ARG;
    }
    const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)n * B * 2 * real_sz;
    DQ_CU(cudaMalloc(&bs->slabs, slab * (m + 2)));
    DQ_CU(cudaMemsetAsync(bs->slabs, 0, slab * (m + 2), c->stream));
    DQ_CU(cudaMalloc(&bs->diag, (size_t)n * B * real_sz));
    DQ_CU(cudaMalloc(&bs->eps, sizeof(double) * (size_t)n * B));
    DQ_CU(cudaMalloc(&bs->deps, sizeof(double) * (size_t)n * B));
    if (c->cfg.noise_model == DQ_NOISE_ZZ) {
        DQ_CU(cudaMalloc(&bs->zzD, sizeof(double) * (size_t)kZZBlock * n * B));
        DQ_CU(cudaMalloc(&bs->zz_start, sizeof(int)));
        DQ_CU(cudaMemsetAsync(bs->zz_start, 0xC0, sizeof(int), c->stream));   // no block stored
    }
    const size_t LB = (size_t)kMaxL * B;
    // partial capacity: up to 16 CTAs per SM over all chunks, 2 doubles per trajectory
    bs->partial_cap = (size_t)std::min(kMaxCtasPerChunk, bs->sms * 16) * B * 2;
    const size_t corr_n = (size_t)(c->cfg.max_steps + 1) * B * 2;   // chunks <= B
    const size_t total = LB * 2 + LB + LB + LB * 2 + B + B + 2 * bs->partial_cap + corr_n;
    DQ_CU(cudaMalloc(&bs->scal_mem, sizeof(double) * total));
    DQ_CU(cudaMemsetAsync(bs->scal_mem, 0, sizeof(double) * total, c->stream));
    double* p = bs->scal_mem;
    bs->s.alpha = p; p += LB * 2;
    bs->s.beta = p; p += LB;
    bs->s.sc = p; p += LB;
    bs->s.yt = p; p += LB * 2;
    bs->s.nav = p; p += B;
    bs->s.norm2 = p; p += B;
    bs->s.partial = p; p += 2 * bs->partial_cap;
    bs->s.corr = p; p += corr_n;
    const size_t nt = kTicketWords * (size_t)B + 8;
    DQ_CU(cudaMalloc(&bs->s.tickets, sizeof(unsigned int) * nt));
    DQ_CU(cudaMemsetAsync(bs->s.tickets, 0, sizeof(unsigned int) * nt, c->stream));
    DQ_CU(cudaMalloc(&bs->s.status, sizeof(int) * 2));
    bs->s.step = bs->s.status + 1;
    DQ_CU(cudaMemsetAsync(bs->s.status, 0, sizeof(int) * 2, c->stream));
    bs->s.mtraj = bs->s.cdone = bs->s.mchunk = nullptr;
    if (c->cfg.m_min > 0) {
        DQ_CU(cudaMalloc(&bs->s.mtraj, sizeof(int) * 3 * (size_t)B));
        DQ_CU(cudaMemsetAsync(bs->s.mtraj, 0, sizeof(int) * 3 * (size_t)B, c->stream));
        bs->s.cdone = bs->s.mtraj + B;
        bs->s.mchunk = bs->s.cdone + B;
    }
    DQ_CU(raise_smem_limit(k_pade_b, (int)pade_smem_bytes(m + 2)));
    DQ_CU(raise_smem_limit(k_mcheck_b, (int)pade_smem_bytes(m + 2)));
    // default tiling (dq_autotune refines it); left out when the caller sets
    // one right away, so only that tiling's coupling blocks are built
    if (!default_tiling) return DQ_OK;
    return batched_default_tiling(c);
}

dq_status batched_default_tiling(dq_ctx* c) {
    BatchedState* bs = c->bat;
    const int B = bs->B;
    int tpt = bs->mixed ? 2 : 1;
    int tc = 16;
    while (tc > tpt && B % tc) tc >>= 1;
    if (B % tc) tc = tpt;
    dq_status st = batched_set_tiling(c, tc, tpt, 2, 4, 0, 1);
    if (st) {
        c->err = "batched: no valid tiling for n_traj";
        return st;
    }
    return DQ_OK;
}

dq_status batched_alloc(dq_ctx* c, bool default_tiling) {
    BatchedState* bs = new BatchedState();
    return alloc_ws_into(c, bs, c->cfg.n_traj, c->cfg.precision == DQ_PREC_MIXED, default_tiling);
}

BatchedState* batched_alloc_ws(dq_ctx* c, int B, bool mixed, dq_status* st) {
    BatchedState* saved = c->bat;
    BatchedState* bs = new BatchedState();
    *st = alloc_ws_into(c, bs, B, mixed);
    c->bat = saved;
    if (*st) {
        batched_free_ws(bs);
        return nullptr;
    }
    return bs;
}

void batched_free(dq_ctx* c) {
    batched_free_ws(c->bat);
    c->bat = nullptr;
}

void batched_free_ws(BatchedState* bs) {
    if (!bs) return;
    drop_graph(bs);
    if (!bs->fmt_borrowed)
        for (auto& f : bs->fmt) free_fmt(f);
    cudaFree(bs->wB);
    cudaFree(bs->slabs); cudaFree(bs->diag); cudaFree(bs->eps); cudaFree(bs->deps);
    cudaFree(bs->zzD); cudaFree(bs->zz_start);
    cudaFree(bs->scal_mem); cudaFree(bs->s.tickets); cudaFree(bs->s.status); cudaFree(bs->s.mtraj);
    delete bs;
}

dq_status batched_reset(dq_ctx* c) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B;
    const int blocks = std::min(n, bs->sms * 8);
    const int thr = std::min(256, ((B + 31) / 32) * 32);
    // a setter may have re-allocated a parameter array the captured step reads
    drop_graph(bs);
    k_traj_init_b<<<blocks, thr, 0, c->stream>>>(n, B, c->traj0, c->cfg.seed, c->d_h0, c->d_static, c->cfg.sigma_static,
                                                 c->d_sigma, c->cfg.noise_model, bs->eps, bs->deps);
    if (c->cfg.noise_model == DQ_NOISE_ZZ) {
        if (!bs->zzD) {
            // the density was set after this workspace was made
            DQ_CU(cudaMalloc(&bs->zzD, sizeof(double) * (size_t)kZZBlock * n * B));
            DQ_CU(cudaMalloc(&bs->zz_start, sizeof(int)));
        }
        DQ_CU(cudaMemsetAsync(bs->zz_start, 0xC0, sizeof(int), c->stream));   // no block stored
    }
    const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)n * B * 2 * real_sz;
    if (bs->mixed)
        k_set_psi0_b<float><<<blocks, thr, 0, c->stream>>>(n, B, c->d_psi0, (float*)((char*)bs->slabs + slab));
    else
        k_set_psi0_b<double><<<blocks, thr, 0, c->stream>>>(n, B, c->d_psi0, (double*)((char*)bs->slabs + slab));
    DQ_CU(cudaMemsetAsync(bs->s.tickets, 0, sizeof(unsigned int) * (kTicketWords * (size_t)B + 8), c->stream));
    k_set_norms_b<<<1, 256, 0, c->stream>>>(n, B, c->d_psi0, bs->s);
    k_init_obs_b<<<std::max(1, std::min(bs->sms, (n + 255) / 256)), 256, 0, c->stream>>>(n, B, c->d_psi0, c->d_pops,
                                                                                        bs->s, bs->chunks,
                                                                                        c->d_bra != nullptr);
    if (c->ipr_on) k_ipr_init_b<<<1, 256, 0, c->stream>>>(n, B, c->d_psi0, c->d_ipr);
    DQ_CU(cudaGetLastError());
    return DQ_OK;
}

// Optional per-kernel timing of an eagerly launched step: an event is
// recorded before every launch; the time to the next event is charged to the
// kernel kind launched in between.
struct StepTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    void mark(int k, cudaStream_t st) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev.push_back(e);
        kind.push_back(k);
    }
    void collect(double* ms, int* cnt, int nk) {
        for (size_t i = 0; i + 1 < ev.size(); ++i) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            if (kind[i] >= 0 && kind[i] < nk) { ms[kind[i]] += t; cnt[kind[i]] += 1; }
        }
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
        kind.clear();
    }
};

// The forms that run k_spmm_blk (L1 gathers, 256- or 512-thread CTAs).
static bool spmm_subtracts_prev(const BatchedState* bs) {
    return bs->staged == 0 || bs->staged == 5 || bs->staged >= 9;
}

template <typename Real, int TPT, bool kBil, bool kWrite>
static void launch_spmm(dq_ctx* c, int j, const Real* rj, const Real* rjm, Real* w, int cy0, int ncy) {
    BatchedState* bs = c->bat;
    const BlockFmt& f = bs->fmt[r_index(bs->R)];
    const int n = c->n, B = bs->B, TC = bs->TC;
    const Real* cf = (const Real*)f.bcoef;
    const Real* d = (const Real*)bs->diag;
    if (bs->staged == 1) {
        const dim3 grid(bs->gxw, ncy);
        const CUtensorMap& tm = bs->tmaps[j];
#define DQ_WIN_R(RR)                                                                                       \
    k_spmm_win<Real, TPT, RR, kBil, kWrite><<<grid, kBThreads, bs->win_smem, c->stream>>>(                  \
        n, B, TC, bs->rpc_win, bs->halo, bs->wmask, j, f.bptr, f.bcol, cf, d, w, bs->s, cy0, bs->chunks, tm)
        switch (bs->R) {
            case 1: DQ_WIN_R(1); break;
            case 2: DQ_WIN_R(2); break;
            case 3: if constexpr (sizeof(Real) == 4) DQ_WIN_R(3); break;
            case 4: DQ_WIN_R(4); break;
            default: DQ_WIN_R(8); break;
        }
#undef DQ_WIN_R
        return;
    }
    if (bs->staged == 6 || bs->staged == 7) {
        if constexpr (sizeof(Real) == 4 && TPT == 2) {
            const dim3 grid(bs->f_gx, ncy);
            const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
            const CUtensorMap& tm = bs->tmaps[j];
#define DQ_RING_R(RR, LT)                                                                                          \
    k_spmm_ring<RR, kBil, kWrite, LT><<<grid, kRingThreads, bs->f_smem, c->stream>>>(                              \
        n, B, bs->f_rpc, bs->f_hb, bs->f_D, j, f.bptr, rec, d, w, bs->s, bs->chunks, tm)
            if (bs->staged == 7) {
                switch (bs->R) {
                    case 1: DQ_RING_R(1, 4); break;
                    case 2: DQ_RING_R(2, 4); break;
                    default: DQ_RING_R(3, 4); break;
                }
            } else {
                switch (bs->R) {
                    case 1: DQ_RING_R(1, 2); break;
                    case 2: DQ_RING_R(2, 2); break;
                    default: DQ_RING_R(3, 2); break;
                }
            }
#undef DQ_RING_R
        }
        return;
    }
    if (bs->staged == 9) {
        if constexpr (sizeof(Real) == 4 && TPT == 2) {
            const dim3 grid(bs->gxs, ncy);
            const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
            const size_t sm = cpa_smem_bytes();
#define DQ_CPA_R(RR)                                                                                          \
    k_spmm_cpa<RR, kBil, kWrite><<<grid, 512, sm, c->stream>>>(n, B, bs->bpc, f.nb, j, f.bptr, rec, d, rj, rjm, w, \
                                                               bs->s, bs->chunks)
            switch (bs->R) {
                case 1: DQ_CPA_R(1); break;
                case 2: DQ_CPA_R(2); break;
                default: DQ_CPA_R(3); break;
            }
#undef DQ_CPA_R
        }
        return;
    }
    if (bs->staged == 12) {
        if constexpr (sizeof(Real) == 4 && TPT == 2) {
            const dim3 grid(bs->gxs, ncy);
            const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
#define DQ_LEAN_R(RR, NT)                                                                                         \
    k_spmm_lean<RR, kBil, kWrite, NT><<<grid, NT, 0, c->stream>>>(n, B, TC, bs->bpc, f.nb, j, f.bptr, rec, d, rj, rjm, \
                                                                  w, bs->s, cy0, bs->chunks)
            if (bs->ctas_per_sm == 1) {
                switch (bs->R) {
                    case 1: DQ_LEAN_R(1, 1024); break;
                    case 2: DQ_LEAN_R(2, 1024); break;
                    default: DQ_LEAN_R(3, 1024); break;
                }
            } else {
                switch (bs->R) {
                    case 1: DQ_LEAN_R(1, 512); break;
                    case 2: DQ_LEAN_R(2, 512); break;
                    default: DQ_LEAN_R(3, 512); break;
                }
            }
#undef DQ_LEAN_R
        }
        return;
    }
    if (bs->staged == 10 || bs->staged == 11) {
        if constexpr (sizeof(Real) == 4 && TPT == 2) {
            const dim3 grid(bs->gxs, ncy);
            const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
#define DQ_WG_R(RR)                                                                                          \
    k_spmm_wg<RR, kBil, kWrite><<<grid, 512, 0, c->stream>>>(n, B, bs->bpc, f.nb, j, f.bptr, rec, d, rj, rjm, w, \
                                                             bs->s, cy0, bs->chunks)
            switch (bs->R) {
                case 1: DQ_WG_R(1); break;
                case 2: DQ_WG_R(2); break;
                default: DQ_WG_R(3); break;
            }
#undef DQ_WG_R
        }
        return;
    }
    if (bs->staged == 3) {
        if constexpr (sizeof(Real) == 4) {
            const dim3 grid(bs->gxs, ncy);
            const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
#define DQ_WARP_R(RR)                                                                                             \
    k_spmm_warp<TPT, RR, kBil, kWrite><<<grid, kBThreads, 0, c->stream>>>(n, B, bs->bpc, f.nb, j, f.bptr, rec, d, rj, w, \
                                                                      bs->s, cy0, bs->chunks)
            switch (bs->R) {
                case 1: DQ_WARP_R(1); break;
                case 2: DQ_WARP_R(2); break;
                default: DQ_WARP_R(3); break;
            }
#undef DQ_WARP_R
        }
        return;
    }
    const dim3 grid(bs->gxs, ncy);
    // staged = 5: the same L1 SpMM in 512-thread CTAs (one per SM, one
    // sliding gather window per SM instead of two competing ones)
#define DQ_SPMM_R(RR)                                                                                             \
    if (bs->staged == 5)                                                                                         \
        k_spmm_blk<Real, TPT, RR, kBil, kWrite, 512><<<grid, 512, 0, c->stream>>>(n, B, TC, bs->bpc, f.nb, j,     \
                                                                                 f.bptr, f.bcol, cf, d, rj, rjm, w, \
                                                                                 bs->s, cy0, bs->chunks);        \
    else                                                                                                         \
        k_spmm_blk<Real, TPT, RR, kBil, kWrite><<<grid, kBThreads, 0, c->stream>>>(n, B, TC, bs->bpc, f.nb, j,    \
                                                                                   f.bptr, f.bcol, cf, d, rj, rjm, w, \
                                                                                   bs->s, cy0, bs->chunks)
    switch (bs->R) {
        case 1: DQ_SPMM_R(1); break;
        case 2: DQ_SPMM_R(2); break;
        case 3: if constexpr (sizeof(Real) == 4) DQ_SPMM_R(3); break;
        case 4: DQ_SPMM_R(4); break;
        default: DQ_SPMM_R(8); break;
    }
#undef DQ_SPMM_R
}

// Fused iteration producing r_j (2 <= j <= m+1; j = m+1 is the last one,
// which also gives ||H q_{m+1}||).  w ping-pongs between slab 0 and wB:
// the SpMM of r_j writes wB for even j and slab 0 for odd j.
template <typename Real, int TPT, bool kBil, bool kLast>
static void launch_fused(dq_ctx* c, int j) {
    BatchedState* bs = c->bat;
    const BlockFmt& f = bs->fmt[r_index(bs->R)];
    const int n = c->n, B = bs->B, m = c->cfg.m;
    const size_t se = (size_t)n * B;
    Real* slabs = (Real*)bs->slabs;
    FusedMaps maps;
    maps.w = (j % 2 == 0) ? bs->fmaps[0] : bs->fmaps[m + 1];
    maps.r1 = bs->fmaps[j - 1];
    maps.r2 = bs->fmaps[j >= 3 ? j - 2 : j - 1];
    Real* r_out = slabs + 2 * se * j;
    Real* w_out = kLast ? nullptr : ((j % 2 == 0) ? (Real*)bs->wB : slabs);
    const dim3 grid(bs->f_gx, bs->chunks);
#define DQ_FUSED_R(RR)                                                                                           \
    k_lanczos_fused<Real, TPT, RR, kBil, kLast><<<grid, kBThreads, bs->f_smem, c->stream>>>(                      \
        n, B, bs->TC, bs->f_rpc, bs->f_hb, bs->f_D, j, j == 2, f.bptr, f.bcol, (const Real*)f.bcoef,             \
        (const Real*)bs->diag, r_out, w_out, bs->s, bs->chunks, maps)
    switch (bs->R) {
        case 1: DQ_FUSED_R(1); break;
        case 2: DQ_FUSED_R(2); break;
        case 3: if constexpr (sizeof(Real) == 4) DQ_FUSED_R(3); break;
        case 4: DQ_FUSED_R(4); break;
        default: DQ_FUSED_R(8); break;
    }
#undef DQ_FUSED_R
}

template <int TPT, bool kBil, bool kLast>
static void launch_fw(dq_ctx* c, int j) {
    BatchedState* bs = c->bat;
    const BlockFmt& f = bs->fmt[r_index(bs->R)];
    const int n = c->n, B = bs->B, m = c->cfg.m;
    const size_t se = (size_t)n * B;
    float* slabs = (float*)bs->slabs;
    FusedMaps maps;
    maps.w = (j % 2 == 0) ? bs->fmaps[0] : bs->fmaps[m + 1];
    maps.r1 = bs->fmaps[j - 1];
    maps.r2 = bs->fmaps[j >= 3 ? j - 2 : j - 1];
    float* r_out = slabs + 2 * se * j;
    float* w_out = kLast ? nullptr : ((j % 2 == 0) ? (float*)bs->wB : slabs);
    const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
    const dim3 grid(bs->f_gx, bs->chunks);
#define DQ_FW_R(RR)                                                                                               \
    k_lanczos_fw<TPT, RR, kBil, kLast><<<grid, kFwThreads, bs->f_smem, c->stream>>>(                               \
        n, B, bs->f_rpc, bs->f_hb, bs->f_D, bs->f_rb, j, j == 2, f.bptr, rec, (const float*)bs->diag, r_out, w_out, \
        bs->s, bs->chunks, maps)
    switch (bs->R) {
        case 1: DQ_FW_R(1); break;
        case 2: DQ_FW_R(2); break;
        default: DQ_FW_R(3); break;
    }
#undef DQ_FW_R
}

// One launch of the p-form iteration (staged = 8) for iteration j of m:
// j = 1 gathers psi (slab 1) and writes p_2; 2 <= j <= m gathers p_j, writes
// q_j and p_{j+1}; j = m + 1 writes q_{m+1} and ||H q_{m+1}||.  p_j lives in
// slab 0 for even j and in wB for odd j, so no launch reads the buffer it
// writes.
template <typename Real, int TPT, bool kBil, int kMode>
static void launch_pform_m(dq_ctx* c, int j) {
    BatchedState* bs = c->bat;
    const BlockFmt& f = bs->fmt[r_index(bs->R)];
    const int n = c->n, B = bs->B;
    const size_t se = (size_t)n * B;
    Real* slabs = (Real*)bs->slabs;
    auto slab = [&](int k) { return slabs + 2 * se * k; };
    auto pbuf = [&](int k) { return (k % 2 == 0) ? slabs : (Real*)bs->wB; };
    const Real* pin = kMode == 0 ? slab(1) : pbuf(j);
    const Real* qm1 = kMode == 0 ? nullptr : slab(j - 1);
    const Real* qm2 = (kMode != 0 && j >= 3) ? slab(j - 2) : nullptr;
    Real* qout = kMode == 0 ? nullptr : slab(j);
    Real* pout = kMode == 2 ? nullptr : pbuf(j + 1);
    const dim3 grid(bs->gxs, bs->chunks);
#define DQ_PF_R(RR)                                                                                               \
    k_lanczos_p<Real, TPT, RR, kBil, kMode, 512><<<grid, 512, 0, c->stream>>>(                                     \
        n, B, bs->TC, bs->bpc, f.nb, j, f.bptr, f.bcol, (const Real*)f.bcoef, (const Real*)bs->diag, pin, qm1, qm2, \
        qout, pout, bs->s, bs->chunks)
    switch (bs->R) {
        case 1: DQ_PF_R(1); break;
        case 2: DQ_PF_R(2); break;
        case 3: if constexpr (sizeof(Real) == 4) DQ_PF_R(3); break;
        case 4: DQ_PF_R(4); break;
        default: DQ_PF_R(8); break;
    }
#undef DQ_PF_R
}

template <typename Real, int TPT>
static void launch_pform(dq_ctx* c, int j) {
    const int m = c->cfg.m;
    const bool bil = c->cfg.dot_mode == DQ_DOT_BILINEAR;
    if (j == 1) {
        if (bil) launch_pform_m<Real, TPT, true, 0>(c, j);
        else launch_pform_m<Real, TPT, false, 0>(c, j);
    } else if (j <= m) {
        if (bil) launch_pform_m<Real, TPT, true, 1>(c, j);
        else launch_pform_m<Real, TPT, false, 1>(c, j);
    } else {
        if (bil) launch_pform_m<Real, TPT, true, 2>(c, j);
        else launch_pform_m<Real, TPT, false, 2>(c, j);
    }
}

template <typename Real, int TPT, bool kLast>
static void launch_fused_any(dq_ctx* c, int j) {
    if constexpr (sizeof(Real) == 4) {
        if (c->bat->staged == 4) {
            if (c->cfg.dot_mode == DQ_DOT_BILINEAR) launch_fw<TPT, true, kLast>(c, j);
            else launch_fw<TPT, false, kLast>(c, j);
            return;
        }
    }
    if (c->cfg.dot_mode == DQ_DOT_BILINEAR) launch_fused<Real, TPT, true, kLast>(c, j);
    else launch_fused<Real, TPT, false, kLast>(c, j);
}

// Iteration j of staged 11: the SpMM of k_spmm_wg and the axpy in one
// cooperative launch (every block resident, so the chunk barrier ends).
template <bool kBil>
static cudaError_t launch_iter_wg(dq_ctx* c, int j, const float* rj, const float* rjm, float* w, float* rjp, int cy0,
                                  int ncy) {
    BatchedState* bs = c->bat;
    const BlockFmt& f = bs->fmt[r_index(bs->R)];
    const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
    const float* d = (const float*)bs->diag;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(bs->gxs, ncy);
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const int n = c->n, B = bs->B, bpc = bs->bpc, nb = f.nb, nch = bs->chunks;
    const int* bptr = f.bptr;
    switch (bs->R) {
        case 1: return cudaLaunchKernelEx(&cfg, k_spmm_wg<1, kBil, true, true>, n, B, bpc, nb, j, bptr, rec, d, rj, rjm,
                                          w, bs->s, cy0, nch, rjp);
        case 2: return cudaLaunchKernelEx(&cfg, k_spmm_wg<2, kBil, true, true>, n, B, bpc, nb, j, bptr, rec, d, rj, rjm,
                                          w, bs->s, cy0, nch, rjp);
        default: return cudaLaunchKernelEx(&cfg, k_spmm_wg<3, kBil, true, true>, n, B, bpc, nb, j, bptr, rec, d, rj,
                                           rjm, w, bs->s, cy0, nch, rjp);
    }
}

template <typename Real, int TPT>
static dq_status enqueue_iteration(dq_ctx* c, int j, StepTimer* tm, int cy0, int ncy) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B, TC = bs->TC, rpc = bs->rpc;
    cudaStream_t st = c->stream;
    const size_t se = (size_t)n * B;
    Real* slabs = (Real*)bs->slabs;
    auto slab = [&](int k) { return slabs + 2 * se * k; };
    const dim3 grid(bs->gx, ncy);
    const bool fused = bs->staged == 2 || bs->staged == 4;
    if (bs->staged == 11) {
        if constexpr (sizeof(Real) == 4 && TPT == 2) {
            // SpMM (minus beta_{j-1} q_{j-1}) and axpy in one launch: r_{j+1} into slab j + 1
            if (tm) tm->mark(DQ_KIND_FUSED, st);
            const float* rjm = j > 1 ? slab(j - 1) : nullptr;
            const cudaError_t e = c->cfg.dot_mode == DQ_DOT_BILINEAR
                                      ? launch_iter_wg<true>(c, j, slab(j), rjm, slab(0), slab(j + 1), cy0, ncy)
                                      : launch_iter_wg<false>(c, j, slab(j), rjm, slab(0), slab(j + 1), cy0, ncy);
            if (e != cudaSuccess) return check_cuda(c, e, "cooperative iteration launch");
        }
        return DQ_OK;
    }
    if (bs->staged == 8) {
        // p-form: one launch per iteration, and the last one gives ||H q_{m+1}||
        if (tm) tm->mark(j == 1 ? DQ_KIND_SPMM : DQ_KIND_FUSED, st);
        launch_pform<Real, TPT>(c, j);
        if (j == c->cfg.m) {
            if (tm) tm->mark(DQ_KIND_SPMM_NORM, st);
            launch_pform<Real, TPT>(c, j + 1);
        }
        return DQ_OK;
    }
    if (fused && j >= 2) {
        // iteration j of the fused form produces r_j; the last one also r_{m+1}
        if (tm) tm->mark(DQ_KIND_FUSED, st);
        launch_fused_any<Real, TPT, false>(c, j);
        if (j == c->cfg.m) {
            if (tm) tm->mark(DQ_KIND_FUSED, st);
            launch_fused_any<Real, TPT, true>(c, j + 1);
        }
        return DQ_OK;
    }
    if (tm) tm->mark(DQ_KIND_SPMM, st);
    // the row-blocked L1 forms subtract beta_{j-1} q_{j-1} themselves
    const Real* rjm = (!fused && j > 1 && spmm_subtracts_prev(bs)) ? slab(j - 1) : nullptr;
    if (c->cfg.dot_mode == DQ_DOT_BILINEAR) launch_spmm<Real, TPT, true, true>(c, j, slab(j), rjm, slab(0), cy0, ncy);
    else launch_spmm<Real, TPT, false, true>(c, j, slab(j), rjm, slab(0), cy0, ncy);
    if (fused) {
        // fused form: the first SpMM only; r_2 comes from the next fused launch
        if (j == c->cfg.m) {
            if (tm) tm->mark(DQ_KIND_FUSED, st);
            launch_fused_any<Real, TPT, true>(c, j + 1);
        }
        return DQ_OK;
    }
    if (tm) tm->mark(DQ_KIND_AXPY, st);
    k_axpy_beta<Real, TPT><<<grid, kBThreads, 0, st>>>(n, B, TC, rpc, j, slab(0), slab(j),
                                                       rjm ? nullptr : slab(j - 1), slab(j + 1), bs->s, cy0,
                                                       bs->chunks);
    if (c->cfg.reorth) {
        if (tm) tm->mark(DQ_KIND_AXPY, st);
        // every h_k in one launch: about four CTAs per SM over (rows, chunks, blocks of k)
        const int nkb = (j + kReorthKB - 1) / kReorthKB;
        const int RPCr = kBThreads / TC;
        int gxr = std::max(1, (4 * bs->sms) / (ncy * nkb));
        // the partials of every (block of k, chunk, CTA) fit the two partial regions
        while (gxr > 1 && (size_t)nkb * gxr * 2 * kReorthKB * B > 2 * bs->partial_cap) --gxr;
        int rpcr = (n + gxr - 1) / gxr;
        rpcr = ((rpcr + 2 * RPCr - 1) / (2 * RPCr)) * (2 * RPCr);
        gxr = (n + rpcr - 1) / rpcr;
        k_reorth_dots_b<Real><<<dim3(gxr, ncy, nkb), kBThreads, 0, st>>>(
            n, B, TC, rpcr, j, slabs, se, bs->s, bs->s.tickets + kReorthTicket * (size_t)B, cy0, bs->chunks);
        k_reorth_apply_b<Real, TPT><<<grid, kBThreads, 0, st>>>(n, B, TC, rpc, j, slabs, se, bs->s, cy0, bs->chunks);
    }
    return DQ_OK;
}

static ZZParams zz_params(const dq_ctx* c) {
    ZZParams zz;
    if (c->cfg.noise_model == DQ_NOISE_ZZ) {
        zz.n_osc = c->zz_n_osc;
        zz.omega = c->d_zz_omega;
        zz.coeff = c->d_zz_coeff;
        zz.dt = c->cfg.dt;
    }
    return zz;
}

// Advances the device step counter when a recomputed step records nothing.
__global__ void k_advance_step(BatchedScalars S) {
    if (threadIdx.x == 0) *S.step = *S.step + 1;
}

template <typename Real, int TPT>
static dq_status enqueue_step(dq_ctx* c, StepTimer* tm, const std::function<void()>* after_noise = nullptr,
                              bool skip_pop = false) {
    BatchedState* bs = c->bat;
    auto mark = [&](int k) { if (tm) tm->mark(k, c->stream); };
    const int n = c->n, B = bs->B, m = c->cfg.m, TC = bs->TC, rpc = bs->rpc;
    cudaStream_t st = c->stream;
    const size_t se = (size_t)n * B;
    Real* slabs = (Real*)bs->slabs;
    auto slab = [&](int k) { return slabs + 2 * se * k; };
    const int ns = c->cfg.ka_substeps > 0 ? c->cfg.ka_substeps : 1;
    const double subdt = c->cfg.dt / (double)ns;
    const double sqrt_subdt = sqrt(subdt);
    const dim3 grid(bs->gx, bs->chunks);
    mark(DQ_KIND_NOISE);
    if (c->cfg.noise_model == DQ_NOISE_ZZ) {
        const long long pairs = (long long)n * ((B + 1) / 2);
        k_zz_block_b<<<(unsigned)((pairs + kZZThreads - 1) / kZZThreads), kZZThreads, 0, st>>>(
            n, B, c->traj0, c->cfg.seed, zz_params(c), bs->s, bs->zz_start, bs->zzD);
        k_zz_mark<<<1, 1, 0, st>>>(bs->s, bs->zz_start);
    }
    k_noise_b<Real, TPT><<<grid, kBThreads, 0, st>>>(n, B, c->traj0, TC, rpc, c->cfg.noise_model, ns, subdt, sqrt_subdt,
                                                     c->cfg.seed, c->d_sigma, c->d_invtau, c->d_coeff, bs->eps,
                                                     bs->deps, (Real*)bs->diag, bs->s, bs->zzD, bs->zz_start);
    if (after_noise) (*after_noise)();
    const bool adaptive = bs->s.mtraj != nullptr;
    if (adaptive) {
        // adaptive Krylov dimension: checks after iterations m_min, m_min + 4, ...;
        // chunks whose trajectories all chose skip their remaining iterations
        const int m_min = c->cfg.m_min;
        const double tol = c->cfg.m_tol > 0 ? c->cfg.m_tol : 1e-7;
        k_adapt_reset<<<(B + 255) / 256, 256, 0, st>>>(B, bs->chunks, m, bs->s);
        for (int j = 1; j <= m; ++j) {
            enqueue_iteration<Real, TPT>(c, j, tm, 0, bs->chunks);
            if (j >= m_min && j < m && (j - m_min) % kMCheckStride == 0) {
                mark(DQ_KIND_PADE);
                k_mcheck_b<<<B, 128, pade_smem_bytes(j + 2), st>>>(j, B, TC, c->tau_im, c->cfg.norm_mode, tol, bs->s);
                k_chunk_flags<<<bs->chunks, 64, 0, st>>>(TC, m, 0, bs->s);
            }
        }
        k_chunk_flags<<<bs->chunks, 64, 0, st>>>(TC, m, 1, bs->s);
    } else {
        // trajectory groups one after another: a group's Krylov slabs stay in
        // L2 across its m iterations
        const int cpg = bs->chunks / bs->groups;
        for (int g = 0; g < bs->groups; ++g) {
            for (int j = 1; j <= m; ++j) enqueue_iteration<Real, TPT>(c, j, tm, g * cpg, cpg);
            if (bs->staged != 2 && bs->staged != 4 && bs->staged != 8) {   // the fused forms' last launch gave ||H q_{m+1}||
                mark(DQ_KIND_SPMM_NORM);
                launch_spmm<Real, TPT, false, false>(c, m + 1, slab(m + 1), nullptr, nullptr, g * cpg, cpg);
            }
        }
    }
    mark(DQ_KIND_PADE);
    k_pade_b<<<B, 128, pade_smem_bytes(m + 2), st>>>(m, B, c->tau_im, c->cfg.norm_mode, bs->s, c->d_erracc);
    mark(DQ_KIND_COMBINE);
    k_combine_b<Real, TPT><<<grid, kBThreads, 0, st>>>(n, B, TC, rpc, m, slabs, se, corr_bra(c), bs->s);
    const int pblocks = std::max(1, std::min(bs->sms * 4, (n + 7) / 8));
    mark(DQ_KIND_POP);
    if (c->ipr_on && !skip_pop)
        k_ipr_b<Real><<<dim3(std::min(n, kIprRowGroups), (B + 127) / 128), 128, 0, st>>>(
            n, B, slab(1), bs->s, c->d_ipr_partial, c->d_ipr_ticket, c->d_ipr);
    if (skip_pop) k_advance_step<<<1, 32, 0, st>>>(bs->s);
    else
        k_pop_b<Real><<<pblocks, 256, 0, st>>>(n, B, c->cfg.pop_every, slab(1), c->d_pops, bs->s,
                                               bs->s.tickets + 8 * B);
    mark(-1);
    return check_cuda(c, cudaGetLastError(), "batched step launch");
}

static dq_status enqueue_step_any(dq_ctx* c, StepTimer* tm, const std::function<void()>* after_noise = nullptr,
                                  bool skip_pop = false) {
    BatchedState* bs = c->bat;
    if (!bs->mixed) return enqueue_step<double, 1>(c, tm, after_noise, skip_pop);
    return bs->TPT == 2 ? enqueue_step<float, 2>(c, tm, after_noise, skip_pop)
                        : enqueue_step<float, 1>(c, tm, after_noise, skip_pop);
}

// One ensemble step of c enqueued on c's stream (stream capture by a group).
dq_status batched_enqueue_step(dq_ctx* c) { return enqueue_step_any(c, nullptr); }

dq_status batched_step_eager(dq_ctx* c, const std::function<void()>* after_noise, bool skip_pop) {
    return enqueue_step_any(c, nullptr, after_noise, skip_pop);
}

static dq_status enqueue_iteration_any(dq_ctx* c, int j) {
    BatchedState* bs = c->bat;
    const int cpg = bs->chunks / bs->groups;
    for (int g = 0; g < bs->groups; ++g) {
        if (!bs->mixed) enqueue_iteration<double, 1>(c, j, nullptr, g * cpg, cpg);
        else if (bs->TPT == 2) enqueue_iteration<float, 2>(c, j, nullptr, g * cpg, cpg);
        else enqueue_iteration<float, 1>(c, j, nullptr, g * cpg, cpg);
    }
    return DQ_OK;
}

dq_status batched_iteration(dq_ctx* c, BatchedState* ws, int j) {
    BatchedState* saved = c->bat;
    c->bat = ws;
    dq_status st = enqueue_iteration_any(c, j);
    c->bat = saved;
    return st;
}

dq_status batched_run(dq_ctx* c, int n_steps) {
    BatchedState* bs = c->bat;
    if (n_steps == 0) return DQ_OK;
    if (!bs->exec) {
        DQ_CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        dq_status st = enqueue_step_any(c, nullptr);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (st) return st;
        DQ_CU(e);
        bs->graph = g;
        DQ_CU(cudaGraphInstantiate(&bs->exec, bs->graph, 0));
    }
    for (int k = 0; k < n_steps; ++k) DQ_CU(cudaGraphLaunch(bs->exec, c->stream));
    DQ_CU(cudaStreamSynchronize(c->stream));
    int status = 0;
    DQ_CU(cudaMemcpy(&status, bs->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    c->steps_done += n_steps;
    if (status) return read_status(c, status, "run");
    return DQ_OK;
}

// Device status word of the ensemble (after a synchronisation).
dq_status batched_read_status(dq_ctx* c) {
    int status = 0;
    DQ_CU(cudaMemcpy(&status, c->bat->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return read_status(c, status, "run");
    return DQ_OK;
}

dq_status batched_profile(dq_ctx* c, int n_steps, double* ms, int* cnt, int nk) {
    BatchedState* bs = c->bat;
    StepTimer tm;
    for (int k = 0; k < n_steps; ++k) {
        dq_status st = enqueue_step_any(c, &tm);
        if (st) return st;
        DQ_CU(cudaStreamSynchronize(c->stream));
        tm.collect(ms, cnt, nk);
    }
    int status = 0;
    DQ_CU(cudaMemcpy(&status, bs->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    c->steps_done += n_steps;
    if (status) return read_status(c, status, "profile");
    return DQ_OK;
}

// Mean device time of one Lanczos iteration (SpMM + axpy) under the current
// tiling: reps launches of iteration 1 between two events.
static void fused_iteration_any(dq_ctx* c, int j) {
    BatchedState* bs = c->bat;
    if (!bs->mixed) launch_fused_any<double, 1, false>(c, j);
    else if (bs->TPT == 2) launch_fused_any<float, 2, false>(c, j);
    else launch_fused_any<float, 1, false>(c, j);
}

// Device time of one Lanczos iteration: SpMM + axpy of iteration 1, or, in
// the fused form, one fused launch of iteration min(3, m) (after iterations
// 1 and 2 have filled its inputs).
dq_status batched_time_iteration(dq_ctx* c, int reps, double* ms) {
    cudaEvent_t e0, e1;
    DQ_CU(cudaEventCreate(&e0));
    DQ_CU(cudaEventCreate(&e1));
    const bool fused = c->bat->staged == 2 || c->bat->staged == 4;
    const bool pform = c->bat->staged == 8;
    const int jt = std::min(3, c->cfg.m);
    auto pf = [&](int j) {
        BatchedState* bs = c->bat;
        if (!bs->mixed) launch_pform<double, 1>(c, j);
        else if (bs->TPT == 2) launch_pform<float, 2>(c, j);
        else launch_pform<float, 1>(c, j);
    };
    // the standard forms are timed on iteration 2 (after one of iteration 1),
    // whose SpMM also streams q_{j-1} like every later one
    const int js = std::min(2, c->cfg.m);
    auto one = [&]() {
        if (fused) fused_iteration_any(c, jt);
        else if (pform) pf(jt);
        else enqueue_iteration_any(c, js);
    };
    if (!fused && !pform && js == 2) enqueue_iteration_any(c, 1);
    if (fused) {
        enqueue_iteration_any(c, 1);
        if (jt == 3) fused_iteration_any(c, 2);
    }
    if (pform) {
        pf(1);
        if (jt == 3) pf(2);
    }
    one();   // warm-up
    DQ_CU(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < reps; ++r) one();
    DQ_CU(cudaEventRecord(e1, c->stream));
    DQ_CU(cudaEventSynchronize(e1));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / reps;
    return check_cuda(c, cudaGetLastError(), "time iteration");
}

// Gather floor of the packed column-union form (complex64, R <= 3, 2
// trajectories per lane): the row-block walk, record stream and 16-byte
// gathers of k_spmm_blk in 512-thread CTAs over the same grid, with the
// coupling FMAs, the diagonal, q_{j-1}, alpha and all but one store per block
// left out.  Its time is what the gathers of this access pattern alone take
// on this GPU, the measured floor under the SpMM forms that gather through L1.
template <int R>
__global__ void __launch_bounds__(512, 1) k_gather_floor(int n, int B, int TC, int bpc, int nb,
                                                        const int* __restrict__ bptr, const float4* __restrict__ rec,
                                                        const float* __restrict__ x, float* __restrict__ out) {
    const int TPR = TC / 2;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    const int b0 = blockIdx.y * TC + tr * 2;
    const int k0 = blockIdx.x * bpc, k1 = min(nb, k0 + bpc);
    const float* src = x + 2 * (size_t)b0;
    for (int k = k0 + rl; k < k1; k += RPC) {
        const int pb = __ldg(bptr + k), pe = __ldg(bptr + k + 1);
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int e = pb; e < pe; e += 4) {   // a multiple of 4 records per block
            float4 r[4], y[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) r[u] = __ldg(rec + e + u);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                y[u] = __ldg(reinterpret_cast<const float4*>(src + 2 * (size_t)__float_as_int(r[u].x) * B));
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a.x += y[u].x; a.y += y[u].y; a.z += y[u].z; a.w += y[u].w;
            }
        }
        *reinterpret_cast<float4*>(out + 2 * ((size_t)min(k * R, n - 1) * B + b0)) = a;
    }
}

dq_status batched_time_gather_floor(dq_ctx* c, int reps, double* ms) {
    BatchedState* bs = c->bat;
    const BlockFmt& f = bs->fmt[r_index(bs->R)];
    if (!bs->mixed || bs->TPT != 2 || bs->R > 3 || !f.packed) {
        c->err = "gather floor: needs the complex64 packed form (vec 2, rows_per_block <= 3)";
        return DQ_ERR_STATE;
    }
    const size_t se = (size_t)c->n * bs->B;
    float* slabs = (float*)bs->slabs;
    const float4* rec = reinterpret_cast<const float4*>(f.bcoef);
    // one launch's chunks (with chunk groups, an SpMM launch covers one group)
    const dim3 grid(bs->gxs, bs->chunks / bs->groups);
    auto launch = [&]() {
        switch (bs->R) {
            case 1: k_gather_floor<1><<<grid, 512, 0, c->stream>>>(c->n, bs->B, bs->TC, bs->bpc, f.nb, f.bptr, rec, slabs + 2 * se, slabs); break;
            case 2: k_gather_floor<2><<<grid, 512, 0, c->stream>>>(c->n, bs->B, bs->TC, bs->bpc, f.nb, f.bptr, rec, slabs + 2 * se, slabs); break;
            default: k_gather_floor<3><<<grid, 512, 0, c->stream>>>(c->n, bs->B, bs->TC, bs->bpc, f.nb, f.bptr, rec, slabs + 2 * se, slabs); break;
        }
    };
    const int carve = cudaSharedmemCarveoutMaxL1;
    cudaFuncSetAttribute((const void*)k_gather_floor<1>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    cudaFuncSetAttribute((const void*)k_gather_floor<2>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    cudaFuncSetAttribute((const void*)k_gather_floor<3>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    cudaGetLastError();
    cudaEvent_t e0, e1;
    DQ_CU(cudaEventCreate(&e0));
    DQ_CU(cudaEventCreate(&e1));
    launch();   // warm-up
    DQ_CU(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < reps; ++r) launch();
    DQ_CU(cudaEventRecord(e1, c->stream));
    DQ_CU(cudaEventSynchronize(e1));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / reps;
    return check_cuda(c, cudaGetLastError(), "gather floor");
}

void batched_get_tiling(dq_ctx* c, int* tc, int* tpt, int* cps, int* R, int* staged, int* groups) {
    if (staged) *staged = c->bat->staged;
    if (groups) *groups = c->bat->groups;
    if (tc) *tc = c->bat->TC;
    if (tpt) *tpt = c->bat->TPT;
    if (cps) *cps = c->bat->ctas_per_sm;
    if (R) *R = c->bat->R;
}

dq_status batched_get_states(dq_ctx* c, dq_cdouble* out) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B;
    cd* tmp = nullptr;
    DQ_CU(cudaMalloc(&tmp, sizeof(cd) * (size_t)n * B));
    const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)n * B * 2 * real_sz;
    const int blocks = std::min(n, bs->sms * 8);
    const int thr = std::min(256, ((B + 31) / 32) * 32);
    if (bs->mixed)
        k_get_states_b<float><<<blocks, thr, 0, c->stream>>>(n, B, (const float*)((char*)bs->slabs + slab), bs->s, tmp);
    else
        k_get_states_b<double><<<blocks, thr, 0, c->stream>>>(n, B, (const double*)((char*)bs->slabs + slab), bs->s, tmp);
    cudaError_t e = cudaMemcpyAsync(out, tmp, sizeof(cd) * (size_t)n * B, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    return check_cuda(c, e, "get_states");
}

void batched_noise_arrays(dq_ctx* c, const double** eps, const double** deps) {
    *eps = c->bat->eps;
    *deps = c->bat->deps;
}

dq_status batched_collect_corr(dq_ctx* c) {
    BatchedState* bs = c->bat;
    const int np = c->steps_done + 1;
    k_corr_collect<<<std::max(1, std::min(bs->sms, (np + 255) / 256)), 256, 0, c->stream>>>(np, bs->chunks, bs->s.corr,
                                                                                              c->d_corr);
    return check_cuda(c, cudaGetLastError(), "corr collect");
}

// dq_debug_set_wait_cycles: the budget every bounded wait of this device reads
// (negative: the forced-timeout test mode of the ring SpMM)
dq_status batched_set_wait_cycles(dq_ctx* c, int cycles) {
    const long long v = cycles != 0 ? (long long)cycles : kWaitCycles;
    return check_cuda(c, cudaMemcpyToSymbol(g_dq_wait_cycles, &v, sizeof(v)), "wait budget");
}

}  // namespace dq
