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
//   w[site][traj]      : SpMM output of the current iteration
//   d[site][traj]      : this step's diagonal, real (float or double)
//   eps, deps          : FP64 static energies and OU offsets [site][traj]
// Per-trajectory FP64 scalars live in [j][traj] arrays.
//
// Grid: blockIdx.y picks a chunk of TC trajectories, blockIdx.x strides over
// rows; a thread owns TPT consecutive trajectories of one row at a time
// (16-byte vector loads).  Per-trajectory reductions (alpha, beta, norms,
// correlation) go through per-chunk partials and a per-chunk last-block
// ticket, so they are deterministic and need no extra launch.
//
// One time step (propagate.cu:199-259 for all trajectories at once):
//   k_noise_b, m x {k_spmm_alpha, k_axpy_beta}, k_spmm_norm, k_pade_b,
//   k_combine_b, k_pop_b
// captured once into a CUDA graph and replayed per step; the step index lives
// in device memory.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "dq_internal.h"
#include "dq_rng.cuh"

namespace dq {

template <typename Real> struct VecT;
template <> struct VecT<float> {
    static constexpr int TPT = 2;   // complex64 per thread: one float4
    using L = float4;
};
template <> struct VecT<double> {
    static constexpr int TPT = 1;   // complex128 per thread: one double2
    using L = double2;
};

template <typename Real>
struct CV {   // TPT complex values held in registers
    Real re[VecT<Real>::TPT], im[VecT<Real>::TPT];
};

template <typename Real>
__device__ __forceinline__ CV<Real> ldv(const Real* base, size_t idx2) {
    // idx2 = index in complex elements; base points at interleaved re/im
    CV<Real> v;
    typename VecT<Real>::L t = *reinterpret_cast<const typename VecT<Real>::L*>(base + 2 * idx2);
    if constexpr (VecT<Real>::TPT == 2) {
        v.re[0] = t.x; v.im[0] = t.y; v.re[1] = t.z; v.im[1] = t.w;
    } else {
        v.re[0] = t.x; v.im[0] = t.y;
    }
    return v;
}

template <typename Real>
__device__ __forceinline__ void stv(Real* base, size_t idx2, const CV<Real>& v) {
    typename VecT<Real>::L t;
    if constexpr (VecT<Real>::TPT == 2) {
        t.x = v.re[0]; t.y = v.im[0]; t.z = v.re[1]; t.w = v.im[1];
    } else {
        t.x = v.re[0]; t.y = v.im[0];
    }
    *reinterpret_cast<typename VecT<Real>::L*>(base + 2 * idx2) = t;
}

constexpr int kBThreads = 256;
constexpr int kMaxTC = 64;

struct BatchedScalars {
    // all [kMaxL][B] row-major by j, allocated separately (B is runtime)
    double* alpha;    // complex: 2 doubles per entry
    double* beta;
    double* sc;       // sc[j][b]
    double* yt;       // complex combine weights
    double* nav;      // [B]
    double* norm2;    // [B] ||psi||^2 of the stored (unnormalised) psi
    double* partial;  // [chunks][gx][TC][2]
    unsigned int* tickets;  // [8][chunks]
    int* status;      // [1]
    int* step;        // [1] current step index
    double* corr;     // [(max_steps+1)][chunks][2]
};

}  // namespace dq

struct dq::BatchedState {
    int B = 0, TC = 0, chunks = 0, gx = 0;
    bool mixed = true;
    void* slabs = nullptr;      // (m+2) slabs (slab 0 = w)
    void* diag = nullptr;       // Real [n][B]
    double* eps = nullptr;      // [n][B]
    double* deps = nullptr;     // [n][B]
    dq::BatchedScalars s{};
    double* scal_mem = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace dq {

// ---------------------------------------------------------------------------
// per-chunk reduction of TC complex partials per block
// ---------------------------------------------------------------------------
// acc[t] for this thread's TPT trajectories; threads with the same traj lane
// across the RPC row lanes are summed in shared memory, the block partial
// goes to partial[chunk][blockIdx.x][TC]; the last block of the chunk sums the
// gx partials in order.  Returns true in the last block; red_out[tcl] holds
// the chunk's totals (TC complex) in shared memory for threads < TC.
template <int TPT>
__device__ __forceinline__ bool chunk_reduce(const double (&ar)[TPT], const double (&ai)[TPT], int TC,
                                             double* partial, unsigned int* ticket, double2* red_out) {
    __shared__ double2 sm[kBThreads * 2];   // RPC * TC <= kBThreads * TPT
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
#pragma unroll
    for (int t = 0; t < TPT; ++t) sm[rl * TC + tr * TPT + t] = make_double2(ar[t], ai[t]);
    __syncthreads();
    const int chunk = blockIdx.y;
    double* mypart = partial + ((size_t)chunk * gridDim.x + blockIdx.x) * TC * 2;
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
        if (threadIdx.x < TC) {
            double sr = 0.0, si = 0.0;
            const double* base = partial + (size_t)chunk * gridDim.x * TC * 2;
            for (unsigned int g = 0; g < gridDim.x; ++g) {
                sr += __ldcg(&base[((size_t)g * TC + threadIdx.x) * 2]);
                si += __ldcg(&base[((size_t)g * TC + threadIdx.x) * 2 + 1]);
            }
            red_out[threadIdx.x] = make_double2(sr, si);
        }
        if (threadIdx.x == 0) ticket[chunk] = 0;
        __syncthreads();
    }
    return last;
}

// ---------------------------------------------------------------------------
__global__ void k_traj_init_b(int n, int B, uint64_t seed, const double* __restrict__ h0,
                              const double* __restrict__ static_eps, double sigma_static,
                              const double* __restrict__ sigma, int noise, double* __restrict__ eps,
                              double* __restrict__ deps) {
    size_t total = (size_t)n * B;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(x / B), b = (int)(x % B);
        double e;
        if (static_eps) e = static_eps[i];
        else e = __dadd_rn(__dmul_rn(sigma_static, normal(seed, P_STATIC, b, 0, i, 0)), h0[i]);
        eps[x] = e;
        deps[x] = (noise == DQ_NOISE_OU) ? __dmul_rn(sigma[i], normal(seed, P_OU_INIT, b, 0, i, 0)) : 0.0;
    }
}

template <typename Real>
__global__ void k_set_psi0_b(int n, int B, const cd* __restrict__ psi0, Real* __restrict__ r1) {
    size_t total = (size_t)n * B;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(x / B);
        r1[2 * x] = (Real)psi0[i].x;
        r1[2 * x + 1] = (Real)psi0[i].y;
    }
}

template <typename Real>
__global__ void k_noise_b(int n, int B, int noise, int ns, double subdt, double sqrt_subdt, uint64_t seed,
                          const double* __restrict__ sigma, const double* __restrict__ invtau,
                          const double* __restrict__ coeff, const double* __restrict__ eps,
                          double* __restrict__ deps, Real* __restrict__ d, BatchedScalars S) {
    const int step = *S.step;
    size_t total = (size_t)n * B;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(x / B), b = (int)(x % B);
        double v;
        if (noise == DQ_NOISE_OU) {
            double cur = ou_update(deps[x], invtau[i], coeff[i], subdt, sqrt_subdt, ns, seed, b, step, i);
            deps[x] = cur;
            v = __dadd_rn(cur, eps[x]);
        } else if (noise == DQ_NOISE_GAUSS) {
            double xi = normal(seed, P_GAUSS, b, step, i, 0);
            v = __dadd_rn(__dmul_rn(xi, sigma[i]), eps[x]);
        } else {
            v = eps[x];
        }
        d[x] = (Real)v;
    }
}

// w = H q_j for all trajectories; alpha_j[b] = <q_j, w>_b
template <typename Real, bool kBilinear, bool kWrite>
__global__ void __launch_bounds__(kBThreads) k_spmm(int n, int B, int TC, int j, const int* __restrict__ rowptr,
                                                   const int* __restrict__ col, const Real* __restrict__ val,
                                                   const Real* __restrict__ d, const Real* __restrict__ rj,
                                                   Real* __restrict__ w, BatchedScalars S) {
    constexpr int TPT = VecT<Real>::TPT;
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    const int b0 = blockIdx.y * TC + tr * TPT;
    double sc[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) sc[t] = S.sc[(size_t)j * B + b0 + t];
    double ar[TPT], ai[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { ar[t] = 0.0; ai[t] = 0.0; }
    for (int row = blockIdx.x * RPC + rl; row < n; row += gridDim.x * RPC) {
        const size_t base = (size_t)row * B + b0;
        CV<Real> x = ldv(rj, base);
        CV<Real> u;
        {
            const Real* dp = d + base;
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                Real dd = dp[t];
                u.re[t] = dd * x.re[t];
                u.im[t] = dd * x.im[t];
            }
        }
        const int p1 = rowptr[row + 1];
        for (int p = rowptr[row]; p < p1; ++p) {
            const int c = __ldg(col + p);
            const Real v = __ldg(val + p);
            CV<Real> y = ldv(rj, (size_t)c * B + b0);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                u.re[t] = fma(v, y.re[t], u.re[t]);
                u.im[t] = fma(v, y.im[t], u.im[t]);
            }
        }
        if (kWrite) {
            CV<Real> o;
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                o.re[t] = (Real)(sc[t] * (double)u.re[t]);
                o.im[t] = (Real)(sc[t] * (double)u.im[t]);
            }
            stv(w, base, o);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                // alpha partial of the unscaled product; sc^2 applied at the end
                double xr = x.re[t], xi = x.im[t], ur = u.re[t], ui = u.im[t];
                if (kBilinear) { ar[t] += xr * ur - xi * ui; ai[t] += xr * ui + xi * ur; }
                else { ar[t] += xr * ur + xi * ui; ai[t] += xr * ui - xi * ur; }
            }
        } else {
#pragma unroll
            for (int t = 0; t < TPT; ++t) ar[t] += (double)u.re[t] * u.re[t] + (double)u.im[t] * u.im[t];
        }
    }
    __shared__ double2 red[kMaxTC];
    if (chunk_reduce<TPT>(ar, ai, TC, S.partial, S.tickets + (kWrite ? 0 : 2) * gridDim.y, red)) {
        if (threadIdx.x < TC) {
            const int b = blockIdx.y * TC + threadIdx.x;
            const double s = S.sc[(size_t)j * B + b];
            double2 v = red[threadIdx.x];
            if (kWrite) {
                S.alpha[2 * ((size_t)j * B + b)] = v.x * s * s;
                S.alpha[2 * ((size_t)j * B + b) + 1] = v.y * s * s;
            } else {
                S.nav[b] = sqrt(v.x) * s;
            }
        }
    }
}

// r_{j+1} = w - alpha_j q_j - beta_{j-1} q_{j-1}; beta_j = ||r_{j+1}||
template <typename Real>
__global__ void __launch_bounds__(kBThreads) k_axpy_beta(int n, int B, int TC, int j, const Real* __restrict__ w,
                                                        const Real* __restrict__ rj, const Real* __restrict__ rjm,
                                                        Real* __restrict__ rjp, BatchedScalars S) {
    constexpr int TPT = VecT<Real>::TPT;
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    const int b0 = blockIdx.y * TC + tr * TPT;
    double ajr[TPT], aji[TPT], sj[TPT], bm[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        const size_t k = (size_t)j * B + b0 + t;
        ajr[t] = S.alpha[2 * k] * S.sc[k];
        aji[t] = S.alpha[2 * k + 1] * S.sc[k];
        sj[t] = S.sc[k];
        bm[t] = (j > 1) ? S.beta[(size_t)(j - 1) * B + b0 + t] * S.sc[(size_t)(j - 1) * B + b0 + t] : 0.0;
    }
    double nn[TPT], dummy[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { nn[t] = 0.0; dummy[t] = 0.0; }
    for (int row = blockIdx.x * RPC + rl; row < n; row += gridDim.x * RPC) {
        const size_t base = (size_t)row * B + b0;
        CV<Real> u = ldv(w, base);
        CV<Real> x = ldv(rj, base);
        CV<Real> xm;
        if (j > 1) xm = ldv(rjm, base);
        CV<Real> o;
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            // alpha * (sc_j r_j): (ajr + i aji) (xr + i xi)
            double xr = x.re[t], xi = x.im[t];
            double rr = (double)u.re[t] - (ajr[t] * xr - aji[t] * xi);
            double ri = (double)u.im[t] - (ajr[t] * xi + aji[t] * xr);
            if (j > 1) {
                rr -= bm[t] * (double)xm.re[t];
                ri -= bm[t] * (double)xm.im[t];
            }
            o.re[t] = (Real)rr;
            o.im[t] = (Real)ri;
            nn[t] += (double)o.re[t] * o.re[t] + (double)o.im[t] * o.im[t];
        }
        stv(rjp, base, o);
    }
    (void)sj;
    __shared__ double2 red[kMaxTC];
    if (chunk_reduce<TPT>(nn, dummy, TC, S.partial, S.tickets + 1 * gridDim.y, red)) {
        if (threadIdx.x < TC) {
            const int b = blockIdx.y * TC + threadIdx.x;
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

// one CTA per trajectory: exp(tau Tbar), combine weights, error estimate
__global__ void k_pade_b(int m, int B, double tau_im, int norm_mode, BatchedScalars S, double* erracc) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ cd al[kMaxL], be[kMaxL], y[kMaxM];
    const int b = blockIdx.x;
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
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
        const size_t k = (size_t)(j + 1) * B + b;
        cd v = cscale(y[j], S.sc[k]);
        S.yt[2 * k] = v.x;
        S.yt[2 * k + 1] = v.y;
    }
    if (threadIdx.x == 0) {
        double est = expokit_error(be[m].x, S.nav[b], o.e_m1_m, o.e_m1_mp1);
        erracc[b] += est;
    }
}

// psi = sum_j yt_j r_j written over slab 1; ||psi||^2 and <psi0|psi> per
// trajectory; correlation point step+1 per chunk.
template <typename Real>
__global__ void __launch_bounds__(kBThreads) k_combine_b(int n, int B, int TC, int m, Real* __restrict__ slabs,
                                                        size_t slab_stride, const cd* __restrict__ psi0,
                                                        BatchedScalars S) {
    constexpr int TPT = VecT<Real>::TPT;
    const int TPR = TC / TPT;
    const int tr = threadIdx.x % TPR, rl = threadIdx.x / TPR;
    const int RPC = blockDim.x / TPR;
    const int b0 = blockIdx.y * TC + tr * TPT;
    const int step = *S.step;
    double nn[TPT], cr[TPT], ci[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) { nn[t] = 0.0; cr[t] = 0.0; ci[t] = 0.0; }
    Real* r1 = slabs + 2 * slab_stride;   // slab 1
    for (int row = blockIdx.x * RPC + rl; row < n; row += gridDim.x * RPC) {
        const size_t base = (size_t)row * B + b0;
        double accr[TPT], acci[TPT];
#pragma unroll
        for (int t = 0; t < TPT; ++t) { accr[t] = 0.0; acci[t] = 0.0; }
        for (int j = 1; j <= m; ++j) {
            CV<Real> x = ldv(slabs + 2 * slab_stride * j, base);
#pragma unroll
            for (int t = 0; t < TPT; ++t) {
                const size_t k = (size_t)j * B + b0 + t;
                const double yr = S.yt[2 * k], yi = S.yt[2 * k + 1];
                accr[t] += yr * x.re[t] - yi * x.im[t];
                acci[t] += yr * x.im[t] + yi * x.re[t];
            }
        }
        CV<Real> o;
        const cd p0 = psi0[row];
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
            o.re[t] = (Real)accr[t];
            o.im[t] = (Real)acci[t];
            const double vr = o.re[t], vi = o.im[t];
            nn[t] += vr * vr + vi * vi;
            cr[t] += p0.x * vr + p0.y * vi;   // conj(psi0) * psi
            ci[t] += p0.x * vi - p0.y * vr;
        }
        stv(r1, base, o);
    }
    __shared__ double2 red[kMaxTC];
    // norms
    double zero[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) zero[t] = 0.0;
    if (chunk_reduce<TPT>(nn, zero, TC, S.partial, S.tickets + 3 * gridDim.y, red)) {
        if (threadIdx.x < TC) {
            const int b = blockIdx.y * TC + threadIdx.x;
            double n2 = red[threadIdx.x].x;
            S.norm2[b] = n2;
            double s1 = 1.0 / sqrt(n2);
            S.sc[B + b] = s1;   // sc[1][b]: next step's q_1 = psi / ||psi||
            if (!(n2 > 0.0) || !isfinite(n2)) atomicCAS(S.status, 0, DQ_ERR_NAN);
        }
    }
    __syncthreads();
    // correlation, normalised per trajectory by this step's ||psi||: the
    // norms are final once the norm reduction above has completed in every
    // block; the correlation therefore uses a second partial pass whose last
    // block divides by the norms (published by then through the ticket order)
    double* part2 = S.partial + (size_t)gridDim.y * gridDim.x * TC * 2;
    if (chunk_reduce<TPT>(cr, ci, TC, part2, S.tickets + 4 * gridDim.y, red)) {
        if (threadIdx.x == 0) {
            double sr = 0.0, si = 0.0;
            for (int t = 0; t < TC; ++t) {
                const int b = blockIdx.y * TC + t;
                const double s1 = 1.0 / sqrt(__ldcg(&S.norm2[b]));
                sr += red[t].x * s1;
                si += red[t].y * s1;
            }
            double* cp = S.corr + ((size_t)(step + 1) * gridDim.y + blockIdx.y) * 2;
            cp[0] = sr;
            cp[1] = si;
        }
    }
}

// populations: one warp per row, all trajectories, fixed order; advances the
// step counter in its last block.
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

// initial record: pops[0] += B |psi0|^2, corr[0] = B <psi0|psi0>, norms
__global__ void k_init_obs_b(int n, int B, const cd* __restrict__ psi0, double* pops, BatchedScalars S,
                             int chunks) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        pops[i] += (double)B * cabs2(psi0[i]);
    if (blockIdx.x == 0) {
        __shared__ double scratch[32];
        double s = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) s += cabs2(psi0[i]);
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) {
            for (int ch = 0; ch < chunks; ++ch) {
                S.corr[2 * ch] = (ch == 0) ? (double)B * s : 0.0;
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
    size_t total = (size_t)n * B;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(x / B), b = (int)(x % B);
        double s = 1.0 / sqrt(S.norm2[b]);
        out[(size_t)b * n + i] = cmk(r1[2 * x] * s, r1[2 * x + 1] * s);
    }
}

// ---------------------------------------------------------------------------
#define DQ_CU(call)                                                     \
    do {                                                                \
        dq_status _s = check_cuda(c, (call), #call);                    \
        if (_s != DQ_OK) return _s;                                     \
    } while (0)

static int pick_tc(int B, int tpt) {
    for (int tc = kMaxTC; tc >= tpt; tc >>= 1)
        if (B % tc == 0 && tc / tpt <= kBThreads) return tc;
    return 0;
}

dq_status batched_alloc(dq_ctx* c) {
    const int n = c->n, B = c->cfg.n_traj, m = c->cfg.m;
    BatchedState* bs = new BatchedState();
    c->bat = bs;
    bs->B = B;
    bs->mixed = c->cfg.precision == DQ_PREC_MIXED;
    const int tpt = bs->mixed ? VecT<float>::TPT : VecT<double>::TPT;
    bs->TC = pick_tc(B, tpt);
    if (!bs->TC) {
        c->err = "batched: n_traj must be a multiple of 2 for the mixed path";
        return DQ_ERR_ARG;
    }
    bs->chunks = B / bs->TC;
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->cfg.device);
    const int TPR = bs->TC / tpt, RPC = kBThreads / TPR;
    int gx = std::max(1, (dev_sms * 4) / bs->chunks);
    gx = std::min(gx, (n + RPC - 1) / RPC);
    bs->gx = gx;
    const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)n * B * 2 * real_sz;
    DQ_CU(cudaMalloc(&bs->slabs, slab * (m + 2)));
    DQ_CU(cudaMemsetAsync(bs->slabs, 0, slab * (m + 2), c->stream));
    DQ_CU(cudaMalloc(&bs->diag, (size_t)n * B * real_sz));
    DQ_CU(cudaMalloc(&bs->eps, sizeof(double) * (size_t)n * B));
    DQ_CU(cudaMalloc(&bs->deps, sizeof(double) * (size_t)n * B));
    // scalars
    const size_t LB = (size_t)kMaxL * B;
    const size_t partial_n = (size_t)bs->chunks * gx * bs->TC * 2 * 2;
    const size_t corr_n = (size_t)(c->cfg.max_steps + 1) * bs->chunks * 2;
    const size_t total = LB * 2 /*alpha*/ + LB /*beta*/ + LB /*sc*/ + LB * 2 /*yt*/ + B + B + partial_n + corr_n;
    DQ_CU(cudaMalloc(&bs->scal_mem, sizeof(double) * total));
    DQ_CU(cudaMemsetAsync(bs->scal_mem, 0, sizeof(double) * total, c->stream));
    double* p = bs->scal_mem;
    bs->s.alpha = p; p += LB * 2;
    bs->s.beta = p; p += LB;
    bs->s.sc = p; p += LB;
    bs->s.yt = p; p += LB * 2;
    bs->s.nav = p; p += B;
    bs->s.norm2 = p; p += B;
    bs->s.partial = p; p += partial_n;
    bs->s.corr = p; p += corr_n;
    DQ_CU(cudaMalloc(&bs->s.tickets, sizeof(unsigned int) * 8 * bs->chunks + sizeof(unsigned int) * 8));
    DQ_CU(cudaMemsetAsync(bs->s.tickets, 0, sizeof(unsigned int) * 8 * bs->chunks + sizeof(unsigned int) * 8, c->stream));
    DQ_CU(cudaMalloc(&bs->s.status, sizeof(int) * 2));
    bs->s.step = bs->s.status + 1;
    DQ_CU(cudaMemsetAsync(bs->s.status, 0, sizeof(int) * 2, c->stream));
    DQ_CU(cudaFuncSetAttribute(k_pade_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pade_smem_bytes(m + 2)));
    return DQ_OK;
}

void batched_free(dq_ctx* c) {
    BatchedState* bs = c->bat;
    if (!bs) return;
    if (bs->exec) cudaGraphExecDestroy(bs->exec);
    if (bs->graph) cudaGraphDestroy(bs->graph);
    cudaFree(bs->slabs); cudaFree(bs->diag); cudaFree(bs->eps); cudaFree(bs->deps);
    cudaFree(bs->scal_mem); cudaFree(bs->s.tickets); cudaFree(bs->s.status);
    delete bs;
    c->bat = nullptr;
}

dq_status batched_reset(dq_ctx* c) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B;
    size_t total = (size_t)n * B;
    int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    k_traj_init_b<<<blocks, 256, 0, c->stream>>>(n, B, c->cfg.seed, c->d_h0, c->d_static, c->cfg.sigma_static,
                                                 c->d_sigma, c->cfg.noise_model, bs->eps, bs->deps);
    const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)n * B * 2 * real_sz;
    if (bs->mixed)
        k_set_psi0_b<float><<<blocks, 256, 0, c->stream>>>(n, B, c->d_psi0, (float*)((char*)bs->slabs + slab));
    else
        k_set_psi0_b<double><<<blocks, 256, 0, c->stream>>>(n, B, c->d_psi0, (double*)((char*)bs->slabs + slab));
    k_set_norms_b<<<1, 256, 0, c->stream>>>(n, B, c->d_psi0, bs->s);
    k_init_obs_b<<<std::max(1, std::min(148, (n + 255) / 256)), 256, 0, c->stream>>>(n, B, c->d_psi0, c->d_pops,
                                                                                     bs->s, bs->chunks);
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

template <typename Real>
static dq_status enqueue_step(dq_ctx* c, StepTimer* tm = nullptr) {
    BatchedState* bs = c->bat;
    auto mark = [&](int k) { if (tm) tm->mark(k, c->stream); };
    const int n = c->n, B = bs->B, m = c->cfg.m, TC = bs->TC;
    cudaStream_t st = c->stream;
    const size_t slab_elems = (size_t)n * B;   // complex elements per slab
    Real* slabs = (Real*)bs->slabs;
    auto slab = [&](int j) { return slabs + 2 * slab_elems * j; };
    Real* w = slab(0);
    const int ns = c->cfg.ka_substeps > 0 ? c->cfg.ka_substeps : 1;
    const double subdt = c->cfg.dt / (double)ns;
    const double sqrt_subdt = sqrt(subdt);
    size_t total = (size_t)n * B;
    int nblocks = (int)std::min<size_t>((total + 255) / 256, 148 * 8);
    mark(DQ_KIND_NOISE);
    k_noise_b<Real><<<nblocks, 256, 0, st>>>(n, B, c->cfg.noise_model, ns, subdt, sqrt_subdt, c->cfg.seed, c->d_sigma,
                                             c->d_invtau, c->d_coeff, bs->eps, bs->deps, (Real*)bs->diag, bs->s);
    const Real* val = bs->mixed ? (const Real*)c->d_valf : (const Real*)c->d_val;
    dim3 grid(bs->gx, bs->chunks);
    const bool bil = c->cfg.dot_mode == DQ_DOT_BILINEAR;
    for (int j = 1; j <= m; ++j) {
        mark(DQ_KIND_SPMM);
        if (bil)
            k_spmm<Real, true, true><<<grid, kBThreads, 0, st>>>(n, B, TC, j, c->d_rowptr, c->d_col, val,
                                                                 (const Real*)bs->diag, slab(j), w, bs->s);
        else
            k_spmm<Real, false, true><<<grid, kBThreads, 0, st>>>(n, B, TC, j, c->d_rowptr, c->d_col, val,
                                                                  (const Real*)bs->diag, slab(j), w, bs->s);
        mark(DQ_KIND_AXPY);
        k_axpy_beta<Real><<<grid, kBThreads, 0, st>>>(n, B, TC, j, w, slab(j), slab(j - 1), slab(j + 1), bs->s);
    }
    mark(DQ_KIND_SPMM_NORM);
    k_spmm<Real, false, false><<<grid, kBThreads, 0, st>>>(n, B, TC, m + 1, c->d_rowptr, c->d_col, val,
                                                           (const Real*)bs->diag, slab(m + 1), nullptr, bs->s);
    mark(DQ_KIND_PADE);
    k_pade_b<<<B, 128, pade_smem_bytes(m + 2), st>>>(m, B, c->tau_im, c->cfg.norm_mode, bs->s, c->d_erracc);
    mark(DQ_KIND_COMBINE);
    k_combine_b<Real><<<grid, kBThreads, 0, st>>>(n, B, TC, m, slabs, slab_elems, c->d_psi0, bs->s);
    int pblocks = std::max(1, std::min(148 * 4, (n + 7) / 8));
    mark(DQ_KIND_POP);
    k_pop_b<Real><<<pblocks, 256, 0, st>>>(n, B, c->cfg.pop_every, slab(1), c->d_pops, bs->s,
                                           bs->s.tickets + 8 * bs->chunks);
    mark(-1);
    return check_cuda(c, cudaGetLastError(), "batched step launch");
}

dq_status batched_run(dq_ctx* c, int n_steps) {
    BatchedState* bs = c->bat;
    if (n_steps == 0) return DQ_OK;
    if (!bs->exec) {
        DQ_CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        dq_status st = bs->mixed ? enqueue_step<float>(c) : enqueue_step<double>(c);
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

dq_status batched_profile(dq_ctx* c, int n_steps, double* ms, int* cnt, int nk) {
    BatchedState* bs = c->bat;
    StepTimer tm;
    for (int k = 0; k < n_steps; ++k) {
        dq_status st = bs->mixed ? enqueue_step<float>(c, &tm) : enqueue_step<double>(c, &tm);
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

dq_status batched_get_states(dq_ctx* c, dq_cdouble* out) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B;
    cd* tmp = nullptr;
    DQ_CU(cudaMalloc(&tmp, sizeof(cd) * (size_t)n * B));
    const size_t real_sz = bs->mixed ? sizeof(float) : sizeof(double);
    const size_t slab = (size_t)n * B * 2 * real_sz;
    int blocks = (int)std::min<size_t>(((size_t)n * B + 255) / 256, 148 * 16);
    if (bs->mixed)
        k_get_states_b<float><<<blocks, 256, 0, c->stream>>>(n, B, (const float*)((char*)bs->slabs + slab), bs->s, tmp);
    else
        k_get_states_b<double><<<blocks, 256, 0, c->stream>>>(n, B, (const double*)((char*)bs->slabs + slab), bs->s, tmp);
    cudaError_t e = cudaMemcpyAsync(out, tmp, sizeof(cd) * (size_t)n * B, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    return check_cuda(c, e, "get_states");
}

void batched_noise_arrays(dq_ctx* c, const double** eps, const double** deps) {
    *eps = c->bat->eps;
    *deps = c->bat->deps;
}

// correlation sums over chunks -> d_corr (called by the getter)
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

dq_status batched_collect_corr(dq_ctx* c) {
    BatchedState* bs = c->bat;
    const int np = c->steps_done + 1;
    k_corr_collect<<<std::max(1, std::min(148, (np + 255) / 256)), 256, 0, c->stream>>>(np, bs->chunks, bs->s.corr,
                                                                                          c->d_corr);
    return check_cuda(c, cudaGetLastError(), "corr collect");
}

}  // namespace dq
