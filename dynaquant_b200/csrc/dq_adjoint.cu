// dq_adjoint.cu — gradient of a spectrum-fitting loss by the adjoint method.
//
// No counterpart in the reference (it computes no gradients).  Forward: the
// ensemble step of dq_batched.cu, unchanged.  The states at segment starts
// are kept; each segment is recomputed before its backward pass, and its
// steps' Krylov bases (psi(t), r_2..r_{m+1}), Lanczos scalars and diagonals
// stay resident in HBM while it is processed (the last segment's are kept by
// the forward pass itself), so the backward pass never repeats the forward
// Lanczos.  Backward, per step t from the last one down, for every
// trajectory at once:
//
//   V, T_V  = the forward step's basis and tridiagonal (kept)
//   W, T_W  = Lanczos(H_t, lambda(t+1)/|lambda|)
//   E       = exp([[tau T_W, e1 e1^T], [0, tau T_V]])          (2m x 2m)
//   N       = E[0:m, m:2m]    (Fréchet derivative of the exponential,
//                              C. Van Loan, IEEE TAC 23 (1978) 395)
//   dL/deps_i   += Re tau |lambda| sum_ab conj(W_ia) N_ab V_ib
//   dL/dcoupl   += the same form with (H_off V)_ib, H_off V from the
//                  Lanczos three-term relation (no extra SpMM)
//   lambda(t)    = s_t + |lambda| W conj(E[0:m, 0])       (exp(-tau H) = conj)
//
// with tau = -i dt/hbar, s_t = conj(G_t)/B psi0 and G the inverse DFT of the
// loss derivative with respect to the spectrum.  The adjoint of the
// renormalisation vanishes to first order (the step is unitary), so it is
// not differentiated.  The host FP64 restatement of the same recursion is
// the oracle's dqo_spectrum_loss_grad, checked against finite differences.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "dq_batched.cuh"

namespace dq {

constexpr int kAdjMaxM = 24;      // the 2m x 2m exponential fits one CTA's shared memory
constexpr int kAdjTraj = 8;       // trajectories per CTA of the gradient kernel
constexpr int kAdjThreads = 256;  // 32 row lanes x 8 trajectory lanes
constexpr int kAdjMaxClasses = 8; // coupling classes with a gradient of their own

// alpha (2 LB), beta (LB) and sc (LB) of one step, LB = kMaxL * B: the
// contiguous head of a workspace's scalar block
inline size_t scal_block(int B) { return (size_t)4 * kMaxL * B; }

template <typename Real> struct R2;
template <> struct R2<float> { using T = float2; };
template <> struct R2<double> { using T = double2; };

struct AdjointState {
    int T = 0, len = 0, K = 0, n_seg = 0;
    double scale = 0.0;
    double inv_norm = 0.0;   // 1 / trajectories of the ensemble mean (all shards)
    bool forward_done = false;
    size_t slab_bytes = 0, diag_bytes = 0;
    double* d_target = nullptr;
    cd* d_spec = nullptr;
    cd* d_g = nullptr;
    cd* d_G = nullptr;
    double* d_loss = nullptr;
    // segment slots: (m+1) slabs each (psi(t) as slab 1 held it, then
    // r_2..r_{m+1}), the step's alpha/beta/sc block and its diagonal
    unsigned char* seg_V = nullptr;
    double* seg_sc = nullptr;            // K x kScalBlock(B)
    unsigned char* seg_diag = nullptr;   // K diagonals
    // a second set of segment slots: while the backward sweep reads one set,
    // the next segment is recomputed into the other on a second stream
    // (absent when the memory is short; the sweep then waits for each recompute)
    unsigned char* seg_V2 = nullptr;
    double* seg_sc2 = nullptr;
    unsigned char* seg_diag2 = nullptr;
    cudaStream_t rstream = nullptr;
    cudaEvent_t ev_go = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_sweep[2] = {nullptr, nullptr};
    int cur_set = 0;
    unsigned char* ck_psi = nullptr;     // states at the starts of segments 0..n_seg-2
    double* ck_n2 = nullptr;
    double* ck_deps = nullptr;           // OU offsets at those starts
    BatchedState* ws2 = nullptr;         // the lambda Lanczos workspace
    void* d_coef = nullptr;              // B x CS complex coefficients
    double* d_lpart = nullptr;           // row CTAs x B
    double* d_gsite = nullptr;           // n x (B / kAdjTraj)
    double* d_gcpl = nullptr;
    double* d_gout = nullptr;            // n + final partials
    double* d_erracc_save = nullptr;
    int row_ctas = 0, rows_per_cta = 0, fin_blocks = 0;
    // more than one coupling class: per-entry class and base value, and the
    // per-(site, trajectory group, class) accumulators of the gather kernel
    int n_cls = 0;
    int* d_cls = nullptr;
    double* d_vbase = nullptr;
    double* d_gcls = nullptr;            // n x G x n_cls
    double* d_gcls_out = nullptr;        // fin_blocks x n_cls
};

// ---------------------------------------------------------------------------
__global__ void k_adj_loss(int len, double scale, const double* __restrict__ target, const cd* __restrict__ spec,
                           cd* __restrict__ g, double* __restrict__ loss) {
    __shared__ double scratch[32];
    double acc = 0.0;
    for (int j = threadIdx.x; j < len; j += blockDim.x) {
        const double a = scale * spec[j].x - target[j];
        acc += a * a;
        g[j] = cmk(2.0 * scale * a, 0.0);
    }
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) *loss = acc;
}

__global__ void k_set_step(BatchedScalars S, int v) {
    if (threadIdx.x == 0) *S.step = v;
}

__global__ void k_set_sc1(int B, BatchedScalars S) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
        const double n2 = S.norm2[b];
        S.sc[B + b] = n2 > 0.0 ? 1.0 / sqrt(n2) : 0.0;
    }
}

// lambda(T) = conj(G_T)/B psi0 in every trajectory, and its norm
template <typename Real>
__global__ void k_lambda_init(int n, int B, const cd* __restrict__ psi0, const cd* __restrict__ Gt, double invB,
                              Real* __restrict__ w1) {
    const cd g = Gt[0];
    const double sr = g.x * invB, si = -g.y * invB;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const cd p = psi0[i];
        const Real lr = (Real)(sr * p.x - si * p.y), li = (Real)(sr * p.y + si * p.x);
        for (int b = threadIdx.x; b < B; b += blockDim.x) {
            const size_t x = (size_t)i * B + b;
            w1[2 * x] = lr;
            w1[2 * x + 1] = li;
        }
    }
}

template <typename Real>
__global__ void k_lambda_init_norm(int n, int B, const cd* __restrict__ psi0, const cd* __restrict__ Gt,
                                   double invB, BatchedScalars S) {
    __shared__ double scratch[32];
    const cd g = Gt[0];
    const double sr = g.x * invB, si = -g.y * invB;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const cd p = psi0[i];
        const double lr = (Real)(sr * p.x - si * p.y), li = (Real)(sr * p.y + si * p.x);
        s += lr * lr + li * li;
    }
    s = block_sum(s, scratch);
    __shared__ double tot;
    if (threadIdx.x == 0) tot = s;
    __syncthreads();
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        S.norm2[b] = tot;
        S.sc[B + b] = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
    }
}

// One CTA per trajectory: the block-triangular exponential and the
// coefficient sets of the gradient kernel,
//   M[a][b]  = tau |lam| scW_a N_ab scV_b                  (a, b = 1..m)
//   P[a][c]  = sum_b M'_ab K_bc, H q^V_b = sum_c K_bc r^V_c (c = 1..m+1)
//   yw[a]    = |lam| conj(E_a0) scW_a
// with M'_ab = tau |lam| scW_a N_ab and K from beta_b q_{b+1} = H q_b -
// alpha_b q_b - beta_{b-1} q_{b-1} (complex alpha), q_c = sc_c r_c.
template <typename Real>
__global__ void k_adj_small(int m, int B, double tau_im, BatchedScalars SV, BatchedScalars SW,
                            typename R2<Real>::T* __restrict__ coef) {
    using T2 = typename R2<Real>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    const int b = blockIdx.x, L = 2 * m;
    cd* A = reinterpret_cast<cd*>(smem);
    auto tri = [&](const BatchedScalars& S, int i, int j) -> double {
        // real symmetric tridiagonal (Hermitian Lanczos), 0-based indices
        if (i == j) return S.alpha[2 * ((size_t)(i + 1) * B + b)];
        if (j == i + 1) return S.beta[(size_t)(i + 1) * B + b];
        if (i == j + 1) return S.beta[(size_t)(j + 1) * B + b];
        return 0.0;
    };
    for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
        const int i = e / L, j = e - i * L;
        cd t = cmk(0.0, 0.0);
        if (i < m && j < m) t = cmk(0.0, tau_im * tri(SW, i, j));
        else if (i >= m && j >= m) t = cmk(0.0, tau_im * tri(SV, i - m, j - m));
        else if (i == 0 && j == m) t = cmk(1.0, 0.0);
        A[e] = t;
    }
    __syncthreads();
    cd* E = nullptr;
    const int s = pade_exp_sm(L, DQ_NORM_COMPLEX, smem, &E);
    if (s < 0) {
        if (threadIdx.x == 0) atomicCAS(SV.status, 0, s == -1 ? DQ_ERR_SCALING : DQ_ERR_SINGULAR);
        return;
    }
    const double ln = sqrt(SW.norm2[b]);
    const int CS = m * (2 * m + 2);
    T2* out = coef + (size_t)b * CS;
    auto scv = [&](int j) { return SV.sc[(size_t)j * B + b]; };   // 1-based
    auto scw = [&](int j) { return SW.sc[(size_t)j * B + b]; };
    // M'(a, bb), 1-based
    auto mp = [&](int a, int bb) -> cd {
        const cd nab = E[(a - 1) * L + m + (bb - 1)];
        return cmul(cmk(0.0, tau_im * ln * scw(a)), nab);
    };
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int a = e / m + 1, bb = e % m + 1;
        const cd v = cscale(mp(a, bb), scv(bb));
        T2 o;
        o.x = (Real)v.x;
        o.y = (Real)v.y;
        out[e] = o;
    }
    for (int e = threadIdx.x; e < m * (m + 1); e += blockDim.x) {
        const int a = e / (m + 1) + 1, cc = e % (m + 1) + 1;
        cd p = cmk(0.0, 0.0);
        // H q_{c-1} holds r_c with weight beta_{c-1} sc_c (1 when the slab keeps
        // the unnormalised residual, beta_{c-1} when it keeps q_c itself)
        if (cc - 1 >= 1) p = cadd(p, cscale(mp(a, cc - 1), SV.beta[(size_t)(cc - 1) * B + b] * scv(cc)));
        if (cc <= m) {
            const size_t k = (size_t)cc * B + b;
            p = cadd(p, cmul(mp(a, cc), cmk(SV.alpha[2 * k] * scv(cc), SV.alpha[2 * k + 1] * scv(cc))));
        }
        if (cc + 1 <= m) p = cadd(p, cscale(mp(a, cc + 1), SV.beta[(size_t)cc * B + b] * scv(cc)));
        T2 o;
        o.x = (Real)p.x;
        o.y = (Real)p.y;
        out[m * m + e] = o;
    }
    for (int a = threadIdx.x; a < m; a += blockDim.x) {
        const cd z = cconj(E[a * L]);
        const cd v = cscale(z, ln * scw(a + 1));
        T2 o;
        o.x = (Real)v.x;
        o.y = (Real)v.y;
        out[m * m + m * (m + 1) + a] = o;
    }
}

// Per (site, trajectory): the site and coupling forms of this step and the
// new lambda (written over the lambda workspace's slab 1, which holds the
// old one: each element is read by its own thread before it is replaced).
// Sums over the CTA's trajectories go to gsite/gcpl[row][traj group] (one
// writer each, deterministic); |lambda|^2 partials to lpart[cta][b].
template <typename Real, int MM>
__global__ void __launch_bounds__(kAdjThreads, 2) k_adj_grad(int n, int B, int m, int rows_per_cta, int G,
                                                         const Real* __restrict__ sV, Real* sW, size_t slab_reals,
                                                         const Real* __restrict__ d, const cd* __restrict__ psi0,
                                                         const cd* __restrict__ Gt, double invB, int write_lam,
                                                         const typename R2<Real>::T* __restrict__ coef,
                                                         double* __restrict__ lpart, double* __restrict__ gsite,
                                                         double* __restrict__ gcpl) {
    using T2 = typename R2<Real>::T;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T2* cs = reinterpret_cast<T2*>(sm_raw);
    const int CS = m * (2 * m + 2);
    const int tl = threadIdx.x % kAdjTraj, rl = threadIdx.x / kAdjTraj;
    constexpr int kRowLanes = kAdjThreads / kAdjTraj;
    const int b = blockIdx.y * kAdjTraj + tl;
    for (int e = threadIdx.x; e < CS * kAdjTraj; e += blockDim.x) {
        const int t = e % kAdjTraj, idx = e / kAdjTraj;
        cs[e] = coef[(size_t)(blockIdx.y * kAdjTraj + t) * CS + idx];
    }
    __syncthreads();
    const T2* Mc = cs;
    const T2* Pc = cs + (size_t)m * m * kAdjTraj;
    const T2* Yc = Pc + (size_t)m * (m + 1) * kAdjTraj;
    const cd g = Gt[0];
    const double sr = g.x * invB, si = -g.y * invB;
    const int r0 = blockIdx.x * rows_per_cta, r1 = min(n, r0 + rows_per_cta);
    double lnn = 0.0;
    // uniform trip count across the warp: the trajectory-lane shuffles below
    // need every lane
    for (int base = r0; base < r1; base += kRowLanes) {
        const int row = base + rl;
        const bool valid = row < r1;
        const size_t x = (size_t)(valid ? row : r0) * B + b;
        Real vr[MM + 1], vi[MM + 1];
#pragma unroll
        for (int c = 0; c <= MM; ++c) {
            if (c <= m) {
                const T2 v = *reinterpret_cast<const T2*>(sV + (size_t)c * slab_reals + 2 * x);
                vr[c] = v.x;
                vi[c] = v.y;
            } else {
                vr[c] = 0;
                vi[c] = 0;
            }
        }
        Real site = 0, cpl = 0;
        const cd p0 = psi0[valid ? row : r0];
        Real lr = (Real)(sr * p0.x - si * p0.y), li = (Real)(sr * p0.y + si * p0.x);
        // W column streamed four entries ahead (a register pipeline), so its
        // loads overlap the products
        auto ldw = [&](int a) {
            T2 v;
            if (a < m) v = *reinterpret_cast<const T2*>(sW + (size_t)(a + 1) * slab_reals + 2 * x);
            else { v.x = 0; v.y = 0; }
            return v;
        };
        auto body = [&](int a, const T2& w) {
            Real Xr = 0, Xi = 0, Yr = 0, Yi = 0;
#pragma unroll
            for (int c = 0; c < MM; ++c) {
                if (c < m) {
                    const T2 M = Mc[(a * m + c) * kAdjTraj + tl];
                    Xr = fma(M.x, vr[c], fma(-M.y, vi[c], Xr));
                    Xi = fma(M.x, vi[c], fma(M.y, vr[c], Xi));
                }
            }
#pragma unroll
            for (int c = 0; c <= MM; ++c) {
                if (c <= m) {
                    const T2 P = Pc[(a * (m + 1) + c) * kAdjTraj + tl];
                    Yr = fma(P.x, vr[c], fma(-P.y, vi[c], Yr));
                    Yi = fma(P.x, vi[c], fma(P.y, vr[c], Yi));
                }
            }
            site = fma(w.x, Xr, fma(w.y, Xi, site));
            cpl = fma(w.x, Yr, fma(w.y, Yi, cpl));
            const T2 y = Yc[a * kAdjTraj + tl];
            lr = fma(y.x, w.x, fma(-y.y, w.y, lr));
            li = fma(y.x, w.y, fma(y.y, w.x, li));
        };
        T2 w0 = ldw(0), w1 = ldw(1), w2 = ldw(2), w3 = ldw(3);
        for (int a = 0; a < m; a += 4) {
            const T2 n0 = ldw(a + 4), n1 = ldw(a + 5), n2 = ldw(a + 6), n3 = ldw(a + 7);
            body(a, w0);
            if (a + 1 < m) body(a + 1, w1);
            if (a + 2 < m) body(a + 2, w2);
            if (a + 3 < m) body(a + 3, w3);
            w0 = n0;
            w1 = n1;
            w2 = n2;
            w3 = n3;
        }
        double s_d = valid ? (double)site : 0.0;
        double c_d = valid ? (double)cpl - (double)d[x] * (double)site : 0.0;
        if (valid && write_lam) {
            T2 o;
            o.x = lr;
            o.y = li;
            *reinterpret_cast<T2*>(sW + slab_reals + 2 * x) = o;
            lnn += (double)lr * lr + (double)li * li;
        }
#pragma unroll
        for (int o = 1; o < kAdjTraj; o <<= 1) {
            s_d += __shfl_xor_sync(0xffffffffu, s_d, o);
            c_d += __shfl_xor_sync(0xffffffffu, c_d, o);
        }
        if (valid && tl == 0) {
            gsite[(size_t)row * G + blockIdx.y] += s_d;
            gcpl[(size_t)row * G + blockIdx.y] += c_d;
        }
    }
    __shared__ double red[kAdjThreads];
    red[threadIdx.x] = lnn;
    __syncthreads();
    if (rl == 0) {
        double s = 0.0;
        for (int r = 0; r < kRowLanes; ++r) s += red[r * kAdjTraj + tl];
        lpart[(size_t)blockIdx.x * B + b] = s;
    }
}

// Coupling-class gradients when there are several classes:
//   dL/dscale_c += sum_{p in c} vbase_p Re sum_b t_b(i) rV_b(col_p),
//   t_b(i) = sum_a M_ab conj(rW_a(i)),
// gathering the V basis at every neighbour column (m loads per entry).  With
// skip0, class-0 entries are left out: their sum follows on the host from the
// total off-diagonal form (free from the Lanczos relation in k_adj_grad).
template <typename Real, int MM>
__global__ void __launch_bounds__(kAdjThreads, 2) k_adj_cls(int n, int B, int m, int rows_per_cta, int G, int C,
                                                        const Real* __restrict__ sV, const Real* __restrict__ sW,
                                                        size_t slab_reals, const int* __restrict__ rowptr,
                                                        const int* __restrict__ col, const int* __restrict__ cls,
                                                        const double* __restrict__ vbase,
                                                        const typename R2<Real>::T* __restrict__ coef,
                                                        double* __restrict__ gcls, int skip0) {
    using T2 = typename R2<Real>::T;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T2* Mc = reinterpret_cast<T2*>(sm_raw);
    const int CS = m * (2 * m + 2);
    const int tl = threadIdx.x % kAdjTraj, rl = threadIdx.x / kAdjTraj;
    constexpr int kRowLanes = kAdjThreads / kAdjTraj;
    const int b = blockIdx.y * kAdjTraj + tl;
    for (int e = threadIdx.x; e < m * m * kAdjTraj; e += blockDim.x) {
        const int t = e % kAdjTraj, idx = e / kAdjTraj;
        Mc[e] = coef[(size_t)(blockIdx.y * kAdjTraj + t) * CS + idx];
    }
    __syncthreads();
    const int r0 = blockIdx.x * rows_per_cta, r1 = min(n, r0 + rows_per_cta);
    for (int base = r0; base < r1; base += kRowLanes) {
        const int row = base + rl;
        const bool valid = row < r1;
        const size_t x = (size_t)(valid ? row : r0) * B + b;
        Real tr[MM], ti[MM];
#pragma unroll
        for (int c = 0; c < MM; ++c) { tr[c] = 0; ti[c] = 0; }
        for (int a = 0; a < m; ++a) {
            const T2 w = *reinterpret_cast<const T2*>(sW + (size_t)(a + 1) * slab_reals + 2 * x);
#pragma unroll
            for (int c = 0; c < MM; ++c) {
                if (c < m) {
                    const T2 M = Mc[(a * m + c) * kAdjTraj + tl];
                    tr[c] = fma(M.x, w.x, fma(M.y, w.y, tr[c]));    // M conj(w)
                    ti[c] = fma(M.y, w.x, fma(-M.x, w.y, ti[c]));
                }
            }
        }
        double acc[kAdjMaxClasses];
#pragma unroll
        for (int q = 0; q < kAdjMaxClasses; ++q) acc[q] = 0.0;
        if (valid) {
            // the row's couplings (of the gathered classes) in batches of KP:
            // for each Krylov index the batch's gathers are independent loads,
            // so a batch keeps up to KP x m loads in flight instead of a chain
            // per entry (KP = 8 against 4 and 2: 179 vs 203 and 204 us per
            // launch on the 64 x 64 lattice, 232 us one entry at a time)
            constexpr int KP = 8;
            const int pe = rowptr[row + 1];
            int p = rowptr[row];
            while (p < pe) {
                size_t xk[KP];
                int qk[KP];
                double vk[KP];
#pragma unroll
                for (int k = 0; k < KP; ++k) { xk[k] = x; qk[k] = 0; vk[k] = 0.0; }
                int nk = 0;
                for (; p < pe && nk < KP; ++p) {
                    const int q = cls[p];
                    if (skip0 && q == 0) continue;
                    const size_t xv = (size_t)col[p] * B + b;
                    const double vv = vbase[p];
#pragma unroll
                    for (int k = 0; k < KP; ++k)   // register slots, no indexed local array
                        if (k == nk) { xk[k] = xv; qk[k] = q; vk[k] = vv; }
                    ++nk;
                }
                if (nk == 0) break;   // the rest of the row is class 0
                Real rr[KP];
#pragma unroll
                for (int k = 0; k < KP; ++k) rr[k] = 0;
#pragma unroll
                for (int c = 0; c < MM; ++c) {
                    if (c < m) {
#pragma unroll
                        for (int k = 0; k < KP; ++k) {   // unused slots read the own row, weight 0
                            const T2 v = *reinterpret_cast<const T2*>(sV + (size_t)c * slab_reals + 2 * xk[k]);
                            rr[k] = fma(tr[c], v.x, fma(-ti[c], v.y, rr[k]));   // Re(t v)
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < KP; ++k) {
                    const double contrib = vk[k] * (double)rr[k];
#pragma unroll
                    for (int q = 0; q < kAdjMaxClasses; ++q) acc[q] += (q == qk[k]) ? contrib : 0.0;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kAdjMaxClasses; ++q) {
#pragma unroll
            for (int o = 1; o < kAdjTraj; o <<= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        }
        if (valid && tl == 0)
            for (int q = 0; q < C; ++q) gcls[((size_t)row * G + blockIdx.y) * C + q] += acc[q];
    }
}

__global__ void k_cls_final(int n, int G, int C, const double* __restrict__ gcls, double* __restrict__ out) {
    __shared__ double scratch[32];
    for (int q = 0; q < C; ++q) {
        double c = 0.0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            for (int g = 0; g < G; ++g) c += gcls[((size_t)i * G + g) * C + q];
        c = block_sum(c, scratch);
        if (threadIdx.x == 0) out[(size_t)blockIdx.x * C + q] = c;
    }
}

__global__ void k_lam_norm(int B, int nblk, const double* __restrict__ lpart, BatchedScalars S) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < nblk; ++k) s += lpart[(size_t)k * B + b];
        S.norm2[b] = s;
        S.sc[B + b] = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    }
}

__global__ void k_grad_final(int n, int G, const double* __restrict__ gsite, const double* __restrict__ gcpl,
                             double* __restrict__ out) {
    __shared__ double scratch[32];
    double c = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0, t = 0.0;
        for (int g = 0; g < G; ++g) {
            s += gsite[(size_t)i * G + g];
            t += gcpl[(size_t)i * G + g];
        }
        out[i] = s;
        c += t;
    }
    c = block_sum(c, scratch);
    if (threadIdx.x == 0) out[n + blockIdx.x] = c;
}

// ---------------------------------------------------------------------------
#define DQ_CU(call)                                                     \
    do {                                                                \
        dq_status _s = check_cuda(c, (call), #call);                    \
        if (_s != DQ_OK) return _s;                                     \
    } while (0)

static void free_adj_buffers(AdjointState* a) {
    cudaFree(a->d_target); cudaFree(a->d_spec); cudaFree(a->d_g); cudaFree(a->d_G); cudaFree(a->d_loss);
    // the two sets swap places (use_set); both fields always hold one each
    cudaFree(a->seg_V); cudaFree(a->seg_sc); cudaFree(a->seg_diag);
    cudaFree(a->seg_V2); cudaFree(a->seg_sc2); cudaFree(a->seg_diag2);
    if (a->rstream) cudaStreamDestroy(a->rstream);
    if (a->ev_go) cudaEventDestroy(a->ev_go);
    for (int k = 0; k < 2; ++k) {
        if (a->ev_rec[k]) cudaEventDestroy(a->ev_rec[k]);
        if (a->ev_sweep[k]) cudaEventDestroy(a->ev_sweep[k]);
    }
    cudaFree(a->ck_psi); cudaFree(a->ck_n2); cudaFree(a->ck_deps);
    cudaFree(a->d_coef); cudaFree(a->d_lpart); cudaFree(a->d_gsite); cudaFree(a->d_gcpl); cudaFree(a->d_gout);
    cudaFree(a->d_erracc_save);
    cudaFree(a->d_cls); cudaFree(a->d_vbase); cudaFree(a->d_gcls); cudaFree(a->d_gcls_out);
    batched_free_ws(a->ws2);
}

void adjoint_free(dq_ctx* c) {
    if (!c->adj) return;
    free_adj_buffers(c->adj);
    delete c->adj;
    c->adj = nullptr;
}

static int mm_bucket(int m) { return m <= 8 ? 8 : m <= 16 ? 16 : 24; }

template <typename Real, int MM>
static cudaError_t grad_attr(int bytes) {
    cudaError_t e = raise_smem_limit(k_adj_grad<Real, MM>, bytes);
    if (e != cudaSuccess) return e;
    return raise_smem_limit(k_adj_cls<Real, MM>, bytes);
}

// Makes set k (segment s uses set s % 2) the one seg_V / seg_sc / seg_diag
// name; with a single set every segment uses it.
static void use_set(AdjointState* a, int k) {
    if (!a->seg_V2 || a->cur_set == k) return;
    std::swap(a->seg_V, a->seg_V2);
    std::swap(a->seg_sc, a->seg_sc2);
    std::swap(a->seg_diag, a->seg_diag2);
    a->cur_set = k;
}

static unsigned char* slot_V(AdjointState* a, int m, int slot) {
    return a->seg_V + (size_t)slot * (m + 1) * a->slab_bytes;
}

template <typename Real>
static void launch_grad(dq_ctx* c, AdjointState* a, int t, int slot, int write_lam) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B, m = c->cfg.m, G = B / kAdjTraj;
    const size_t slab_reals = (size_t)n * B * 2;
    const int CS = m * (2 * m + 2);
    const size_t smem = (size_t)CS * kAdjTraj * sizeof(typename R2<Real>::T);
    const dim3 grid(a->row_ctas, G);
    using T2 = typename R2<Real>::T;
#define DQ_GRAD(MMV)                                                                                               \
    k_adj_grad<Real, MMV><<<grid, kAdjThreads, smem, c->stream>>>(                                                  \
        n, B, m, a->rows_per_cta, G, (const Real*)slot_V(a, m, slot), (Real*)a->ws2->slabs, slab_reals,          \
        (const Real*)(a->seg_diag + (size_t)slot * a->diag_bytes),                                                 \
        c->d_psi0, a->d_G + t, a->inv_norm, write_lam, (const T2*)a->d_coef, a->d_lpart, a->d_gsite, a->d_gcpl)
    switch (mm_bucket(m)) {
        case 8: DQ_GRAD(8); break;
        case 16: DQ_GRAD(16); break;
        default: DQ_GRAD(24); break;
    }
#undef DQ_GRAD
}

template <typename Real>
static void launch_cls(dq_ctx* c, AdjointState* a, int slot) {
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B, m = c->cfg.m, G = B / kAdjTraj;
    const size_t slab_reals = (size_t)n * B * 2;
    const size_t smem = (size_t)m * m * kAdjTraj * sizeof(typename R2<Real>::T);
    const dim3 grid(a->row_ctas, G);
    using T2 = typename R2<Real>::T;
#define DQ_CLS(MMV)                                                                                                  \
    k_adj_cls<Real, MMV><<<grid, kAdjThreads, smem, c->stream>>>(n, B, m, a->rows_per_cta, G, a->n_cls,                \
                                                               (const Real*)slot_V(a, m, slot),                      \
                                                               (const Real*)a->ws2->slabs,                           \
                                                               slab_reals, c->d_rowptr, c->d_col, a->d_cls,           \
                                                               a->d_vbase, (const T2*)a->d_coef, a->d_gcls,    \
                                                               c->scales[0] != 0.0)
    switch (mm_bucket(m)) {
        case 8: DQ_CLS(8); break;
        case 16: DQ_CLS(16); break;
        default: DQ_CLS(24); break;
    }
#undef DQ_CLS
}

template <typename Real>
static cudaError_t set_attrs(int m) {
    const int CS = m * (2 * m + 2);
    const int smem = CS * kAdjTraj * (int)sizeof(typename R2<Real>::T);
    cudaError_t e = raise_smem_limit(k_adj_small<Real>, (int)pade_smem_bytes(2 * m));
    if (e != cudaSuccess) return e;
    switch (mm_bucket(m)) {
        case 8: return grad_attr<Real, 8>(smem);
        case 16: return grad_attr<Real, 16>(smem);
        default: return grad_attr<Real, 24>(smem);
    }
}

// Copies of one step's state (slab 1 and norms) and diagonal.
static dq_status save_state(dq_ctx* c, AdjointState* a, unsigned char* psi_dst, double* n2_dst) {
    BatchedState* bs = c->bat;
    DQ_CU(cudaMemcpyAsync(psi_dst, (unsigned char*)bs->slabs + a->slab_bytes, a->slab_bytes, cudaMemcpyDeviceToDevice,
                          c->stream));
    DQ_CU(cudaMemcpyAsync(n2_dst, bs->s.norm2, sizeof(double) * bs->B, cudaMemcpyDeviceToDevice, c->stream));
    return DQ_OK;
}

// Runs steps [s0, s1) from the current ensemble state and keeps, in slot
// k - s0, the step's starting state, diagonal, Krylov residuals r_2..r_{m+1}
// and Lanczos scalars.
static dq_status run_segment(dq_ctx* c, AdjointState* a, int s0, int s1, bool record_pops) {
    BatchedState* bs = c->bat;
    const int m = c->cfg.m;
    dq_status hook_st = DQ_OK;
    for (int k = s0; k < s1; ++k) {
        const int slot = k - s0;
        unsigned char* V = slot_V(a, m, slot);
        double* scb = a->seg_sc + (size_t)slot * scal_block(bs->B);
        const size_t LB = (size_t)kMaxL * bs->B;
        DQ_CU(cudaMemcpyAsync(V, (unsigned char*)bs->slabs + a->slab_bytes, a->slab_bytes, cudaMemcpyDeviceToDevice,
                              c->stream));
        // sc_1 = 1/|psi(k)| now; the step's combine replaces it with the next state's
        DQ_CU(cudaMemcpyAsync(scb + 3 * LB + bs->B, bs->s.sc + bs->B, sizeof(double) * bs->B, cudaMemcpyDeviceToDevice,
                              c->stream));
        std::function<void()> hook = [&]() {
            cudaError_t e = cudaMemcpyAsync(a->seg_diag + (size_t)slot * a->diag_bytes, bs->diag, a->diag_bytes,
                                            cudaMemcpyDeviceToDevice, c->stream);
            if (e != cudaSuccess) hook_st = check_cuda(c, e, "adjoint diagonal copy");
        };
        dq_status st;
        if ((st = batched_step_eager(c, &hook, !record_pops))) return st;
        if (hook_st) return hook_st;
        // the combine replaced slab 1; slabs 2..m+1 still hold this step's basis
        DQ_CU(cudaMemcpyAsync(V + a->slab_bytes, (unsigned char*)bs->slabs + 2 * a->slab_bytes, m * a->slab_bytes,
                              cudaMemcpyDeviceToDevice, c->stream));
        // alpha, beta and sc_0, then sc_2.. (sc_1 was kept before the step)
        DQ_CU(cudaMemcpyAsync(scb, bs->s.alpha, sizeof(double) * (3 * LB + bs->B), cudaMemcpyDeviceToDevice,
                              c->stream));
        DQ_CU(cudaMemcpyAsync(scb + 3 * LB + 2 * bs->B, bs->s.sc + 2 * bs->B, sizeof(double) * (LB - 2 * bs->B),
                              cudaMemcpyDeviceToDevice, c->stream));
    }
    return DQ_OK;
}

static dq_status read_device_status(dq_ctx* c, const char* what) {
    int status = 0;
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(&status, c->bat->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return read_status(c, status, what);
    return DQ_OK;
}

}  // namespace dq

using namespace dq;

namespace {
dq_status fail(dq_ctx* c, int code, const char* msg) {
    c->err = msg;
    return code;
}
}  // namespace

extern "C" {

dq_status dq_adjoint_setup(dq_ctx* c, int n_steps, int fft_len, double scale, const double* target,
                           int checkpoint_every) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (c->cfg.dot_mode != DQ_DOT_HERMITIAN) return fail(c, DQ_ERR_ARG, "adjoint: needs the Hermitian Lanczos dot");
    if (c->cfg.reorth) return fail(c, DQ_ERR_ARG, "adjoint: not with reorthogonalisation (the recurrence is used)");
    if (c->cfg.m_min > 0) return fail(c, DQ_ERR_ARG, "adjoint: needs a fixed Krylov dimension (m_min = 0)");
    if (c->tk_p > 0) return fail(c, DQ_ERR_ARG, "adjoint: Lanczos mode only (not Taylor-Krylov)");
    if (c->d_bra) return fail(c, DQ_ERR_ARG, "adjoint: the loss uses the correlation with psi0 (no separate bra)");
    if (c->cfg.m > kAdjMaxM) return fail(c, DQ_ERR_ARG, "adjoint: m must be <= 24");
    if (n_steps < 1 || n_steps > c->cfg.max_steps) return fail(c, DQ_ERR_ARG, "adjoint: n_steps out of range");
    if (fft_len < n_steps + 1 || (fft_len & (fft_len - 1))) {
        return fail(c, DQ_ERR_ARG, "adjoint: fft_len must be a power of two >= n_steps + 1");
    }
    if (!target || !std::isfinite(scale) || checkpoint_every < 0) return fail(c, DQ_ERR_ARG, "adjoint: bad arguments");
    if (c->scales.size() > (size_t)kAdjMaxClasses) return fail(c, DQ_ERR_ARG, "adjoint: at most 8 coupling classes");
    if (c->cfg.n_traj % kAdjTraj) return fail(c, DQ_ERR_ARG, "adjoint: n_traj must be a multiple of 8");
    dq_status st;
    if (!c->bat) {
        if ((st = batched_alloc(c))) return st;
        c->ready = false;
    }
    adjoint_free(c);
    AdjointState* a = new AdjointState();
    c->adj = a;
    BatchedState* bs = c->bat;
    const int n = c->n, B = bs->B, m = c->cfg.m;
    const size_t rsz = bs->mixed ? sizeof(float) : sizeof(double);
    a->T = n_steps;
    a->len = fft_len;
    a->scale = scale;
    a->slab_bytes = (size_t)n * B * 2 * rsz;
    a->diag_bytes = (size_t)n * B * rsz;
    const size_t per_step = a->slab_bytes * (m + 1) + a->diag_bytes + sizeof(double) * scal_block(B);
    const size_t per_ck = a->slab_bytes + sizeof(double) * B + sizeof(double) * (size_t)n * B;
    size_t free_b = 0, total_b = 0;
    DQ_CU(cudaMemGetInfo(&free_b, &total_b));
    // the lambda workspace and the gradient buffers come first
    const size_t ws_bytes = a->slab_bytes * (m + 2) + a->diag_bytes + sizeof(double) * (size_t)n * B * 2 + (64u << 20);
    const size_t avail = free_b > ws_bytes ? free_b - ws_bytes : 0;
    int K = checkpoint_every;
    if (K == 0) {
        if ((size_t)n_steps * per_step <= avail / 2) K = n_steps;
        else K = std::max(1, (int)std::ceil(std::sqrt((double)n_steps)));
    }
    K = std::min(K, n_steps);
    const int n_seg = (n_steps + K - 1) / K;
    if ((size_t)K * per_step + (size_t)(n_seg - 1) * per_ck > avail) {
        adjoint_free(c);
        return fail(c, DQ_ERR_CUDA, "adjoint: not enough device memory for the stored states");
    }
    a->K = K;
    a->n_seg = n_seg;
    do {
        if ((st = check_cuda(c, cudaMalloc(&a->d_target, sizeof(double) * fft_len), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMemcpy(a->d_target, target, sizeof(double) * fft_len, cudaMemcpyHostToDevice),
                             "adjoint target"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_spec, sizeof(cd) * fft_len), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_g, sizeof(cd) * fft_len), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_G, sizeof(cd) * fft_len), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_loss, sizeof(double)), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->seg_V, a->slab_bytes * (m + 1) * K), "adjoint Krylov bases"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->seg_sc, sizeof(double) * scal_block(B) * K), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->seg_diag, a->diag_bytes * K), "adjoint diagonals"))) break;
        if (n_seg > 1 && (size_t)2 * K * per_step + (size_t)(n_seg - 1) * per_ck <= avail) {
            // second set of segment slots for the overlapped backward; without it the
            // backward runs its recomputes and sweeps one after another
            if (cudaMalloc(&a->seg_V2, a->slab_bytes * (m + 1) * K) != cudaSuccess ||
                cudaMalloc(&a->seg_sc2, sizeof(double) * scal_block(B) * K) != cudaSuccess ||
                cudaMalloc(&a->seg_diag2, a->diag_bytes * K) != cudaSuccess ||
                cudaStreamCreateWithFlags(&a->rstream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&a->ev_go, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&a->ev_rec[0], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&a->ev_rec[1], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&a->ev_sweep[0], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&a->ev_sweep[1], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                cudaFree(a->seg_V2); cudaFree(a->seg_sc2); cudaFree(a->seg_diag2);
                a->seg_V2 = nullptr; a->seg_sc2 = nullptr; a->seg_diag2 = nullptr;
            }
        }
        if (n_seg > 1) {
            if ((st = check_cuda(c, cudaMalloc(&a->ck_psi, a->slab_bytes * (n_seg - 1)), "adjoint checkpoints"))) break;
            if ((st = check_cuda(c, cudaMalloc(&a->ck_n2, sizeof(double) * B * (n_seg - 1)), "adjoint alloc"))) break;
            if ((st = check_cuda(c, cudaMalloc(&a->ck_deps, sizeof(double) * (size_t)n * B * (n_seg - 1)),
                                 "adjoint checkpoints"))) break;
        }
        const int CS = m * (2 * m + 2);
        if ((st = check_cuda(c, cudaMalloc(&a->d_coef, 2 * rsz * (size_t)B * CS), "adjoint alloc"))) break;
        const int G = B / kAdjTraj;
        a->row_ctas = std::max(1, std::min((bs->sms * 4 + G - 1) / G, (n + 31) / 32));
        a->rows_per_cta = (n + a->row_ctas - 1) / a->row_ctas;
        a->row_ctas = (n + a->rows_per_cta - 1) / a->rows_per_cta;
        if ((st = check_cuda(c, cudaMalloc(&a->d_lpart, sizeof(double) * (size_t)a->row_ctas * B), "adjoint alloc")))
            break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_gsite, sizeof(double) * (size_t)n * G), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_gcpl, sizeof(double) * (size_t)n * G), "adjoint alloc"))) break;
        a->fin_blocks = std::max(1, std::min(bs->sms * 2, (n + 255) / 256));
        if ((st = check_cuda(c, cudaMalloc(&a->d_gout, sizeof(double) * (n + a->fin_blocks)), "adjoint alloc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&a->d_erracc_save, sizeof(double) * B), "adjoint alloc"))) break;
        a->ws2 = batched_alloc_ws(c, B, bs->mixed, &st);
        if (st) break;
        cudaError_t e = bs->mixed ? set_attrs<float>(m) : set_attrs<double>(m);
        if ((st = check_cuda(c, e, "adjoint kernel attributes"))) break;
    } while (0);
    if (st) {
        adjoint_free(c);
        return st;
    }
    return DQ_OK;
}

}  // extern "C"

namespace dq {
// The forward run of the adjoint: every step of this context's trajectories
// with checkpoints and the stored last segment; the correlation sums end in
// c->d_corr.
static dq_status forward_run(dq_ctx* c) {
    AdjointState* a = c->adj;
    if (!a) return fail(c, DQ_ERR_STATE, "forward: call dq_adjoint_setup first");
    if (c->scales.size() > (size_t)kAdjMaxClasses) return fail(c, DQ_ERR_ARG, "adjoint: at most 8 coupling classes");
    dq_status st;
    a->forward_done = false;
    if ((st = dq_reset(c))) return st;
    BatchedState* bs = c->bat;
    const int B = bs->B, n = c->n;
    // several coupling classes: the gather kernel needs each entry's class and base value
    const int C = c->scales.size() > 1 ? (int)c->scales.size() : 0;
    cudaFree(a->d_cls); cudaFree(a->d_vbase); cudaFree(a->d_gcls); cudaFree(a->d_gcls_out);
    a->d_cls = nullptr; a->d_vbase = nullptr; a->d_gcls = nullptr; a->d_gcls_out = nullptr;
    a->n_cls = C;
    if (C) {
        const size_t nnz = std::max<size_t>(c->cls.size(), 1);
        DQ_CU(cudaMalloc(&a->d_cls, sizeof(int) * nnz));
        DQ_CU(cudaMalloc(&a->d_vbase, sizeof(double) * nnz));
        if (!c->cls.empty()) {
            DQ_CU(cudaMemcpy(a->d_cls, c->cls.data(), sizeof(int) * c->cls.size(), cudaMemcpyHostToDevice));
            DQ_CU(cudaMemcpy(a->d_vbase, c->val_base.data(), sizeof(double) * c->cls.size(), cudaMemcpyHostToDevice));
        }
        DQ_CU(cudaMalloc(&a->d_gcls, sizeof(double) * (size_t)n * (B / kAdjTraj) * C));
        DQ_CU(cudaMalloc(&a->d_gcls_out, sizeof(double) * (size_t)a->fin_blocks * C));
    }
    const int last_s0 = (a->n_seg - 1) * a->K;
    for (int s = 0; s + 1 < a->n_seg; ++s) {
        // checkpoint at the segment start, then run the segment unrecorded
        if ((st = save_state(c, a, a->ck_psi + (size_t)s * a->slab_bytes, a->ck_n2 + (size_t)s * B))) return st;
        DQ_CU(cudaMemcpyAsync(a->ck_deps + (size_t)s * n * B, bs->deps, sizeof(double) * (size_t)n * B,
                              cudaMemcpyDeviceToDevice, c->stream));
        for (int k = s * a->K; k < (s + 1) * a->K; ++k)
            if ((st = batched_step_eager(c, nullptr, false))) return st;
    }
    use_set(a, (a->n_seg - 1) % 2);
    if ((st = run_segment(c, a, last_s0, a->T, true))) return st;
    c->steps_done = a->T;
    c->last_path = 1;
    if ((st = batched_collect_corr(c))) return st;
    return read_device_status(c, "forward");
}

// Loss of the ensemble-mean correlation (c->d_corr holds the sums over
// n_total trajectories) and the adjoint source of the backward pass.
static dq_status forward_loss(dq_ctx* c, int n_total, double* loss) {
    AdjointState* a = c->adj;
    dq_status st;
    a->inv_norm = 1.0 / n_total;
    if ((st = fft_inverse(c, a->len, c->d_corr, a->T + 1, a->inv_norm, a->d_spec))) return st;
    k_adj_loss<<<1, 1024, 0, c->stream>>>(a->len, a->scale, a->d_target, a->d_spec, a->d_g, a->d_loss);
    if ((st = fft_inverse(c, a->len, a->d_g, a->len, 1.0, a->d_G))) return st;
    if ((st = read_device_status(c, "forward"))) return st;
    if (loss) DQ_CU(cudaMemcpy(loss, a->d_loss, sizeof(double), cudaMemcpyDeviceToHost));
    a->forward_done = true;
    return DQ_OK;
}
}  // namespace dq

extern "C" {

dq_status dq_forward(dq_ctx* c, double* loss) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    dq_status st;
    if ((st = forward_run(c))) return st;
    return forward_loss(c, c->bat->B, loss);
}

dq_status dq_forward_shard(dq_ctx* c, dq_cdouble* corr_sums) {
    DeviceScope dev_scope(c);
    if (!c || !corr_sums) return DQ_ERR_ARG;
    dq_status st;
    if ((st = forward_run(c))) return st;
    DQ_CU(cudaMemcpy(corr_sums, c->d_corr, sizeof(cd) * (size_t)(c->adj->T + 1), cudaMemcpyDeviceToHost));
    return DQ_OK;
}

dq_status dq_forward_reduced(dq_ctx* c, const dq_cdouble* corr_sums, int n_traj_total, double* loss) {
    DeviceScope dev_scope(c);
    if (!c || !corr_sums) return DQ_ERR_ARG;
    AdjointState* a = c->adj;
    if (!a || !c->bat || c->steps_done != a->T || c->last_path != 1)
        return fail(c, DQ_ERR_STATE, "forward_reduced: run dq_forward_shard first");
    if (n_traj_total < c->bat->B) return fail(c, DQ_ERR_ARG, "forward_reduced: fewer trajectories than this shard");
    DQ_CU(cudaMemcpy(c->d_corr, corr_sums, sizeof(cd) * (size_t)(a->T + 1), cudaMemcpyHostToDevice));
    return forward_loss(c, n_traj_total, loss);
}

dq_status dq_backward(dq_ctx* c, double* grad_sites, double* grad_classes) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    AdjointState* a = c->adj;
    if (!a || !a->forward_done || !c->bat || c->steps_done != a->T)
        return fail(c, DQ_ERR_STATE, "backward: run dq_forward first");
    if (!grad_sites) return fail(c, DQ_ERR_ARG, "backward: grad_sites is null");
    BatchedState* bs = c->bat;
    BatchedState* w2 = a->ws2;
    const int n = c->n, B = bs->B, m = c->cfg.m, G = B / kAdjTraj;
    dq_status st;
    if ((st = batched_mirror_tiling(c, w2))) return st;
    DQ_CU(cudaMemcpyAsync(a->d_erracc_save, c->d_erracc, sizeof(double) * B, cudaMemcpyDeviceToDevice, c->stream));
    DQ_CU(cudaMemsetAsync(a->d_gsite, 0, sizeof(double) * (size_t)n * G, c->stream));
    DQ_CU(cudaMemsetAsync(a->d_gcpl, 0, sizeof(double) * (size_t)n * G, c->stream));
    if (a->n_cls) DQ_CU(cudaMemsetAsync(a->d_gcls, 0, sizeof(double) * (size_t)n * G * a->n_cls, c->stream));
    const int init_blocks = std::min(n, bs->sms * 8);
    const int thr = std::min(256, ((B + 31) / 32) * 32);
    unsigned char* w_slab1 = (unsigned char*)w2->slabs + a->slab_bytes;
    if (bs->mixed) k_lambda_init<float><<<init_blocks, thr, 0, c->stream>>>(n, B, c->d_psi0, a->d_G + a->T, a->inv_norm,
                                                                            (float*)w_slab1);
    else k_lambda_init<double><<<init_blocks, thr, 0, c->stream>>>(n, B, c->d_psi0, a->d_G + a->T, a->inv_norm,
                                                                   (double*)w_slab1);
    if (bs->mixed) k_lambda_init_norm<float><<<1, 256, 0, c->stream>>>(n, B, c->d_psi0, a->d_G + a->T, a->inv_norm, w2->s);
    else k_lambda_init_norm<double><<<1, 256, 0, c->stream>>>(n, B, c->d_psi0, a->d_G + a->T, a->inv_norm, w2->s);
    DQ_CU(cudaGetLastError());
    const size_t small_smem = pade_smem_bytes(2 * m);
    const int sc_blocks = (B + 255) / 256;
    // restore segment s's start and recompute its steps into set s % 2, on
    // the stream c->stream names
    auto recompute = [&](int s) -> dq_status {
        const int s0 = s * a->K, s1 = std::min(a->T, s0 + a->K);
        use_set(a, s % 2);
        DQ_CU(cudaMemcpyAsync((unsigned char*)bs->slabs + a->slab_bytes, a->ck_psi + (size_t)s * a->slab_bytes,
                              a->slab_bytes, cudaMemcpyDeviceToDevice, c->stream));
        DQ_CU(cudaMemcpyAsync(bs->s.norm2, a->ck_n2 + (size_t)s * B, sizeof(double) * B, cudaMemcpyDeviceToDevice,
                              c->stream));
        DQ_CU(cudaMemcpyAsync(bs->deps, a->ck_deps + (size_t)s * n * B, sizeof(double) * (size_t)n * B,
                              cudaMemcpyDeviceToDevice, c->stream));
        k_set_sc1<<<sc_blocks, 256, 0, c->stream>>>(B, bs->s);
        k_set_step<<<1, 32, 0, c->stream>>>(bs->s, s0);
        return run_segment(c, a, s0, s1, false);
    };
    // With two slot sets the recompute of segment s - 1 runs on a second
    // stream while the sweep of segment s runs here: the recompute touches the
    // main workspace and set (s - 1) % 2 only, the sweep the second workspace
    // and set s % 2; events order a set's recompute before its sweep and its
    // previous sweep before its next recompute.
    const bool overlap = a->seg_V2 != nullptr && a->n_seg > 1;
    cudaStream_t main_stream = c->stream;
    if (overlap) {
        DQ_CU(cudaEventRecord(a->ev_go, main_stream));
        DQ_CU(cudaStreamWaitEvent(a->rstream, a->ev_go, 0));
    }
    for (int s = a->n_seg - 1; s >= 0; --s) {
        const int s0 = s * a->K, s1 = std::min(a->T, s0 + a->K);
        if (overlap) {
            if (s >= 1) {
                if (s + 1 < a->n_seg) DQ_CU(cudaStreamWaitEvent(a->rstream, a->ev_sweep[(s + 1) % 2], 0));
                c->stream = a->rstream;
                st = recompute(s - 1);
                c->stream = main_stream;
                if (st) return st;
                DQ_CU(cudaEventRecord(a->ev_rec[(s - 1) % 2], a->rstream));
            }
            if (s + 1 < a->n_seg) DQ_CU(cudaStreamWaitEvent(main_stream, a->ev_rec[s % 2], 0));
            use_set(a, s % 2);
        } else if (s + 1 < a->n_seg) {
            if ((st = recompute(s))) return st;
        }
        for (int t = s1 - 1; t >= s0; --t) {
            const int slot = t - s0;
            DQ_CU(cudaMemcpyAsync(w2->diag, a->seg_diag + (size_t)slot * a->diag_bytes, a->diag_bytes,
                                  cudaMemcpyDeviceToDevice, c->stream));
            for (int j = 1; j <= m; ++j)
                if ((st = batched_iteration(c, w2, j))) return st;
            // the kept step's tridiagonal and scales, in the workspace layout
            BatchedScalars SV = bs->s;
            SV.alpha = a->seg_sc + (size_t)slot * scal_block(B);
            SV.beta = SV.alpha + 2 * (size_t)kMaxL * B;
            SV.sc = SV.beta + (size_t)kMaxL * B;
            if (bs->mixed) {
                k_adj_small<float><<<B, 256, small_smem, c->stream>>>(m, B, c->tau_im, SV, w2->s, (float2*)a->d_coef);
                if (a->n_cls) launch_cls<float>(c, a, slot);   // reads lambda(t+1) before k_adj_grad replaces it
                launch_grad<float>(c, a, t, slot, t > 0);
            } else {
                k_adj_small<double><<<B, 256, small_smem, c->stream>>>(m, B, c->tau_im, SV, w2->s,
                                                                       (double2*)a->d_coef);
                if (a->n_cls) launch_cls<double>(c, a, slot);
                launch_grad<double>(c, a, t, slot, t > 0);
            }
            if (t > 0) k_lam_norm<<<sc_blocks, 256, 0, c->stream>>>(B, a->row_ctas, a->d_lpart, w2->s);
            DQ_CU(cudaGetLastError());
        }
        if (overlap) DQ_CU(cudaEventRecord(a->ev_sweep[s % 2], main_stream));
    }
    if (overlap) {
        // every recompute (and its error-estimate sums) done before the restore below
        DQ_CU(cudaEventRecord(a->ev_go, a->rstream));
        DQ_CU(cudaStreamWaitEvent(main_stream, a->ev_go, 0));
    }
    k_grad_final<<<a->fin_blocks, 256, 0, c->stream>>>(n, G, a->d_gsite, a->d_gcpl, a->d_gout);
    if (a->n_cls) k_cls_final<<<a->fin_blocks, 256, 0, c->stream>>>(n, G, a->n_cls, a->d_gcls, a->d_gcls_out);
    DQ_CU(cudaMemcpyAsync(c->d_erracc, a->d_erracc_save, sizeof(double) * B, cudaMemcpyDeviceToDevice, c->stream));
    DQ_CU(cudaGetLastError());
    c->ready = false;   // the ensemble states were overwritten
    if ((st = read_device_status(c, "backward"))) return st;
    int w_status = 0;
    DQ_CU(cudaMemcpy(&w_status, w2->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (w_status) {
        cudaMemsetAsync(w2->s.status, 0, sizeof(int), c->stream);
        return read_status(c, w_status, "backward (adjoint Lanczos)");
    }
    std::vector<double> out(n + a->fin_blocks);
    DQ_CU(cudaMemcpy(out.data(), a->d_gout, sizeof(double) * out.size(), cudaMemcpyDeviceToHost));
    std::memcpy(grad_sites, out.data(), sizeof(double) * n);
    if (grad_classes && a->n_cls) {
        std::vector<double> part((size_t)a->fin_blocks * a->n_cls);
        DQ_CU(cudaMemcpy(part.data(), a->d_gcls_out, sizeof(double) * part.size(), cudaMemcpyDeviceToHost));
        for (int q = 0; q < a->n_cls; ++q) {
            double tot = 0.0;
            for (int k = 0; k < a->fin_blocks; ++k) tot += part[(size_t)k * a->n_cls + q];
            grad_classes[q] = tot;
        }
        if (c->scales[0] != 0.0) {
            // class 0 from the total: sum_p val_p rho_p = sum_c scale_c grad_c
            double total = 0.0;
            for (int k = 0; k < a->fin_blocks; ++k) total += out[n + k];
            double rest = 0.0;
            for (int q = 1; q < a->n_cls; ++q) rest += c->scales[q] * grad_classes[q];
            grad_classes[0] = (total - rest) / c->scales[0];
        }
    } else if (grad_classes) {
        double tot = 0.0;
        for (int k = 0; k < a->fin_blocks; ++k) tot += out[n + k];
        // val = scale * val_base: dL/dscale = (1/scale) sum_p val_p dL/dH_p
        const double s = c->scales.empty() ? 1.0 : c->scales[0];
        if (s == 0.0) return fail(c, DQ_ERR_ARG, "backward: coupling scale is zero");
        grad_classes[0] = tot / s;
    }
    return DQ_OK;
}

}  // extern "C"
