// dq_tk_ensemble.cu — Taylor-Krylov steps of a whole ensemble at once (dq_run
// in Taylor-Krylov mode; taylorKrylovClass.cu:223-434 per trajectory in the
// reference).
//
// FP64 throughout, on [site][traj] slabs of complex128 (coalesced over the
// trajectories of one site).  Every kernel runs on a grid of row groups x
// trajectory blocks: thread (g, b) handles trajectory b on rows g, g + G, ...
// and its per-trajectory sums land in partial[g][b]; the last block to finish
// adds the partials of each trajectory in row-group order (deterministic) and
// writes that trajectory's scalar.  The random draws are the ones of the
// other paths (same Philox keys), so the ensemble reproduces dq_run_plain.
#include <algorithm>

#include "dq_internal.h"
#include "dq_rng.cuh"

namespace dq {

constexpr int kTkRowGroups = 296;   // 2 per SM
constexpr int kTkThreads = 128;

// Device scalars of the ensemble, [j][b] for the Lanczos arrays.
struct TkScal {
    cd* alpha;      // kMaxL x B
    cd* beta;       // kMaxL x B
    double* sc;     // kMaxL x B
    cd* yt;         // kMaxL x B
    double* beta0;  // B
    double* nav;    // B
    double* kerr;   // B
    double* norm;   // B
    double* err;    // B
    double* partial;        // kTkRowGroups x B x 3
    unsigned int* ticket;   // 8
    int* status;
};

struct TkEnsemble {
    int B = 0;
    double* eps = nullptr;   // [site][traj]
    double* deps = nullptr;
    double* diag = nullptr;
    cd* psi = nullptr;       // current states [site][traj]
    cd* Q = nullptr;         // (mb + 2) slabs: r_1 = A^p psi, r_2.. residuals
    cd* x2 = nullptr;        // 2 slabs: A^k psi ping-pong
    cd* acc = nullptr;       // Taylor sum
    cd* w = nullptr;
    double* scal_mem = nullptr;
    TkScal s{};
    int mb_alloc = 0;
};

// ---- per-trajectory reduction over row groups ------------------------------
// Stores this thread's partial values v[0..K) for trajectory b, then returns
// true in the last block, whose threads may read the full sums with tk_sum.
template <int K>
__device__ __forceinline__ bool tk_partials(const double (&v)[K], int b, int B, double* partial,
                                            unsigned int* ticket) {
    if (b < B)
        for (int k = 0; k < K; ++k) partial[((size_t)blockIdx.x * B + b) * 3 + k] = v[k];
    return last_block_ticket(ticket, gridDim.x * gridDim.y);
}

__device__ __forceinline__ double tk_sum(const double* partial, int G, int B, int b, int k) {
    double s = 0.0;
    for (int g = 0; g < G; ++g) s += __ldcg(&partial[((size_t)g * B + b) * 3 + k]);
    return s;
}

// ---- noise (the other paths' draws, gpuSysHelper.cu:32-177) ----------------
__global__ void k_tke_noise(int n, int B, int traj0, int step, int noise, int ns, double subdt, double sqrt_subdt,
                            uint64_t seed, const double* __restrict__ sigma, const double* __restrict__ invtau,
                            const double* __restrict__ coeff, ZZParams zz, const double* __restrict__ eps,
                            double* __restrict__ deps, double* __restrict__ diag) {
    __shared__ double ccw[kMaxZZOsc], csw[kMaxZZOsc];
    if (noise == DQ_NOISE_ZZ) {
        for (int o = threadIdx.x; o < zz.n_osc; o += blockDim.x)
            zz_factors(zz.omega[o], zz.coeff[o], step, zz.dt, ccw[o], csw[o]);
        __syncthreads();
    }
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    if (b >= B) return;
    for (int row = blockIdx.x; row < n; row += gridDim.x) {
        const size_t x = (size_t)row * B + b;
        double v;
        if (noise == DQ_NOISE_OU) {
            const double cur = ou_update(deps[x], invtau[row], coeff[row], subdt, sqrt_subdt, ns, seed, traj0 + b,
                                         step, row);
            deps[x] = cur;
            v = __dadd_rn(cur, eps[x]);
        } else if (noise == DQ_NOISE_GAUSS) {
            v = __dadd_rn(__dmul_rn(normal(seed, P_GAUSS, traj0 + b, step, row, 0), sigma[row]), eps[x]);
        } else if (noise == DQ_NOISE_ZZ) {
            double a = 0.0;
            for (int o = 0; o < zz.n_osc; ++o)
                a = zz_acc(a, ccw[o], csw[o], zz_phase(seed, (uint32_t)(traj0 + b), (uint32_t)row, (uint32_t)o));
            v = __dadd_rn(a, eps[x]);
        } else {
            v = eps[x];
        }
        diag[x] = v;
    }
}

// ---- Taylor part: y = A x; acc += c_k y (k < p); k = p: beta0, sc_1 ---------
__global__ void __launch_bounds__(kTkThreads) k_tke_power(int n, int B, int k, int p, const int* __restrict__ rowptr,
                                                         const int* __restrict__ col,
                                                         const double* __restrict__ val,
                                                         const double* __restrict__ diag, const cd* x,
                                                         cd* __restrict__ y, cd* acc, cd coef, TkScal S) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (b < B) {
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t xi = (size_t)row * B + b;
            cd a = cscale(x[xi], diag[xi]);
            for (int q = rowptr[row]; q < rowptr[row + 1]; ++q) a = cadd(a, cscale(x[(size_t)col[q] * B + b], val[q]));
            y[xi] = a;
            if (k < p) acc[xi] = cadd(k == 1 ? x[xi] : acc[xi], cmul(coef, a));
            v[0] += cabs2(a);
        }
    }
    if (k < p) return;   // uniform over the grid
    if (tk_partials<1>(v, b, B, S.partial, &S.ticket[0])) {
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x) {
            const double nb = sqrt(tk_sum(S.partial, gridDim.x, B, bb, 0));
            if (!(nb > 0.0) || !isfinite(nb)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            S.beta0[bb] = nb;
            S.sc[1 * B + bb] = 1.0 / nb;
        }
        if (threadIdx.x == 0) S.ticket[0] = 0;
    }
}

// ---- Lanczos on B: w = B q_j, alpha_j = <q_j, w> ----------------------------
template <bool kBilinear>
__global__ void __launch_bounds__(kTkThreads) k_tke_spmv_alpha(int n, int B, int j, const int* __restrict__ rowptr,
                                                              const int* __restrict__ col,
                                                              const double* __restrict__ val,
                                                              const double* __restrict__ bdiag, const cd* rj,
                                                              cd* __restrict__ w, TkScal S) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (b < B) {
        const double sc = S.sc[(size_t)j * B + b];
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t xi = (size_t)row * B + b;
            const cd xr = rj[xi];
            cd a = cscale(xr, bdiag[row]);
            for (int q = rowptr[row]; q < rowptr[row + 1]; ++q)
                a = cadd(a, cscale(rj[(size_t)col[q] * B + b], val[q]));
            const cd u = cscale(a, sc);
            w[xi] = u;
            const cd qv = cscale(xr, sc);
            const cd pr = kBilinear ? cmul(qv, u) : cmul(cconj(qv), u);
            v[0] += pr.x;
            v[1] += pr.y;
        }
    }
    if (tk_partials<2>(v, b, B, S.partial, &S.ticket[1])) {
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x)
            S.alpha[(size_t)j * B + bb] =
                cmk(tk_sum(S.partial, gridDim.x, B, bb, 0), tk_sum(S.partial, gridDim.x, B, bb, 1));
        if (threadIdx.x == 0) S.ticket[1] = 0;
    }
}

// r_{j+1} = w - alpha_j q_j - beta_{j-1} q_{j-1}; beta_j = ||r_{j+1}||, sc_{j+1}
__global__ void __launch_bounds__(kTkThreads) k_tke_axpy_norm(int n, int B, int j, const cd* __restrict__ w,
                                                             const cd* rj, const cd* rjm, cd* rjp, TkScal S) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (b < B) {
        const cd a = S.alpha[(size_t)j * B + b];
        const double scj = S.sc[(size_t)j * B + b];
        const cd bm = j > 1 ? S.beta[(size_t)(j - 1) * B + b] : cmk(0.0, 0.0);
        const double scm = j > 1 ? S.sc[(size_t)(j - 1) * B + b] : 0.0;
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t xi = (size_t)row * B + b;
            cd r = csub(w[xi], cmul(a, cscale(rj[xi], scj)));
            if (j > 1) r = csub(r, cmul(bm, cscale(rjm[xi], scm)));
            rjp[xi] = r;
            v[0] += cabs2(r);
        }
    }
    if (tk_partials<1>(v, b, B, S.partial, &S.ticket[2])) {
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x) {
            double nb = sqrt(tk_sum(S.partial, gridDim.x, B, bb, 0));
            if (!isfinite(nb)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            const double scale = sqrt(cabs2(S.alpha[(size_t)j * B + bb])) +
                                 (j > 1 ? S.beta[(size_t)(j - 1) * B + bb].x : 0.0);
            if (nb <= kBreakdownRel * scale) nb = 0.0;
            S.beta[(size_t)j * B + bb] = cmk(nb, 0.0);
            S.sc[(size_t)(j + 1) * B + bb] = nb > 0.0 ? 1.0 / nb : 0.0;
        }
        if (threadIdx.x == 0) S.ticket[2] = 0;
    }
}

// ||B q_{m+1}||
__global__ void __launch_bounds__(kTkThreads) k_tke_nav(int n, int B, int j, const int* __restrict__ rowptr,
                                                       const int* __restrict__ col, const double* __restrict__ val,
                                                       const double* __restrict__ bdiag, const cd* rj, TkScal S) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (b < B) {
        const double sc = S.sc[(size_t)j * B + b];
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t xi = (size_t)row * B + b;
            cd a = cscale(rj[xi], bdiag[row]);
            for (int q = rowptr[row]; q < rowptr[row + 1]; ++q)
                a = cadd(a, cscale(rj[(size_t)col[q] * B + b], val[q]));
            v[0] += cabs2(cscale(a, sc));
        }
    }
    if (tk_partials<1>(v, b, B, S.partial, &S.ticket[3])) {
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x) S.nav[bb] = sqrt(tk_sum(S.partial, gridDim.x, B, bb, 0));
        if (threadIdx.x == 0) S.ticket[3] = 0;
    }
}

// exp(tau Tbar_B) per trajectory (one CTA each): combine weights and the B
// part's EXPOKIT estimate, as k_pade_tk of the per-trajectory path.
__global__ void k_tke_pade(int mb, int p, int B, double tau_im, int norm_mode, TkScal S) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int b = blockIdx.x;
    const int L = mb + p;
    cd* A = reinterpret_cast<cd*>(smem);
    const cd tau = cmk(0.0, tau_im);
    for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
        const int i = e / L, jj = e % L;
        cd v = cmk(0.0, 0.0);
        if (i < mb && jj < mb) {
            if (i == jj) v = S.alpha[(size_t)(i + 1) * B + b];
            else if (jj == i + 1) v = S.beta[(size_t)(i + 1) * B + b];
            else if (i == jj + 1) v = S.beta[(size_t)(jj + 1) * B + b];
        } else if ((i == 0 && jj == mb) || (i >= mb && jj == i + 1)) {
            v = cmk(1.0, 0.0);
        }
        A[e] = cmul(tau, v);
    }
    __syncthreads();
    cd* E = nullptr;
    const int s = pade_exp_sm(L, norm_mode, smem, &E);
    if (s < 0) {
        if (threadIdx.x == 0) atomicCAS(S.status, 0, (s == -1) ? DQ_ERR_SCALING : DQ_ERR_SINGULAR);
        return;
    }
    const double b0 = S.beta0[b];
    if (threadIdx.x < mb)
        S.yt[(size_t)(threadIdx.x + 1) * B + b] =
            cscale(E[threadIdx.x * L + L - 1], b0 * S.sc[(size_t)(threadIdx.x + 1) * B + b]);
    if (threadIdx.x == 0)
        S.kerr[b] = expokit_error(S.beta[(size_t)mb * B + b].x, S.nav[b], E[(mb - 1) * L + mb],
                                  E[(mb - 1) * L + mb + 1]);
}

// psi = sum_j yt_j r_j + Taylor sum; norm and error estimate (added to erracc)
__global__ void __launch_bounds__(kTkThreads) k_tke_combine(int n, int B, int mb, const cd* __restrict__ Q,
                                                           const cd* __restrict__ acc, cd* __restrict__ psi,
                                                           double* erracc, TkScal S) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    const size_t se = (size_t)n * B;
    double v[1] = {0.0};
    if (b < B) {
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t xi = (size_t)row * B + b;
            cd k = cmul(Q[se + xi], S.yt[(size_t)B + b]);
            for (int j = 2; j <= mb; ++j) k = cadd(k, cmul(Q[(size_t)j * se + xi], S.yt[(size_t)j * B + b]));
            const cd u = cadd(k, acc[xi]);
            psi[xi] = u;
            v[0] += cabs2(u);
        }
    }
    if (tk_partials<1>(v, b, B, S.partial, &S.ticket[4])) {
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x) {
            const double nrm = sqrt(tk_sum(S.partial, gridDim.x, B, bb, 0));
            if (!(nrm > 0.0) || !isfinite(nrm)) atomicCAS(S.status, 0, DQ_ERR_NAN);
            S.norm[bb] = nrm;
            double est = S.kerr[bb] + fabs(1.0 - nrm);   // taylorKrylovClass.cu:417-434
            if (est < 1.110223e-16) est = 1.110223e-16;
            S.err[bb] = est;
            erracc[bb] += est;
        }
        if (threadIdx.x == 0) S.ticket[4] = 0;
    }
}

// psi /= ||psi||; corr[step+1] += sum_b <psi0|psi_b>; ipr[step+1] += sum_b 1 / sum |psi_b|^4
__global__ void __launch_bounds__(kTkThreads) k_tke_observe(int n, int B, const cd* __restrict__ psi0, cd* psi,
                                                           cd* corr_pt, double* ipr_pt, TkScal S) {
    const int b = blockIdx.y * blockDim.x + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (b < B) {
        const double inv = 1.0 / S.norm[b];
        for (int row = blockIdx.x; row < n; row += gridDim.x) {
            const size_t xi = (size_t)row * B + b;
            const cd u = cscale(psi[xi], inv);
            psi[xi] = u;
            const cd c = cmul(cconj(psi0[row]), u);
            v[0] += c.x;
            v[1] += c.y;
            const double a = cabs2(u);
            v[2] += a * a;
        }
    }
    if (tk_partials<3>(v, b, B, S.partial, &S.ticket[5])) {
        __shared__ double scratch[32];
        double cr = 0.0, ci = 0.0, ip = 0.0;
        for (int bb = threadIdx.x; bb < B; bb += blockDim.x) {
            cr += tk_sum(S.partial, gridDim.x, B, bb, 0);
            ci += tk_sum(S.partial, gridDim.x, B, bb, 1);
            ip += 1.0 / tk_sum(S.partial, gridDim.x, B, bb, 2);
        }
        cr = block_sum(cr, scratch);
        ci = block_sum(ci, scratch);
        ip = block_sum(ip, scratch);
        if (threadIdx.x == 0) {
            corr_pt->x += cr;
            corr_pt->y += ci;
            if (ipr_pt) *ipr_pt += ip;
            S.ticket[5] = 0;
        }
    }
}

// pops_row[i] += sum_b |psi_ib|^2 (warp per row, fixed lane order)
__global__ void k_tke_pops(int n, int B, const cd* __restrict__ psi, double* __restrict__ pops_row) {
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < n; row += gridDim.x * wpb) {
        double s = 0.0;
        for (int b = lane; b < B; b += 32) s += cabs2(psi[(size_t)row * B + b]);
        s = warp_sum(s);
        if (lane == 0) pops_row[row] += s;
    }
}

__global__ void k_tke_set_psi0(int n, int B, const cd* __restrict__ psi0, cd* __restrict__ psi) {
    const size_t total = (size_t)n * B;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x)
        psi[x] = psi0[x / B];
}

// initial records: pops[0] += B |psi0|^2, corr[0] += B <psi0|psi0> (B with a
// separate bra), ipr[0] += B / sum |psi0|^4
__global__ void k_tke_init_obs(int n, int B, const cd* __restrict__ psi0, double* pops, cd* corr, double* ipr,
                               int unit0) {
    __shared__ double scratch[32];
    double s2 = 0.0, s4 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = cabs2(psi0[i]);
        pops[i] += (double)B * a;
        s2 += a;
        s4 += a * a;
    }
    s2 = block_sum(s2, scratch);
    s4 = block_sum(s4, scratch);
    if (threadIdx.x == 0) {
        corr[0].x += (double)B * (unit0 ? 1.0 : s2);
        if (ipr) ipr[0] += (double)B / s4;
    }
}

// ---------------------------------------------------------------------------
#define DQ_CU(call)                                                     \
    do {                                                                \
        dq_status _s = check_cuda(c, (call), #call);                    \
        if (_s != DQ_OK) return _s;                                     \
    } while (0)

void tk_ensemble_free(dq_ctx* c) {
    TkEnsemble* t = c->tke;
    if (!t) return;
    cudaFree(t->eps); cudaFree(t->deps); cudaFree(t->diag); cudaFree(t->psi); cudaFree(t->Q); cudaFree(t->x2);
    cudaFree(t->acc); cudaFree(t->w); cudaFree(t->scal_mem); cudaFree(t->s.ticket); cudaFree(t->s.status);
    delete t;
    c->tke = nullptr;
}

static dq_status tk_ensemble_alloc(dq_ctx* c) {
    const int n = c->n, B = c->cfg.n_traj, mb = c->tk_m;
    TkEnsemble* t = new TkEnsemble();
    c->tke = t;
    t->B = B;
    t->mb_alloc = mb;
    const size_t se = (size_t)n * B;
    DQ_CU(cudaMalloc(&t->eps, sizeof(double) * se));
    DQ_CU(cudaMalloc(&t->deps, sizeof(double) * se));
    DQ_CU(cudaMalloc(&t->diag, sizeof(double) * se));
    DQ_CU(cudaMalloc(&t->psi, sizeof(cd) * se));
    DQ_CU(cudaMalloc(&t->Q, sizeof(cd) * se * (mb + 2)));
    DQ_CU(cudaMemsetAsync(t->Q, 0, sizeof(cd) * se * (mb + 2), c->stream));
    DQ_CU(cudaMalloc(&t->x2, sizeof(cd) * se * 2));
    DQ_CU(cudaMalloc(&t->acc, sizeof(cd) * se));
    DQ_CU(cudaMalloc(&t->w, sizeof(cd) * se));
    const size_t LB = (size_t)kMaxL * B;
    const size_t total = LB * 2 * 2 + LB + LB * 2 + 5 * (size_t)B + (size_t)kTkRowGroups * B * 3;
    DQ_CU(cudaMalloc(&t->scal_mem, sizeof(double) * total));
    DQ_CU(cudaMemsetAsync(t->scal_mem, 0, sizeof(double) * total, c->stream));
    double* q = t->scal_mem;
    t->s.alpha = reinterpret_cast<cd*>(q); q += LB * 2;
    t->s.beta = reinterpret_cast<cd*>(q); q += LB * 2;
    t->s.sc = q; q += LB;
    t->s.yt = reinterpret_cast<cd*>(q); q += LB * 2;
    t->s.beta0 = q; q += B;
    t->s.nav = q; q += B;
    t->s.kerr = q; q += B;
    t->s.norm = q; q += B;
    t->s.err = q; q += B;
    t->s.partial = q;
    DQ_CU(cudaMalloc(&t->s.ticket, sizeof(unsigned int) * 8));
    DQ_CU(cudaMemsetAsync(t->s.ticket, 0, sizeof(unsigned int) * 8, c->stream));
    DQ_CU(cudaMalloc(&t->s.status, sizeof(int)));
    DQ_CU(cudaMemsetAsync(t->s.status, 0, sizeof(int), c->stream));
    DQ_CU(raise_smem_limit(k_tke_pade, (int)pade_smem_bytes(kMaxL)));
    return DQ_OK;
}

// Draws every trajectory's static energies, OU offsets and ZZ phases, sets
// every state to psi0 and adds the initial observable records (allocates the
// workspace on first use).
dq_status tk_ensemble_reset(dq_ctx* c) {
    dq_status st;
    if (c->tke && (c->tke->B != c->cfg.n_traj || c->tke->mb_alloc < c->tk_m)) tk_ensemble_free(c);
    if (!c->tke && (st = tk_ensemble_alloc(c))) return st;
    TkEnsemble* t = c->tke;
    const int n = c->n, B = t->B;
    const int blocks = std::min(n, 148 * 8);
    const int thr = std::min(256, ((B + 31) / 32) * 32);
    k_traj_init_b<<<blocks, thr, 0, c->stream>>>(n, B, c->traj0, c->cfg.seed, c->d_h0, c->d_static,
                                                 c->cfg.sigma_static, c->d_sigma, c->cfg.noise_model, t->eps, t->deps);
    k_tke_set_psi0<<<148 * 8, 256, 0, c->stream>>>(n, B, c->d_psi0, t->psi);
    k_tke_init_obs<<<1, 256, 0, c->stream>>>(n, B, c->d_psi0, c->d_pops, c->d_corr, c->ipr_on ? c->d_ipr : nullptr,
                                             c->d_bra != nullptr);
    DQ_CU(cudaMemsetAsync(t->s.status, 0, sizeof(int), c->stream));
    DQ_CU(cudaGetLastError());
    return DQ_OK;
}

// n_steps Taylor-Krylov steps of every trajectory (continuing from steps_done).
dq_status tk_ensemble_run(dq_ctx* c, int n_steps) {
    TkEnsemble* t = c->tke;
    const int n = c->n, B = t->B, p = c->tk_p, mb = c->tk_m, pe = c->cfg.pop_every;
    const dim3 grid(std::min(n, kTkRowGroups), (B + kTkThreads - 1) / kTkThreads);
    const size_t se = (size_t)n * B;
    cudaStream_t st = c->stream;
    const int ns = c->cfg.ka_substeps > 0 ? c->cfg.ka_substeps : 1;
    const double subdt = c->cfg.dt / (double)ns, sqrt_subdt = sqrt(subdt);
    ZZParams zz;
    if (c->cfg.noise_model == DQ_NOISE_ZZ) {
        zz.n_osc = c->zz_n_osc;
        zz.omega = c->d_zz_omega;
        zz.coeff = c->d_zz_coeff;
        zz.dt = c->cfg.dt;
    }
    const bool bil = c->cfg.dot_mode == DQ_DOT_BILINEAR;
    for (int k = 0; k < n_steps; ++k) {
        const int step = c->steps_done + k;
        k_tke_noise<<<grid, kTkThreads, 0, st>>>(n, B, c->traj0, step, c->cfg.noise_model, ns, subdt, sqrt_subdt,
                                                 c->cfg.seed, c->d_sigma, c->d_invtau, c->d_coeff, zz, t->eps,
                                                 t->deps, t->diag);
        const cd* x = t->psi;
        for (int kk = 1; kk <= p; ++kk) {
            cd* y = (kk == p) ? t->Q + se : t->x2 + (size_t)(kk & 1) * se;
            k_tke_power<<<grid, kTkThreads, 0, st>>>(n, B, kk, p, c->d_rowptr, c->d_col, c->d_val, t->diag, x, y,
                                                     t->acc, kk < p ? c->tk_coef[kk] : cmk(0.0, 0.0), t->s);
            x = y;
        }
        for (int j = 1; j <= mb; ++j) {
            const cd* rj = t->Q + (size_t)j * se;
            const cd* rjm = j > 1 ? t->Q + (size_t)(j - 1) * se : nullptr;
            cd* rjp = t->Q + (size_t)(j + 1) * se;
            if (bil)
                k_tke_spmv_alpha<true><<<grid, kTkThreads, 0, st>>>(n, B, j, c->d_tk_rowptr, c->d_tk_col,
                                                                    c->d_tk_val, c->d_tk_diag, rj, t->w, t->s);
            else
                k_tke_spmv_alpha<false><<<grid, kTkThreads, 0, st>>>(n, B, j, c->d_tk_rowptr, c->d_tk_col,
                                                                     c->d_tk_val, c->d_tk_diag, rj, t->w, t->s);
            k_tke_axpy_norm<<<grid, kTkThreads, 0, st>>>(n, B, j, t->w, rj, rjm, rjp, t->s);
        }
        k_tke_nav<<<grid, kTkThreads, 0, st>>>(n, B, mb + 1, c->d_tk_rowptr, c->d_tk_col, c->d_tk_val, c->d_tk_diag,
                                               t->Q + (size_t)(mb + 1) * se, t->s);
        k_tke_pade<<<B, 256, pade_smem_bytes(mb + p), st>>>(mb, p, B, c->tau_im, c->cfg.norm_mode, t->s);
        k_tke_combine<<<grid, kTkThreads, 0, st>>>(n, B, mb, t->Q, t->acc, t->psi, c->d_erracc, t->s);
        k_tke_observe<<<grid, kTkThreads, 0, st>>>(n, B, corr_bra(c), t->psi, c->d_corr + step + 1,
                                                   c->ipr_on ? c->d_ipr + step + 1 : nullptr, t->s);
        if ((step + 1) % pe == 0)
            k_tke_pops<<<std::max(1, std::min(148 * 4, (n + 7) / 8)), 256, 0, st>>>(
                n, B, t->psi, c->d_pops + (size_t)((step + 1) / pe) * n);
        DQ_CU(cudaGetLastError());
    }
    DQ_CU(cudaStreamSynchronize(st));
    int status = 0;
    DQ_CU(cudaMemcpy(&status, t->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    c->steps_done += n_steps;
    if (status) return read_status(c, status, "run (Taylor-Krylov)");
    return DQ_OK;
}

// States of the ensemble, [traj][site].
dq_status tk_ensemble_states(dq_ctx* c, dq_cdouble* out) {
    TkEnsemble* t = c->tke;
    const int n = c->n, B = t->B;
    std::vector<cd> h((size_t)n * B);
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(h.data(), t->psi, sizeof(cd) * h.size(), cudaMemcpyDeviceToHost));
    for (int b = 0; b < B; ++b)
        for (int i = 0; i < n; ++i) {
            out[(size_t)b * n + i].re = h[(size_t)i * B + b].x;
            out[(size_t)b * n + i].im = h[(size_t)i * B + b].y;
        }
    return DQ_OK;
}

}  // namespace dq
