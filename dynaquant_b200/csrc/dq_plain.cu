// dq_plain.cu — the plain FP64 per-trajectory form: the drop-in for one
// reference time step (propagate.cu:211-254).
//
// Per step, all on the context's stream, no host synchronisation:
//   k_noise          OU / Gaussian update of this trajectory's diagonal
//                    (gpuSysHelper.cu:32-128, Philox instead of cuRAND)
//   m x { k_spmv_alpha, k_axpy_norm }
//                    one Lanczos iteration (lanczosClass.cu:405-526): the
//                    SpMV, alpha, both axpys, beta and the scaling collapse
//                    into two kernels; the residual is stored unnormalised
//                    with a per-slab scale, so no third pass is needed
//   k_spmv_norm      ||H q_{m+1}|| (lanczosClass.cu:537-570)
//   k_pade           exp(tau Tbar), weights, EXPOKIT error (one CTA)
//   k_combine        psi = V y, ||psi||^2 (propStep.cu:31-44)
//   k_renorm         psi /= ||psi|| (+ population / correlation sums)
// Cross-block reductions use the last-block ticket, so every reduction is
// deterministic and costs no extra launch.
#include <cstdio>
#include <mutex>

#include <algorithm>

#include "dq_internal.h"
#include "dq_rng.cuh"
#include <cuda.h>

namespace dq {

__global__ void k_traj_init_plain(int n, int n_traj, int traj0, uint64_t seed, const double* __restrict__ h0,
                                  const double* __restrict__ static_eps, double sigma_static,
                                  const double* __restrict__ sigma, int noise, double* __restrict__ eps,
                                  double* __restrict__ deps) {
    size_t total = (size_t)n * n_traj;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        int t = traj0 + (int)(x / n), i = (int)(x % n);   // t: trajectory index of the whole ensemble
        double e;
        if (static_eps) e = static_eps[i];
        else e = __dadd_rn(__dmul_rn(sigma_static, normal(seed, P_STATIC, t, 0, i, 0)), h0[i]);
        eps[x] = e;
        deps[x] = (noise == DQ_NOISE_OU) ? __dmul_rn(sigma[i], normal(seed, P_OU_INIT, t, 0, i, 0)) : 0.0;
    }
}

// ZZ diagonal of one trajectory at step: eps + sum_osc c cos(omega t + phi)
// (gpuSysHelper.cu:134-177), summed as two fused multiply-adds per oscillator
// with the step's factors (c cos(omega t), c sin(omega t)) shared in shared
// memory; the phases are drawn from Philox here, one per (site, osc)
__global__ void k_noise_zz(int n, int traj, int step, uint64_t seed, ZZParams zz, const double* __restrict__ eps,
                           double* __restrict__ diag, PlainScalars* ps) {
    __shared__ double ccw[kMaxZZOsc], csw[kMaxZZOsc];
    if (blockIdx.x == 0 && threadIdx.x == 0) ps->sc[1] = 1.0;   // q_1 = psi_in
    for (int o = threadIdx.x; o < zz.n_osc; o += blockDim.x)
        zz_factors(zz.omega[o], zz.coeff[o], step, zz.dt, ccw[o], csw[o]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0;
    for (int o = 0; o < zz.n_osc; ++o)
        acc = zz_acc(acc, ccw[o], csw[o], zz_phase(seed, (uint32_t)traj, (uint32_t)i, (uint32_t)o));
    diag[i] = __dadd_rn(acc, eps[i]);
}

__global__ void k_noise(int n, int traj, int step, int noise, int ns, double subdt, double sqrt_subdt,
                        uint64_t seed, const double* __restrict__ sigma, const double* __restrict__ invtau,
                        const double* __restrict__ coeff, const double* __restrict__ eps,
                        double* __restrict__ deps, double* __restrict__ diag, PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) ps->sc[1] = 1.0;   // q_1 = psi_in
    if (i >= n) return;
    if (noise == DQ_NOISE_OU) {
        double cur = ou_update(deps[i], invtau[i], coeff[i], subdt, sqrt_subdt, ns, seed, traj, step, i);
        deps[i] = cur;
        diag[i] = __dadd_rn(cur, eps[i]);
    } else if (noise == DQ_NOISE_GAUSS) {
        double xi = normal(seed, P_GAUSS, traj, step, i, 0);
        diag[i] = __dadd_rn(__dmul_rn(xi, sigma[i]), eps[i]);
    } else {
        diag[i] = eps[i];
    }
}

// Reduce 2 doubles per block into partial[2*blockIdx]; the last block sums
// the partials in block order into out2 (and returns true in that block).
__device__ __forceinline__ bool reduce2_last(double a, double b, double* partial, unsigned int* ticket,
                                             double* out2) {
    __shared__ double scratch[kPlainThreads / 32];
    double ra = block_sum(a, scratch);
    double rb = block_sum(b, scratch);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = ra; partial[2 * blockIdx.x + 1] = rb; }
    bool last = last_block_ticket(ticket, gridDim.x);
    if (last) {
        // every thread sums a strided share, then a fixed-order block sum
        double sa = 0.0, sb = 0.0;
        for (unsigned int k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
            sa += __ldcg(&partial[2 * k]);
            sb += __ldcg(&partial[2 * k + 1]);
        }
        sa = block_sum(sa, scratch);
        sb = block_sum(sb, scratch);
        if (threadIdx.x == 0) {
            out2[0] = sa;
            out2[1] = sb;
            *ticket = 0;
        }
        __syncthreads();
    }
    return last;
}

// w = H q_j (q_j = sc_j * r_j), alpha_j = <q_j, w> (bilinear or Hermitian)
template <bool kBilinear>
__global__ void __launch_bounds__(kPlainThreads) k_spmv_alpha(int n, int j, const int* __restrict__ rowptr,
                                                             const int* __restrict__ col,
                                                             const double* __restrict__ val,
                                                             const double* __restrict__ diag, const cd* rj,
                                                             cd* __restrict__ w, double* partial,
                                                             PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ar = 0.0, ai = 0.0;
    if (i < n) {
        const double sc = ps->sc[j];
        cd x = rj[i];
        cd acc = cscale(x, diag[i]);
        for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) acc = cadd(acc, cscale(rj[col[p]], val[p]));
        cd u = cscale(acc, sc);
        w[i] = u;
        cd q = cscale(x, sc);
        cd pr = kBilinear ? cmul(q, u) : cmul(cconj(q), u);
        ar = pr.x;
        ai = pr.y;
    }
    __shared__ double out2[2];
    if (reduce2_last(ar, ai, partial, &ps->ticket[0], out2) && threadIdx.x == 0) {
        ps->alpha[j] = cmk(out2[0], out2[1]);
    }
}

// r_{j+1} = w - alpha_j q_j - beta_{j-1} q_{j-1};  beta_j = ||r_{j+1}||
__global__ void __launch_bounds__(kPlainThreads) k_axpy_norm(int n, int j, const cd* __restrict__ w,
                                                            const cd* rj, const cd* rjm, cd* rjp,
                                                            double* partial, PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < n) {
        const cd a = ps->alpha[j];
        cd r = csub(w[i], cmul(a, cscale(rj[i], ps->sc[j])));
        if (j > 1) r = csub(r, cmul(ps->beta[j - 1], cscale(rjm[i], ps->sc[j - 1])));
        rjp[i] = r;
        nn = cabs2(r);
    }
    __shared__ double out2[2];
    if (reduce2_last(nn, 0.0, partial, &ps->ticket[1], out2) && threadIdx.x == 0) {
        double b = sqrt(out2[0]);
        if (!isfinite(b)) atomicCAS(&ps->status, 0, DQ_ERR_NAN);
        // lucky breakdown: the Krylov space is invariant, q_{j+1} = 0 makes
        // the remaining block of T decouple and the result exact
        const double scale = sqrt(cabs2(ps->alpha[j])) + (j > 1 ? ps->beta[j - 1].x : 0.0);
        if (b <= kBreakdownRel * scale) b = 0.0;
        ps->beta[j] = cmk(b, 0.0);
        ps->sc[j + 1] = b > 0.0 ? 1.0 / b : 0.0;
    }
}

// Full reorthogonalisation (Hermitian dot, cfg.reorth): h_k = <q_k, r_{j+1}>
// for one k per launch, then r_{j+1} -= sum_k h_k q_k and beta_j, sc_{j+1}
// from the new norm (classical Gram-Schmidt once, FP64).
__global__ void __launch_bounds__(kPlainThreads) k_reorth_dot(int n, int k, const cd* __restrict__ xk,
                                                             const cd* __restrict__ r, double* partial,
                                                             PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double ar = 0.0, ai = 0.0;
    if (i < n) {
        const cd p = cmul(cconj(cscale(xk[i], ps->sc[k])), r[i]);
        ar = p.x;
        ai = p.y;
    }
    __shared__ double out2[2];
    if (reduce2_last(ar, ai, partial, &ps->ticket_r[0], out2) && threadIdx.x == 0) ps->h[k] = cmk(out2[0], out2[1]);
}

__global__ void __launch_bounds__(kPlainThreads) k_reorth_apply(int n, int j, const cd* __restrict__ x1,
                                                               const cd* __restrict__ Q, cd* r, double* partial,
                                                               PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < n) {
        cd v = r[i];
        for (int k = 1; k <= j; ++k) {
            const cd x = k == 1 ? x1[i] : Q[(size_t)k * n + i];
            v = csub(v, cmul(ps->h[k], cscale(x, ps->sc[k])));
        }
        r[i] = v;
        nn = cabs2(v);
    }
    __shared__ double out2[2];
    if (reduce2_last(nn, 0.0, partial, &ps->ticket_r[1], out2) && threadIdx.x == 0) {
        double b = sqrt(out2[0]);
        if (!isfinite(b)) atomicCAS(&ps->status, 0, DQ_ERR_NAN);
        const double scale = sqrt(cabs2(ps->alpha[j])) + (j > 1 ? ps->beta[j - 1].x : 0.0);
        if (b <= kBreakdownRel * scale) b = 0.0;
        ps->beta[j] = cmk(b, 0.0);
        ps->sc[j + 1] = b > 0.0 ? 1.0 / b : 0.0;
    }
}

// ||H q_{m+1}||
__global__ void __launch_bounds__(kPlainThreads) k_spmv_norm(int n, int j, const int* __restrict__ rowptr,
                                                            const int* __restrict__ col,
                                                            const double* __restrict__ val,
                                                            const double* __restrict__ diag, const cd* rj,
                                                            double* partial, PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < n) {
        cd acc = cscale(rj[i], diag[i]);
        for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) acc = cadd(acc, cscale(rj[col[p]], val[p]));
        nn = cabs2(cscale(acc, ps->sc[j]));
    }
    __shared__ double out2[2];
    if (reduce2_last(nn, 0.0, partial, &ps->ticket[2], out2) && threadIdx.x == 0) ps->nav = sqrt(out2[0]);
}

__global__ void k_pade_plain(int m, double tau_im, int norm_mode, PlainScalars* ps, double* erracc, int traj) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ cd y[kMaxM];
    PadeOut o = pade_exp_tbar(m, ps->alpha, ps->beta, cmk(0.0, tau_im), norm_mode, y, smem);
    if (o.s < 0) {
        if (threadIdx.x == 0) atomicCAS(&ps->status, 0, (o.s == -1) ? DQ_ERR_SCALING : DQ_ERR_SINGULAR);
        return;
    }
    __syncthreads();
    if (threadIdx.x < m) ps->yt[threadIdx.x + 1] = cscale(y[threadIdx.x], ps->sc[threadIdx.x + 1]);
    if (threadIdx.x == 0) {
        ps->s = o.s;
        double est = expokit_error(ps->beta[m].x, ps->nav, o.e_m1_m, o.e_m1_mp1);
        ps->err = est;
        if (erracc) erracc[traj] += est;
    }
}

// psi_out = sum_j yt_j r_j, ||psi_out||^2
__global__ void __launch_bounds__(kPlainThreads) k_combine(int n, int m, const cd* psi_in, const cd* Q,
                                                          cd* __restrict__ out, double* partial,
                                                          PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < n) {
        cd acc = cmul(psi_in[i], ps->yt[1]);
        for (int j = 2; j <= m; ++j) acc = cadd(acc, cmul(Q[(size_t)j * n + i], ps->yt[j]));
        out[i] = acc;
        nn = cabs2(acc);
    }
    __shared__ double out2[2];
    if (reduce2_last(nn, 0.0, partial, &ps->ticket[0], out2) && threadIdx.x == 0) {
        double nrm = sqrt(out2[0]);
        ps->norm = nrm;
        ps->invnorm = 1. / nrm;
        if (!(nrm > 0.0) || !isfinite(nrm)) atomicCAS(&ps->status, 0, DQ_ERR_NAN);
    }
}

// psi_out *= 1/||psi_out||; optionally adds |psi|^2 into pops_row and
// <psi0|psi> into corr_pt.
__global__ void __launch_bounds__(kPlainThreads) k_renorm(int n, cd* out, const cd* __restrict__ psi0,
                                                         double* pops_row, cd* corr_pt, double* partial,
                                                         PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double cr = 0.0, ci = 0.0;
    if (i < n) {
        cd v = cscale(out[i], ps->invnorm);
        out[i] = v;
        if (pops_row) pops_row[i] += cabs2(v);
        if (corr_pt) {
            cd c = cmul(cconj(psi0[i]), v);
            cr = c.x;
            ci = c.y;
        }
    }
    if (corr_pt) {
        __shared__ double out2[2];
        if (reduce2_last(cr, ci, partial, &ps->ticket[3], out2) && threadIdx.x == 0) {
            corr_pt->x += out2[0];
            corr_pt->y += out2[1];
        }
    }
}

// pops_row += |psi0|^2; corr_pt += <psi0|psi0>, or += 1 with a separate bra
// (the reference stores M(0) = 1, spectraClass.cu:296)
__global__ void k_observe_initial(int n, const cd* __restrict__ psi0, double* pops_row, cd* corr_pt,
                                  double* partial, PlainScalars* ps, int unit0) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double cr = 0.0, ci = 0.0;
    if (i < n) {
        cd v = psi0[i];
        pops_row[i] += cabs2(v);
        cd c = cmul(cconj(v), v);
        cr = c.x;
        ci = c.y;
    }
    __shared__ double out2[2];
    if (reduce2_last(cr, ci, partial, &ps->ticket[3], out2) && threadIdx.x == 0) {
        corr_pt->x += unit0 ? 1.0 : out2[0];
        corr_pt->y += unit0 ? 0.0 : out2[1];
    }
}

// ---- Taylor-Krylov mode (taylorKrylovClass.cu:223-434) --------------------
// y = A x (A: the step's Hamiltonian); k < p: acc += c_k y (acc starts at
// psi_in for k = 1); k = p: tk_beta0 = ||y|| and sc_1 = 1 / tk_beta0, so the
// B Lanczos starts from q_1 = y / ||y||.
__global__ void __launch_bounds__(kPlainThreads) k_tk_power(int n, int k, int p, const int* __restrict__ rowptr,
                                                           const int* __restrict__ col,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ diag, const cd* x,
                                                           cd* __restrict__ y, cd* acc, cd coef, double* partial,
                                                           PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < n) {
        cd a = cscale(x[i], diag[i]);
        for (int q = rowptr[i]; q < rowptr[i + 1]; ++q) a = cadd(a, cscale(x[col[q]], val[q]));
        y[i] = a;
        if (k < p) acc[i] = cadd(k == 1 ? x[i] : acc[i], cmul(coef, a));
        nn = cabs2(a);
    }
    if (k < p) return;   // uniform over the grid
    __shared__ double out2[2];
    if (reduce2_last(nn, 0.0, partial, &ps->ticket[2], out2) && threadIdx.x == 0) {
        const double b = sqrt(out2[0]);
        if (!(b > 0.0) || !isfinite(b)) atomicCAS(&ps->status, 0, DQ_ERR_NAN);
        ps->tk_beta0 = b;
        ps->sc[1] = 1.0 / b;
    }
}

// exp(tau Tbar_B) of the (mB + p) augmented matrix (ones at (0, mB) and
// (mB+k, mB+k+1), gpuLanczosHelper.cu:14-60); combine weights from its last
// column scaled by ||A^p psi||; the EXPOKIT estimate of the B part.
__global__ void k_pade_tk(int mb, int p, double tau_im, int norm_mode, PlainScalars* ps) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int L = mb + p;
    cd* A = reinterpret_cast<cd*>(smem);
    const cd tau = cmk(0.0, tau_im);
    for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
        const int i = e / L, j = e % L;
        cd v = cmk(0.0, 0.0);
        if (i < mb && j < mb) {
            if (i == j) v = ps->alpha[i + 1];
            else if (j == i + 1) v = ps->beta[i + 1];
            else if (i == j + 1) v = ps->beta[j + 1];
        } else if ((i == 0 && j == mb) || (i >= mb && j == i + 1)) {
            v = cmk(1.0, 0.0);
        }
        A[e] = cmul(tau, v);
    }
    __syncthreads();
    cd* E = nullptr;
    const int s = pade_exp_sm(L, norm_mode, smem, &E);
    if (s < 0) {
        if (threadIdx.x == 0) atomicCAS(&ps->status, 0, (s == -1) ? DQ_ERR_SCALING : DQ_ERR_SINGULAR);
        return;
    }
    const double b0 = ps->tk_beta0;
    if (threadIdx.x < mb)
        ps->yt[threadIdx.x + 1] = cscale(E[threadIdx.x * L + L - 1], b0 * ps->sc[threadIdx.x + 1]);
    if (threadIdx.x == 0) {
        ps->s = s;
        ps->tk_kerr = expokit_error(ps->beta[mb].x, ps->nav, E[(mb - 1) * L + mb], E[(mb - 1) * L + mb + 1]);
    }
}

// psi_out = sum_j yt_j r_j (r_1 = A^p psi) + Taylor sum, ||psi_out||^2
__global__ void __launch_bounds__(kPlainThreads) k_combine_tk(int n, int mb, const cd* __restrict__ Q,
                                                             const cd* __restrict__ acc, cd* __restrict__ out,
                                                             double* partial, PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < n) {
        cd k = cmul(Q[(size_t)n + i], ps->yt[1]);
        for (int j = 2; j <= mb; ++j) k = cadd(k, cmul(Q[(size_t)j * n + i], ps->yt[j]));
        const cd v = cadd(k, acc[i]);
        out[i] = v;
        nn = cabs2(v);
    }
    __shared__ double out2[2];
    if (reduce2_last(nn, 0.0, partial, &ps->ticket[0], out2) && threadIdx.x == 0) {
        double nrm = sqrt(out2[0]);
        ps->norm = nrm;
        ps->invnorm = 1. / nrm;
        if (!(nrm > 0.0) || !isfinite(nrm)) atomicCAS(&ps->status, 0, DQ_ERR_NAN);
        // taylorKrylovClass.cu:417-434: the B part's estimate plus |1 - norm|
        double est = ps->tk_kerr + fabs(1.0 - nrm);
        if (est < 1.110223e-16) est = 1.110223e-16;
        ps->err = est;
    }
}

__global__ void k_tk_erracc(PlainScalars* ps, double* erracc, int traj) {
    if (threadIdx.x == 0) erracc[traj] += ps->err;
}

// ipr[rec] += 1 / sum_i |psi_i|^4 (systemClass.cu:2219-2257, FP64 sum)
__global__ void __launch_bounds__(kPlainThreads) k_ipr_plain(int n, const cd* __restrict__ psi, double* ipr_pt,
                                                            double* partial, PlainScalars* ps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double q = 0.0;
    if (i < n) {
        const double a = cabs2(psi[i]);
        q = a * a;
    }
    __shared__ double out2[2];
    if (reduce2_last(q, 0.0, partial, &ps->ticket[2], out2) && threadIdx.x == 0) *ipr_pt += 1.0 / out2[0];
}

// ------------------------------------------------------------------------
dq_status check_cuda(dq_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return DQ_OK;
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return DQ_ERR_CUDA;
}

dq_status read_status(dq_ctx* c, int code, const char* what) {
    if (code == DQ_OK) return DQ_OK;
    static const char* names[] = {"ok", "argument", "cuda", "Lanczos breakdown (beta_j == 0)",
                                  "non-finite value", "device wait timed out", "Padé scaling s >= 50",
                                  "call out of order", "Padé denominator singular"};
    c->err = std::string(what) + ": " + (code > 0 && code <= 8 ? names[code] : "unknown device error");
    return code;
}

#define DQ_CU(call)                                                     \
    do {                                                                \
        dq_status _s = check_cuda(c, (call), #call);                    \
        if (_s != DQ_OK) return _s;                                     \
    } while (0)

dq_status plain_alloc(dq_ctx* c) {
    const int n = c->n, B = c->cfg.n_traj, m = c->cfg.m;
    DQ_CU(cudaMalloc(&c->d_eps_p, sizeof(double) * (size_t)n * B));
    DQ_CU(cudaMalloc(&c->d_deps_p, sizeof(double) * (size_t)n * B));
    DQ_CU(cudaMalloc(&c->d_diag, sizeof(double) * n));
    DQ_CU(cudaMalloc(&c->d_Q, sizeof(cd) * (size_t)n * (m + 2)));
    DQ_CU(cudaMalloc(&c->d_w, sizeof(cd) * n));
    DQ_CU(cudaMalloc(&c->d_psi_a, sizeof(cd) * n));
    DQ_CU(cudaMalloc(&c->d_psi_b, sizeof(cd) * n));
    DQ_CU(cudaMalloc(&c->d_partial, sizeof(double) * 2 * kMaxPartials));
    DQ_CU(cudaMalloc(&c->d_ps, sizeof(PlainScalars)));
    DQ_CU(cudaMemsetAsync(c->d_ps, 0, sizeof(PlainScalars), c->stream));
    DQ_CU(cudaMemsetAsync(c->d_Q, 0, sizeof(cd) * (size_t)n * (m + 2), c->stream));
    // the limit is a per-function attribute shared by every context (and by
    // dq_krylov_step_static) on the device, so it is always set to the largest
    // Krylov dimension: a later context or call with a larger m never meets a
    // limit lowered by one with a smaller m
    (void)m;
    DQ_CU(raise_smem_limit(k_pade_plain, (int)pade_smem_bytes(kMaxL)));
    DQ_CU(raise_smem_limit(k_pade_tk, (int)pade_smem_bytes(kMaxL)));
    return DQ_OK;
}

void plain_free(dq_ctx* c) {
    cudaFree(c->d_eps_p); cudaFree(c->d_deps_p); cudaFree(c->d_diag); cudaFree(c->d_Q); cudaFree(c->d_w);
    cudaFree(c->d_psi_a); cudaFree(c->d_psi_b); cudaFree(c->d_partial); cudaFree(c->d_ps);
    c->d_eps_p = c->d_deps_p = c->d_diag = c->d_partial = nullptr;
    c->d_Q = c->d_w = c->d_psi_a = c->d_psi_b = nullptr;
    c->d_ps = nullptr;
}

dq_status plain_traj_init(dq_ctx* c) {
    const int n = c->n, B = c->cfg.n_traj;
    size_t total = (size_t)n * B;
    int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    k_traj_init_plain<<<blocks, 256, 0, c->stream>>>(n, B, c->traj0, c->cfg.seed, c->d_h0, c->d_static, c->cfg.sigma_static,
                                                     c->d_sigma, c->cfg.noise_model, c->d_eps_p, c->d_deps_p);
    DQ_CU(cudaGetLastError());
    DQ_CU(cudaMemsetAsync(&c->d_ps->status, 0, sizeof(int), c->stream));
    return DQ_OK;
}

dq_status plain_clear_observables(dq_ctx* c) {
    DQ_CU(cudaMemsetAsync(c->d_pops, 0, sizeof(double) * (size_t)c->n_rec_max * c->n, c->stream));
    DQ_CU(cudaMemsetAsync(c->d_corr, 0, sizeof(cd) * (size_t)(c->cfg.max_steps + 1), c->stream));
    DQ_CU(cudaMemsetAsync(c->d_erracc, 0, sizeof(double) * c->cfg.n_traj, c->stream));
    if (c->d_ipr) DQ_CU(cudaMemsetAsync(c->d_ipr, 0, sizeof(double) * (size_t)(c->cfg.max_steps + 1), c->stream));
    return DQ_OK;
}

// m Lanczos iterations on (rowptr, col, val, diag) from r_1 = x1 (q_1 =
// sc_1 x1), residuals r_2..r_{m+1} in slabs 2..m+1 of Q, then ||H q_{m+1}||.
static void plain_lanczos(dq_ctx* c, int m, const int* rowptr, const int* col, const double* val,
                          const double* diag, const cd* x1, cd* Q) {
    const int n = c->n, T = kPlainThreads, G = (n + T - 1) / T;
    cudaStream_t st = c->stream;
    for (int j = 1; j <= m; ++j) {
        const cd* rj = (j == 1) ? x1 : Q + (size_t)j * n;
        const cd* rjm = (j <= 1) ? nullptr : (j == 2 ? x1 : Q + (size_t)(j - 1) * n);
        cd* rjp = Q + (size_t)(j + 1) * n;
        if (c->cfg.dot_mode == DQ_DOT_BILINEAR)
            k_spmv_alpha<true><<<G, T, 0, st>>>(n, j, rowptr, col, val, diag, rj, c->d_w, c->d_partial, c->d_ps);
        else
            k_spmv_alpha<false><<<G, T, 0, st>>>(n, j, rowptr, col, val, diag, rj, c->d_w, c->d_partial, c->d_ps);
        k_axpy_norm<<<G, T, 0, st>>>(n, j, c->d_w, rj, rjm, rjp, c->d_partial, c->d_ps);
        if (c->cfg.reorth) {
            for (int k = 1; k <= j; ++k)
                k_reorth_dot<<<G, T, 0, st>>>(n, k, k == 1 ? x1 : Q + (size_t)k * n, rjp, c->d_partial, c->d_ps);
            k_reorth_apply<<<G, T, 0, st>>>(n, j, x1, Q, rjp, c->d_partial, c->d_ps);
        }
    }
    k_spmv_norm<<<G, T, 0, st>>>(n, m + 1, rowptr, col, val, diag, Q + (size_t)(m + 1) * n, c->d_partial, c->d_ps);
}

// Taylor-Krylov step after the noise update: p products with A (Taylor sum
// and A^p psi), mB Lanczos iterations on B from A^p psi, the augmented Padé,
// combine with the Taylor sum, renormalisation and observables.
static dq_status plain_tk_tail(dq_ctx* c, int traj, int step, const cd* psi_in, cd* psi_out, bool observe,
                               int rec) {
    const int n = c->n, p = c->tk_p, mb = c->tk_m, T = kPlainThreads, G = (n + T - 1) / T;
    cudaStream_t st = c->stream;
    const cd* x = psi_in;
    for (int k = 1; k <= p; ++k) {
        // the last product lands in slab 1 of the B basis
        cd* y = (k == p) ? c->d_tk_Q + n : c->d_tk_x + (size_t)(k & 1) * n;
        k_tk_power<<<G, T, 0, st>>>(n, k, p, c->d_rowptr, c->d_col, c->d_val, c->d_diag, x, y, c->d_tk_acc,
                                    k < p ? c->tk_coef[k] : cmk(0.0, 0.0), c->d_partial, c->d_ps);
        x = y;
    }
    plain_lanczos(c, mb, c->d_tk_rowptr, c->d_tk_col, c->d_tk_val, c->d_tk_diag, c->d_tk_Q + n, c->d_tk_Q);
    k_pade_tk<<<1, 256, pade_smem_bytes(mb + p), st>>>(mb, p, c->tau_im, c->cfg.norm_mode, c->d_ps);
    k_combine_tk<<<G, T, 0, st>>>(n, mb, c->d_tk_Q, c->d_tk_acc, psi_out, c->d_partial, c->d_ps);
    if (observe) k_tk_erracc<<<1, 32, 0, st>>>(c->d_ps, c->d_erracc, traj);
    double* prow = (observe && rec >= 0) ? c->d_pops + (size_t)rec * n : nullptr;
    cd* cpt = observe ? c->d_corr + (step + 1) : nullptr;
    k_renorm<<<G, T, 0, st>>>(n, psi_out, corr_bra(c), prow, cpt, c->d_partial, c->d_ps);
    if (observe && c->ipr_on) k_ipr_plain<<<G, T, 0, st>>>(n, psi_out, c->d_ipr + step + 1, c->d_partial, c->d_ps);
    DQ_CU(cudaGetLastError());
    return DQ_OK;
}

// One plain step.  observe: add the result into the observable sums; rec >= 0
// selects the population record to add |psi|^2 into (or -1).
dq_status plain_step(dq_ctx* c, int traj, int step, const cd* psi_in, cd* psi_out, bool observe, int rec) {
    const int n = c->n, m = c->cfg.m;
    const int T = kPlainThreads;
    const int G = (n + T - 1) / T;
    cudaStream_t st = c->stream;
    const int ns = c->cfg.ka_substeps > 0 ? c->cfg.ka_substeps : 1;
    const double subdt = c->cfg.dt / (double)ns;
    const double sqrt_subdt = sqrt(subdt);
    const double* eps = c->d_eps_p + (size_t)traj * n;
    double* deps = c->d_deps_p + (size_t)traj * n;
    if (c->cfg.noise_model == DQ_NOISE_ZZ) {
        ZZParams zz;
        zz.n_osc = c->zz_n_osc;
        zz.omega = c->d_zz_omega;
        zz.coeff = c->d_zz_coeff;
        zz.dt = c->cfg.dt;
        k_noise_zz<<<G, T, 0, st>>>(n, c->traj0 + traj, step, c->cfg.seed, zz, eps, c->d_diag, c->d_ps);
    } else {
        k_noise<<<G, T, 0, st>>>(n, c->traj0 + traj, step, c->cfg.noise_model, ns, subdt, sqrt_subdt, c->cfg.seed, c->d_sigma,
                                 c->d_invtau, c->d_coeff, eps, deps, c->d_diag, c->d_ps);
    }
    if (c->tk_p > 0) return plain_tk_tail(c, traj, step, psi_in, psi_out, observe, rec);
    plain_lanczos(c, m, c->d_rowptr, c->d_col, c->d_val, c->d_diag, psi_in, c->d_Q);
    k_pade_plain<<<1, 256, pade_smem_bytes(m + 2), st>>>(m, c->tau_im, c->cfg.norm_mode, c->d_ps,
                                                         observe ? c->d_erracc : nullptr, traj);
    k_combine<<<G, T, 0, st>>>(n, m, psi_in, c->d_Q, psi_out, c->d_partial, c->d_ps);
    double* prow = (observe && rec >= 0) ? c->d_pops + (size_t)rec * n : nullptr;
    cd* cpt = observe ? c->d_corr + (step + 1) : nullptr;
    k_renorm<<<G, T, 0, st>>>(n, psi_out, corr_bra(c), prow, cpt, c->d_partial, c->d_ps);
    if (observe && c->ipr_on) k_ipr_plain<<<G, T, 0, st>>>(n, psi_out, c->d_ipr + step + 1, c->d_partial, c->d_ps);
    DQ_CU(cudaGetLastError());
    return DQ_OK;
}

dq_status plain_observe_initial(dq_ctx* c) {
    const int n = c->n;
    const int G = (n + kPlainThreads - 1) / kPlainThreads;
    k_observe_initial<<<G, kPlainThreads, 0, c->stream>>>(n, c->d_psi0, c->d_pops, c->d_corr, c->d_partial, c->d_ps,
                                                          c->d_bra != nullptr);
    if (c->ipr_on) k_ipr_plain<<<G, kPlainThreads, 0, c->stream>>>(n, c->d_psi0, c->d_ipr, c->d_partial, c->d_ps);
    DQ_CU(cudaGetLastError());
    return DQ_OK;
}

}  // namespace dq

// ---------------------------------------------------------------------------
// Allocation-free variant of the plain step (dq_krylov_step_static).
//
// Some callers cannot allocate device memory at the point where they step a
// wavefunction: a host application that owns all device memory through its
// own pool and forbids cudaMalloc/cudaFree once its time loop runs (they can
// synchronise the device and fragment the pool), or code embedded in a
// framework that hands out only the buffers it manages.  This entry point
// needs no context and allocates nothing: its Krylov basis, residual,
// reduction partials and scalars live in one file-scope __device__ array of
// kStaticScratchBytes (16 MiB), which every GPU that loads the library holds
// until the process exits.  The caller passes the Hamiltonian (off-diagonal
// CSR + this step's diagonal) and the states, all in device memory.
//
// The array's host-side name is only a stand-in for a device address: on its
// first call on a device the entry point, with that device current, asks the
// runtime for the array's device address (cudaGetSymbolAddress) and raises
// the Padé kernel's shared-memory limit; that first call should come before
// any stream capture.  The address is kept per device together with the
// driver context it belongs to and looked up again when that context changed
// (after a cudaDeviceReset).  Every call on a device shares the one array and leaves
// the last call's contents in it (each call clears what must start at zero),
// so calls that overlap on the GPU (different streams, or host threads
// without ordering) race and must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace dq {
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
}  // namespace dq

static __device__ __align__(256) unsigned char g_dq_static_scratch[dq::kStaticScratchBytes];

namespace {

struct StaticScratch {
    bool init = false;
    unsigned char* ptr = nullptr;
    CUcontext ctx = nullptr;   // the context the address belongs to
};
constexpr int kMaxDevices = 64;
StaticScratch g_static_scratch[kMaxDevices];
std::mutex g_static_mu;

// The current driver context (the device's primary context after the
// runtime's set-up): a cudaDeviceReset replaces it, and with it the module
// and the array's device address, so a cached address is only valid for the
// context it was taken in.
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<Fn>(p);
        looked = true;
    }
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

void write_err(char* buf, int len, const char* msg) {
    if (buf && len > 0) snprintf(buf, (size_t)len, "%s", msg);
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

namespace dq {

// clears what a step expects at zero and starts the recurrence at q_1 =
// psi_in.  The status word is left as it is: a device error of a call that
// did not read it back stays recorded until a call with err_est reports it.
__global__ void k_static_begin(PlainScalars* ps) {
    if (threadIdx.x == 0) {
        ps->sc[1] = 1.0;
        ps->beta[0] = cmk(0.0, 0.0);
        for (int k = 0; k < 4; ++k) ps->ticket[k] = 0;
    }
}

// zeroes the status word once a call has read it back
__global__ void k_static_clear_status(PlainScalars* ps) {
    if (threadIdx.x == 0) ps->status = 0;
}

}  // namespace dq

extern "C" dq_status dq_krylov_step_static(int n, const int* rowptr, const int* col, const double* val,
                                           const double* diag, const dq_cdouble* psi_in, dq_cdouble* psi_out, int m,
                                           double dt, double hbar, int dot_mode, int norm_mode, void* stream,
                                           double* err_est, char* errbuf, int errbuf_len) {
    using namespace dq;
    if (n < 2 || m < 2 || m > kMaxM || m > n || !(dt > 0) || !rowptr || !col || !val || !diag || !psi_in ||
        !psi_out || psi_in == psi_out || (dot_mode != DQ_DOT_BILINEAR && dot_mode != DQ_DOT_HERMITIAN) ||
        (norm_mode != DQ_NORM_REAL_ONLY && norm_mode != DQ_NORM_COMPLEX)) {
        write_err(errbuf, errbuf_len, "krylov_step_static: invalid argument");
        return DQ_ERR_ARG;
    }
    const int T = kPlainThreads;
    const int G = (n + T - 1) / T;
    const size_t off_partial = align256(sizeof(PlainScalars));
    const size_t off_w = off_partial + align256(sizeof(double) * 2 * kMaxPartials);
    const size_t off_q = off_w + align256(sizeof(cd) * (size_t)n);
    const size_t need = off_q + sizeof(cd) * (size_t)n * (size_t)(m + 2);
    if (G > kMaxPartials || need > kStaticScratchBytes) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "krylov_step_static: n=%d, m=%d needs %zu bytes of scratch, above the %zu-byte static limit "
                 "((m+3)*n*16 bytes plus ~70 KB)",
                 n, m, need, kStaticScratchBytes);
        write_err(errbuf, errbuf_len, msg);
        return DQ_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        write_err(errbuf, errbuf_len, "krylov_step_static: no current CUDA device");
        return DQ_ERR_CUDA;
    }
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        StaticScratch& sc = g_static_scratch[dev];
        // NULL on a thread the runtime has not yet bound to the device's context:
        // then the address is simply looked up again below
        CUcontext ctx = current_context();
        if (!sc.init || ctx != sc.ctx) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_dq_static_scratch);
            if (e == cudaSuccess)
                e = raise_smem_limit(k_pade_plain, (int)pade_smem_bytes(kMaxL));
            if (e != cudaSuccess) {
                write_err(errbuf, errbuf_len, cudaGetErrorString(e));
                return DQ_ERR_CUDA;
            }
            sc.ptr = static_cast<unsigned char*>(p);
            sc.ctx = current_context();   // bound by the runtime call above
            sc.init = true;
        }
        base = sc.ptr;
    }
    PlainScalars* ps = reinterpret_cast<PlainScalars*>(base);
    double* partial = reinterpret_cast<double*>(base + off_partial);
    cd* w = reinterpret_cast<cd*>(base + off_w);
    cd* Q = reinterpret_cast<cd*>(base + off_q);
    const cd* pin = reinterpret_cast<const cd*>(psi_in);
    cd* pout = reinterpret_cast<cd*>(psi_out);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!(hbar > 0)) {
        const double pi = atan(1.0) * 4.0;
        hbar = (1 / 100.) * (1e15) * 1. / (299792548. * 2 * pi);   // cppUtility.cpp:19-22
    }
    const double tau_im = -dt / hbar;
    k_static_begin<<<1, 32, 0, st>>>(ps);
    for (int j = 1; j <= m; ++j) {
        const cd* rj = (j == 1) ? pin : Q + (size_t)j * n;
        const cd* rjm = (j <= 1) ? nullptr : (j == 2 ? pin : Q + (size_t)(j - 1) * n);
        cd* rjp = Q + (size_t)(j + 1) * n;
        if (dot_mode == DQ_DOT_BILINEAR)
            k_spmv_alpha<true><<<G, T, 0, st>>>(n, j, rowptr, col, val, diag, rj, w, partial, ps);
        else
            k_spmv_alpha<false><<<G, T, 0, st>>>(n, j, rowptr, col, val, diag, rj, w, partial, ps);
        k_axpy_norm<<<G, T, 0, st>>>(n, j, w, rj, rjm, rjp, partial, ps);
    }
    k_spmv_norm<<<G, T, 0, st>>>(n, m + 1, rowptr, col, val, diag, Q + (size_t)(m + 1) * n, partial, ps);
    k_pade_plain<<<1, 256, pade_smem_bytes(m + 2), st>>>(m, tau_im, norm_mode, ps, nullptr, 0);
    k_combine<<<G, T, 0, st>>>(n, m, pin, Q, pout, partial, ps);
    k_renorm<<<G, T, 0, st>>>(n, pout, nullptr, nullptr, nullptr, partial, ps);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        write_err(errbuf, errbuf_len, cudaGetErrorString(e));
        return DQ_ERR_CUDA;
    }
    if (err_est) {
        double hv[2] = {0.0, 0.0};
        int status = 0;
        e = cudaMemcpyAsync(&hv[0], &ps->err, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&status, &ps->status, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            write_err(errbuf, errbuf_len, cudaGetErrorString(e));
            return DQ_ERR_CUDA;
        }
        *err_est = hv[0];
        if (status) {
            k_static_clear_status<<<1, 32, 0, st>>>(ps);
            write_err(errbuf, errbuf_len,
                      "krylov_step_static: device reported an error (breakdown/NaN/Padé) in this call or in an "
                      "earlier one that passed err_est = NULL");
            return status;
        }
    }
    return DQ_OK;
}
