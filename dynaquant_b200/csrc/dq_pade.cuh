// dq_pade.cuh — exp(tau * Tbar) of the augmented Lanczos matrix for one
// trajectory, computed by one CTA in shared memory in FP64.
//
// Reference: padeClass.cu:206-487 (Padé(6,6) odd/even form, Zgemm/Zgeam +
// CULA Zgesv), padeClass.cu:585-706 (scaling by the row-sum infinity norm and
// repeated squaring), gpuLanczosHelper.cu:14-60 (augmented Tbar, EXPOKIT
// Theorem 1), padeClass.cu:750-782 (EXPOKIT Algorithm 3.2 error estimate).
// Here the whole chain runs in one CTA: the (m+2)^2 matrices live in shared
// memory, the quotient is solved by our own LU with partial pivoting, and
// nothing returns to the host.
#pragma once
#include "dq_common.cuh"

namespace dq {

constexpr int kMaxM = 32;            // Krylov dimension limit
constexpr int kMaxL = kMaxM + 2;     // augmented size
// beta_j <= kBreakdownRel * (|alpha_j| + beta_{j-1}) is treated as an exact
// (lucky) Lanczos breakdown: beta_j = 0 and q_{j+1} = 0 from there on.
constexpr double kBreakdownRel = 1e-12;

// Padé(6,6) coefficients c_k = c_{k-1} (p+1-k)/((2p+1-k) k), p = 6
// (padeClass.cu:161-168), evaluated in the same order on the host.
struct PadeCoeffs { double c[7]; };

__host__ __device__ inline PadeCoeffs pade_coeffs() {
    PadeCoeffs P;
    P.c[0] = 1.0;
    for (int k = 1; k <= 6; ++k) {
        double fk = (double)k;
        P.c[k] = P.c[k - 1] * (6.0 + 1. - fk) / ((2 * 6.0 + 1. - fk) * fk);
    }
    return P;
}

__host__ __device__ inline size_t pade_smem_bytes(int L) { return sizeof(cd) * 6 * (size_t)L * L + 64 * sizeof(double); }

// C = A * B (L x L row-major, shared memory), all threads of the CTA.
__device__ __forceinline__ void sm_matmul(int L, const cd* A, const cd* B, cd* C) {
    for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
        int i = e / L, j = e - i * L;
        cd s = cmk(0, 0);
        for (int k = 0; k < L; ++k) s = cadd(s, cmul(A[i * L + k], B[k * L + j]));
        C[e] = s;
    }
    __syncthreads();
}

struct PadeOut {
    int s;          // squarings (or -1 when s would reach 50, or -2 singular)
    cd e_m1_m;      // E(m-1, m)
    cd e_m1_mp1;    // E(m-1, m+1)
};

// E = exp(A) for the L x L complex matrix A held in the first L*L entries of
// smem_raw (6 L^2 complex + 64 doubles of shared memory): Padé(6,6) in the
// odd/even form with scaling by the row-sum infinity norm (norm_mode 0:
// |Re|-only sums as padeClass.cu:585-706; 1: complex modulus) and repeated
// squaring.  Returns the number of squarings s (or -1 when s would reach 50,
// -2 for a singular quotient) and sets *E_out to the result (A itself or the
// second buffer).  All threads of the CTA call it and all return s.
__device__ inline int pade_exp_sm(int L, int norm_mode, unsigned char* smem_raw, cd** E_out) {
    const int LL = L * L;
    cd* A = reinterpret_cast<cd*>(smem_raw);
    cd* A2 = A + LL;
    cd* A4 = A2 + LL;
    cd* A6 = A4 + LL;
    cd* U = A6 + LL;
    cd* D = U + LL;
    __shared__ int s_sh;
    __shared__ int piv_sh;
    __shared__ int fail_sh;

    const PadeCoeffs P = pade_coeffs();
    if (threadIdx.x == 0) fail_sh = 0;
    __syncthreads();

    // scaling: s = number of halvings until the row-sum norm is <= 0.5
    if (threadIdx.x < 32) {
        double mx = 0.0;
        for (int i = threadIdx.x; i < L; i += 32) {
            double rs = 0.0;
            for (int j = 0; j < L; ++j) {
                cd a = A[i * L + j];
                rs += norm_mode == 0 ? fabs(a.x) : sqrt(cabs2(a));
            }
            mx = fmax(mx, rs);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (threadIdx.x == 0) {
            int s = 0;
            double nrm = mx;
            while (nrm > 0.5 && s < 60) { nrm *= 0.5; s++; }
            s_sh = s;
        }
    }
    __syncthreads();
    const int s = s_sh;
    *E_out = A;
    if (s >= 50) return -1;
    if (s > 0) {
        double sc = ldexp(1.0, -s);
        for (int e = threadIdx.x; e < LL; e += blockDim.x) A[e] = cscale(A[e], sc);
        __syncthreads();
    }
    sm_matmul(L, A, A, A2);
    sm_matmul(L, A2, A2, A4);
    sm_matmul(L, A2, A4, A6);
    // odd part U = A (c1 I + c3 A^2 + c5 A^4); the bracket goes to D first
    for (int e = threadIdx.x; e < LL; e += blockDim.x) {
        int i = e / L, j = e - i * L;
        cd t = cadd(cscale(A2[e], P.c[3]), cscale(A4[e], P.c[5]));
        if (i == j) t.x += P.c[1];
        D[e] = t;
    }
    __syncthreads();
    sm_matmul(L, A, D, U);
    // even part V = c0 I + c2 A^2 + c4 A^4 + c6 A^6; D = V - U
    for (int e = threadIdx.x; e < LL; e += blockDim.x) {
        int i = e / L, j = e - i * L;
        cd t = cadd(cadd(cscale(A2[e], P.c[2]), cscale(A4[e], P.c[4])), cscale(A6[e], P.c[6]));
        if (i == j) t.x += P.c[0];
        D[e] = csub(t, U[e]);
    }
    __syncthreads();

    // LU with partial pivoting: D X = U, X overwrites U (stands in for
    // culaDeviceZgesv, padeClass.cu:715-745)
    for (int k = 0; k < L; ++k) {
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = k;
            for (int i = k + threadIdx.x; i < L; i += 32) {
                double v = cabs2(D[i * L + k]);
                if (v > best) { best = v; bi = i; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (threadIdx.x == 0) {
                piv_sh = bi;
                if (best == 0.0) fail_sh = 1;
            }
        }
        __syncthreads();
        if (fail_sh) break;
        const int p = piv_sh;
        if (p != k) {
            for (int j = threadIdx.x; j < L; j += blockDim.x) {
                cd t = D[k * L + j]; D[k * L + j] = D[p * L + j]; D[p * L + j] = t;
                t = U[k * L + j]; U[k * L + j] = U[p * L + j]; U[p * L + j] = t;
            }
            __syncthreads();
        }
        const cd inv = cdiv(cmk(1.0, 0.0), D[k * L + k]);
        // multipliers into column k below the pivot
        for (int i = k + 1 + threadIdx.x; i < L; i += blockDim.x) D[i * L + k] = cmul(D[i * L + k], inv);
        __syncthreads();
        const int rows = L - k - 1;
        for (int e = threadIdx.x; e < rows * L; e += blockDim.x) {
            int i = k + 1 + e / L, j = e % L;
            cd f = D[i * L + k];
            if (j > k) D[i * L + j] = csub(D[i * L + j], cmul(f, D[k * L + j]));
            U[i * L + j] = csub(U[i * L + j], cmul(f, U[k * L + j]));
        }
        __syncthreads();
    }
    if (fail_sh) return -2;
    for (int k = L - 1; k >= 0; --k) {
        const cd inv = cdiv(cmk(1.0, 0.0), D[k * L + k]);
        for (int j = threadIdx.x; j < L; j += blockDim.x) {
            cd acc = U[k * L + j];
            for (int c = k + 1; c < L; ++c) acc = csub(acc, cmul(D[k * L + c], U[c * L + j]));
            U[k * L + j] = cmul(acc, inv);
        }
        __syncthreads();
    }
    // E = I + 2X
    cd* E = A;
    for (int e = threadIdx.x; e < LL; e += blockDim.x) {
        int i = e / L, j = e - i * L;
        cd t = cscale(U[e], 2.0);
        if (i == j) t.x += 1.0;
        E[e] = t;
    }
    __syncthreads();
    cd* Tmp = A2;
    for (int k = 0; k < s; ++k) {
        sm_matmul(L, E, E, Tmp);
        cd* sw = E; E = Tmp; Tmp = sw;
    }
    *E_out = E;
    return s;
}

// Computes E = exp(tau * Tbar) for Tbar built from alpha[1..m], beta[1..m]
// (complex, shared or global), writes y[j] = E(j, 0) for j = 0..m-1 when
// y != nullptr.  norm_mode 0: reference |Re|-only row sums; 1: |.|.
// Returns in every thread.
__device__ inline PadeOut pade_exp_tbar(int m, const cd* alpha, const cd* beta, cd tau, int norm_mode,
                                        cd* y, unsigned char* smem_raw) {
    const int L = m + 2;
    const int LL = L * L;
    cd* A = reinterpret_cast<cd*>(smem_raw);
    // tau * Tbar (gpuLanczosHelper.cu:14-60, padeClass.cu:240-246)
    for (int e = threadIdx.x; e < LL; e += blockDim.x) {
        int i = e / L, j = e - i * L;
        cd t = cmk(0, 0);
        if (i < m && j < m) {
            if (i == j) t = alpha[i + 1];
            else if (j == i + 1) t = beta[i + 1];
            else if (i == j + 1) t = beta[j + 1];
        } else {
            if (i == 0 && j == m) t = cmk(1.0, 0.0);
            else if (i >= m && j >= m && i == j - 1) t = cmk(1.0, 0.0);
        }
        A[e] = cmul(tau, t);
    }
    __syncthreads();
    cd* E = nullptr;
    PadeOut out;
    out.s = pade_exp_sm(L, norm_mode, smem_raw, &E);
    if (out.s < 0) {
        out.e_m1_m = cmk(0, 0);
        out.e_m1_mp1 = cmk(0, 0);
        return out;
    }
    if (y) for (int j = threadIdx.x; j < m; j += blockDim.x) y[j] = E[j * L];
    out.e_m1_m = E[(m - 1) * L + m];
    out.e_m1_mp1 = E[(m - 1) * L + m + 1];
    __syncthreads();
    return out;
}

// EXPOKIT Algorithm 3.2 as padeClass.cu:750-782 with the floor of
// systemClass.cu:2075-2077.
__device__ __forceinline__ double expokit_error(double beta_m, double norm_av, cd e_m1_m, cd e_m1_mp1) {
    double hm = fabs(beta_m);
    double err1 = hm * sqrt(cabs2(e_m1_m));
    double err2 = hm * norm_av * sqrt(cabs2(e_m1_mp1));
    double est = (err1 > err2) ? err2 / (1 - err2 / err1) : err1;
    if (est < 1.110223e-16) est = 1.110223e-16;
    return est;
}

}  // namespace dq
