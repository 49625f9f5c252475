/*
 * dq_oracle.c — CPU FP64 restatement of DynaQuant's stochastic-Hamiltonian
 * Krylov propagator.  TEST INFRASTRUCTURE ONLY (the checker for the CUDA
 * path; never linked into the product library).
 *
 * Follows, in order (files of nicolassawaya/DynaQuant):
 *   gpuSysHelper.cu:73-128   OU (Kubo-Anderson) Euler-Maruyama noise update
 *   gpuSysHelper.cu:32-66    Gaussian (Haken-Strobl-Reineker) noise
 *   systemClass.cu:993-1036  OU parameters: coeff = sigma*sqrt(2/tau), subdt
 *   systemClass.cu:760-804   static disorder eps = H0_ii + N(0, sigma_static)
 *   lanczosClass.cu:397-531  Lanczos recurrence (q1 = psi, Q column 0 = 0)
 *   lanczosClass.cu:537-570  ||H q_{m+1}|| for the error estimate
 *   gpuLanczosHelper.cu:14-60 augmented tridiagonal T (EXPOKIT Theorem 1)
 *   padeClass.cu:161-168     Padé c_k
 *   padeClass.cu:206-487     Padé(6,6): A^2, A^4, A^6, odd/even parts, solve
 *   padeClass.cu:585-706     scaling (|Re| row sums) and squaring
 *   propStep.cu:31-44        psi_dest = Q[:,1..m] * E[0..m-1, 0]
 *   systemClass.cu:1771-1829 renormalisation
 *   padeClass.cu:750-782     EXPOKIT Algorithm 3.2 error estimate
 *   spectraClass.cu:510-571  correlation <psi0|psi(t)> (Zdotc)
 *   spectraClass.cu:621-626  inverse FFT (cuFFT INVERSE convention)
 *
 * Noise: the reference draws from cuRAND MRG32k3a / Boost mt19937 with
 * wall-clock seeds.  This restatement instead keys Philox4x32-10 (Salmon,
 * Moraes, Dror, Shaw, SC'11) by (seed, purpose, trajectory, step, site,
 * substep) and turns uniforms into normals by Box-Muller with its own log
 * (atanh series after binary range reduction) and sin/cos (octant reduction
 * plus Taylor polynomials), all with explicit fma so the CUDA kernels
 * reproduce every draw bit for bit.  Build with -ffp-contract=off.
 */
#include "dq_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* Philox4x32-10                                                       */
/* ------------------------------------------------------------------ */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void dqo_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += PHILOX_W0; k1 += PHILOX_W1; }
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* ------------------------------------------------------------------ */
/* Elementary functions written from their series (bit-identical with  */
/* the device versions: same operations, explicit fma).                */
/* ------------------------------------------------------------------ */
static const double LOG_C[12] = {
    0x1.0000000000000p+0, 0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
    0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4, 0x1.1111111111111p-4,
    0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5, 0x1.8618618618618p-5, 0x1.642c8590b2164p-5};
static const double LN2_HI = 0x1.62e42fee00000p-1;
static const double LN2_LO = 0x1.a39ef35793c76p-33;
static const double SQRT2 = 0x1.6a09e667f3bcdp+0;
/* sin: (-1)^k/(2k+1)!, cos: (-1)^k/(2k)!, k = 0..9 */
static const double SIN_C[10] = {
    0x1.0000000000000p+0, -0x1.5555555555555p-3, 0x1.1111111111111p-7, -0x1.a01a01a01a01ap-13,
    0x1.71de3a556c734p-19, -0x1.ae64567f544e4p-26, 0x1.6124613a86d09p-33, -0x1.ae7f3e733b81fp-41,
    0x1.952c77030ad4ap-49, -0x1.2f49b46814157p-57};
static const double COS_C[10] = {
    0x1.0000000000000p+0, -0x1.0000000000000p-1, 0x1.5555555555555p-5, -0x1.6c16c16c16c17p-10,
    0x1.a01a01a01a01ap-16, -0x1.27e4fb7789f5cp-22, 0x1.1eed8eff8d898p-29, -0x1.93974a8c07c9dp-37,
    0x1.ae7f3e733b81fp-45, -0x1.6827863b97d97p-53};
static const double PIO4_HI = 0x1.921fb54442d18p-1;
static const double PIO4_LO = 0x1.1a62633145c07p-55;

/* natural log of a positive normal double: x = 2^e f, f in [sqrt(1/2), sqrt(2)),
 * log f = 2 atanh(s), s = (f-1)/(f+1), series in s^2. */
double dqo_log(double x) {
    uint64_t b;
    memcpy(&b, &x, 8);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    uint64_t mb = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double f;
    memcpy(&f, &mb, 8);
    if (f > SQRT2) { f = f * 0.5; e += 1; }
    double s = (f - 1.0) / (f + 1.0);
    double z = s * s;
    double p = LOG_C[11];
    for (int k = 10; k >= 0; --k) p = fma(p, z, LOG_C[k]);
    double ls = (s + s) * p;
    double de = (double)e;
    return fma(de, LN2_HI, fma(de, LN2_LO, ls));
}

static void sincos_pio4(double g, double *s, double *c) {
    /* x = g*pi/4, g in [0,1] */
    double x = fma(g, PIO4_HI, g * PIO4_LO);
    double y = x * x;
    double ps = SIN_C[9];
    for (int k = 8; k >= 0; --k) ps = fma(ps, y, SIN_C[k]);
    double pc = COS_C[9];
    for (int k = 8; k >= 0; --k) pc = fma(pc, y, COS_C[k]);
    *s = x * ps;
    *c = pc;
}

/* sin and cos of 2*pi*u for u in [0,1): octant reduction on 8u (exact). */
void dqo_sincos_2pi(double u, double *s, double *c) {
    double t = u * 8.0;
    int k = (int)t;
    double f = t - (double)k;
    double sa, ca;
    if (k & 1) sincos_pio4(1.0 - f, &sa, &ca);
    else sincos_pio4(f, &sa, &ca);
    double S, C;
    switch (k & 7) {
        case 0: S = sa;  C = ca;  break;
        case 1: S = ca;  C = sa;  break;
        case 2: S = ca;  C = -sa; break;
        case 3: S = sa;  C = -ca; break;
        case 4: S = -sa; C = -ca; break;
        case 5: S = -ca; C = -sa; break;
        case 6: S = -ca; C = sa;  break;
        default: S = -sa; C = ca; break;
    }
    *s = S;
    *c = C;
}

/* Normal draw keyed by (seed, purpose, traj, step, site, sub).  One Philox
 * block gives two uniforms of 53 bits and Box-Muller gives two normals; the
 * block is keyed by the trajectory PAIR (traj >> 1), the even trajectory
 * takes the cosine branch and the odd one the sine branch, so both normals
 * of every block are used. */
double dqo_normal(uint64_t seed, uint32_t purpose, uint32_t traj, uint32_t step,
                  uint32_t site, uint32_t sub) {
    uint32_t ctr[4] = {site, step, traj >> 1, (purpose << 24) | sub};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    dqo_philox4x32_10(ctr, key, o);
    uint64_t a = ((uint64_t)o[1] << 32) | o[0];
    uint64_t b = ((uint64_t)o[3] << 32) | o[2];
    double u1 = (double)((a >> 11) + 1) * 0x1.0p-53; /* (0,1] */
    double u2 = (double)(b >> 11) * 0x1.0p-53;       /* [0,1) */
    double r = sqrt(-2.0 * dqo_log(u1));
    double sn, cs;
    dqo_sincos_2pi(u2, &sn, &cs);
    return (traj & 1) ? r * sn : r * cs;
}

/* hbar in cm^-1 fs exactly as cppUtility.cpp:19-22 computes it (note the
 * reference's speed of light 299792548 m/s). */
double dqo_hbar_reference(void) {
    double pi = atan(1.0) * 4.0;
    double lightspeed = 299792548.;
    return (1 / 100.) * (1e15) * 1. / (lightspeed * 2 * pi);
}

/* padeClass.cu:161-168 */
void dqo_pade_ck(int p, double *ck) {
    ck[0] = 1.0;
    double fp = (double)p;
    for (int k = 1; k <= p; ++k) {
        double fk = (double)k;
        ck[k] = ck[k - 1] * (fp + 1. - fk) / ((2 * fp + 1. - fk) * fk);
    }
}

/* ------------------------------------------------------------------ */
/* complex helpers (interleaved re, im)                                */
/* ------------------------------------------------------------------ */
typedef struct { double re, im; } cx;
static inline cx cmul(cx a, cx b) { cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cx cadd(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cx csub(cx a, cx b) { cx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cx cscale(cx a, double s) { cx r = {a.re * s, a.im * s}; return r; }
static inline cx cconj(cx a) { cx r = {a.re, -a.im}; return r; }
static inline double cabs2(cx a) { return a.re * a.re + a.im * a.im; }
static inline cx cdiv(cx a, cx b) {
    double d = b.re * b.re + b.im * b.im;
    cx r = {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
    return r;
}

/* C = A * B for L x L row-major complex */
static void mat_mul(int L, const cx *A, const cx *B, cx *C) {
    for (int i = 0; i < L; ++i)
        for (int j = 0; j < L; ++j) {
            cx s = {0, 0};
            for (int k = 0; k < L; ++k) s = cadd(s, cmul(A[i * L + k], B[k * L + j]));
            C[i * L + j] = s;
        }
}

/* Solve D X = Nm in place (Nm overwritten with X); LU with partial pivoting
 * by |.|^2.  Stands in for culaDeviceZgesv (padeClass.cu:715-745). */
static int lu_solve(int L, cx *D, cx *Nm) {
    for (int k = 0; k < L; ++k) {
        int piv = k;
        double best = cabs2(D[k * L + k]);
        for (int i = k + 1; i < L; ++i) {
            double v = cabs2(D[i * L + k]);
            if (v > best) { best = v; piv = i; }
        }
        if (best == 0.0) return -1;
        if (piv != k) {
            for (int j = 0; j < L; ++j) {
                cx t = D[k * L + j]; D[k * L + j] = D[piv * L + j]; D[piv * L + j] = t;
                t = Nm[k * L + j]; Nm[k * L + j] = Nm[piv * L + j]; Nm[piv * L + j] = t;
            }
        }
        cx inv = cdiv((cx){1.0, 0.0}, D[k * L + k]);
        for (int i = k + 1; i < L; ++i) {
            cx f = cmul(D[i * L + k], inv);
            D[i * L + k] = f;
            for (int j = k + 1; j < L; ++j) D[i * L + j] = csub(D[i * L + j], cmul(f, D[k * L + j]));
            for (int j = 0; j < L; ++j) Nm[i * L + j] = csub(Nm[i * L + j], cmul(f, Nm[k * L + j]));
        }
    }
    for (int k = L - 1; k >= 0; --k) {
        cx inv = cdiv((cx){1.0, 0.0}, D[k * L + k]);
        for (int j = 0; j < L; ++j) {
            cx s = Nm[k * L + j];
            for (int c = k + 1; c < L; ++c) s = csub(s, cmul(D[k * L + c], Nm[c * L + j]));
            Nm[k * L + j] = cmul(s, inv);
        }
    }
    return 0;
}

/* Padé(6,6) with scaling and squaring (padeClass.cu:206-487, 585-706).
 * A is the already-scaled tau*Tbar. */
int dqo_pade_exp(int L, const double *Ain, double *Eout, int norm_mode) {
    size_t L2 = (size_t)L * L;
    cx *A = (cx *)malloc(L2 * sizeof(cx) * 9);
    cx *A2 = A + L2, *A4 = A2 + L2, *A6 = A4 + L2, *U = A6 + L2, *V = U + L2, *T1 = V + L2,
       *D = T1 + L2, *E = D + L2;
    memcpy(A, Ain, L2 * sizeof(cx));
    double ck[7];
    dqo_pade_ck(6, ck);
    /* infinity norm: reference sums |Re| only (gpuPadeHelper.cu:25) */
    double nrm = 0.0;
    for (int i = 0; i < L; ++i) {
        double rs = 0.0;
        for (int j = 0; j < L; ++j) {
            cx a = A[i * L + j];
            rs += (norm_mode == DQO_NORM_REAL_ONLY) ? fabs(a.re) : sqrt(cabs2(a));
        }
        if (rs > nrm) nrm = rs;
    }
    int s = 0;
    while (nrm > 0.5) { nrm *= 0.5; s++; }
    if (s >= 50) { free(A); return -1; }
    double sc = ldexp(1.0, -s);
    for (size_t i = 0; i < L2; ++i) A[i] = cscale(A[i], sc);
    mat_mul(L, A, A, A2);
    mat_mul(L, A2, A2, A4);
    mat_mul(L, A2, A4, A6);
    /* odd part U = A (c1 I + c3 A^2 + c5 A^4) */
    for (int i = 0; i < L; ++i)
        for (int j = 0; j < L; ++j) {
            size_t x = (size_t)i * L + j;
            cx t = cadd(cscale(A2[x], ck[3]), cscale(A4[x], ck[5]));
            if (i == j) t.re += ck[1];
            T1[x] = t;
        }
    mat_mul(L, A, T1, U);
    /* even part V = c0 I + c2 A^2 + c4 A^4 + c6 A^6 */
    for (int i = 0; i < L; ++i)
        for (int j = 0; j < L; ++j) {
            size_t x = (size_t)i * L + j;
            cx t = cadd(cadd(cscale(A2[x], ck[2]), cscale(A4[x], ck[4])), cscale(A6[x], ck[6]));
            if (i == j) t.re += ck[0];
            V[x] = t;
            D[x] = csub(t, U[x]);
        }
    if (lu_solve(L, D, U) != 0) { free(A); return -2; }
    for (int i = 0; i < L; ++i)
        for (int j = 0; j < L; ++j) {
            size_t x = (size_t)i * L + j;
            cx t = cscale(U[x], 2.0);
            if (i == j) t.re += 1.0;
            E[x] = t;
        }
    for (int k = 0; k < s; ++k) {
        mat_mul(L, E, E, T1);
        memcpy(E, T1, L2 * sizeof(cx));
    }
    memcpy(Eout, E, L2 * sizeof(cx));
    free(A);
    return s;
}

/* ------------------------------------------------------------------ */
/* noise                                                               */
/* ------------------------------------------------------------------ */
void dqo_traj_init(const dqo_system *sys, int traj, double *eps, double *deps) {
    for (int i = 0; i < sys->n; ++i) {
        if (sys->static_eps) {
            eps[i] = sys->static_eps[i];
        } else {
            double z = dqo_normal(sys->seed, DQO_P_STATIC, (uint32_t)traj, 0, (uint32_t)i, 0);
            eps[i] = sys->sigma_static * z + sys->h0diag[i];
        }
        if (sys->noise == DQO_NOISE_OU) {
            double z = dqo_normal(sys->seed, DQO_P_OU_INIT, (uint32_t)traj, 0, (uint32_t)i, 0);
            deps[i] = sys->sigma[i] * z;
        } else {
            deps[i] = 0.0;
        }
    }
}

void dqo_noise_update(const dqo_system *sys, int traj, int step, const double *eps, double *deps,
                      double *diag) {
    int n = sys->n;
    if (sys->noise == DQO_NOISE_OU) {
        int ns = sys->ka_substeps > 0 ? sys->ka_substeps : 1;
        double subdt = sys->dt / (double)ns;
        double sqrt_subdt = sqrt(subdt);
        for (int i = 0; i < n; ++i) {
            double inv_tau = 1. / sys->tau[i];
            double coeff = sys->sigma[i] * sqrt(2. / sys->tau[i]);
            double cur = deps[i];
            for (int s = 0; s < ns; ++s) {
                double xi = dqo_normal(sys->seed, DQO_P_OU, (uint32_t)traj, (uint32_t)step, (uint32_t)i,
                                       (uint32_t)s);
                cur = cur - cur * inv_tau * subdt + coeff * xi * sqrt_subdt;
            }
            deps[i] = cur;
            diag[i] = cur + eps[i];
        }
    } else if (sys->noise == DQO_NOISE_GAUSS) {
        for (int i = 0; i < n; ++i) {
            double xi = dqo_normal(sys->seed, DQO_P_GAUSS, (uint32_t)traj, (uint32_t)step, (uint32_t)i, 0);
            double noise = xi * sys->sigma[i];
            diag[i] = noise + eps[i];
        }
    } else {
        for (int i = 0; i < n; ++i) diag[i] = eps[i];
    }
}

/* ------------------------------------------------------------------ */
/* ZZ real noise                                                       */
/* ------------------------------------------------------------------ */
static const double ZZ_INV_2PI = 0x1.45f306dc9c883p-3; /* 1 / (2 pi) */

void dqo_zz_coefficients(int n_osc, const double *omega_invcm, const double *J, double d_omega, double temperature,
                         double *omega_fs, double *coeff) {
    /* systemClass.cu:1128-1139 with hbar = 1, k_B = 0.695035 cm^-1/K,
     * pi = 3.14159265358979323846 and the 1/cm -> 1/fs factor 5308.84 */
    const double pi = 3.14159265358979323846;
    for (int o = 0; o < n_osc; ++o) {
        const double G = J[o] / (1 - exp(-1. / (0.695035 * temperature) * 1.0 * omega_invcm[o]));
        coeff[o] = sqrt(2.) * sqrt(G * d_omega / pi);
        omega_fs[o] = omega_invcm[o] / 5308.84;
    }
}

float dqo_zz_phase(uint64_t seed, uint32_t traj, uint32_t site, uint32_t osc) {
    uint32_t ctr[4] = {site, osc, traj >> 1, (uint32_t)DQO_P_ZZPHASE << 24};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    dqo_philox4x32_10(ctr, key, o);
    const uint64_t a = (traj & 1) ? (((uint64_t)o[3] << 32) | o[2]) : (((uint64_t)o[1] << 32) | o[0]);
    float u = (float)((double)(a >> 11) * 0x1.0p-53);
    if (u >= 1.0f) u = 0.0f; /* the same phase */
    return u;
}

/* The step's oscillator factors (c cos(omega t), c sin(omega t)), t = step dt,
 * with the angle reduced as frac(omega t / 2 pi). */
void dqo_zz_factors(const dqo_system *sys, int step, double *ccw, double *csw) {
    const double t = (double)step * sys->dt;
    for (int o = 0; o < sys->n_osc; ++o) {
        double w = (sys->zz_omega[o] * t) * ZZ_INV_2PI;
        w = w - floor(w);
        double sw, cw;
        dqo_sincos_2pi(w, &sw, &cw);
        ccw[o] = sys->zz_coeff[o] * cw;
        csw[o] = sys->zz_coeff[o] * sw;
    }
}

/* diag_i = eps_i + sum_o c_o cos(omega_o t + 2 pi u_oi), summed as
 * acc <- fma(c cos(omega t), cos(2 pi u), acc); acc <- fma(-c sin(omega t), sin(2 pi u), acc)
 * in oscillator order (gpuSysHelper.cu:134-177 sums c cos(omega t + phi)). */
void dqo_noise_update_zz(const dqo_system *sys, int step, const double *eps, const float *u, double *diag) {
    const int n = sys->n, no = sys->n_osc;
    double *ccw = (double *)malloc(sizeof(double) * 2 * (size_t)no);
    double *csw = ccw + no;
    dqo_zz_factors(sys, step, ccw, csw);
    for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int o = 0; o < no; ++o) {
            double su, cu;
            dqo_sincos_2pi((double)u[(size_t)o * n + i], &su, &cu);
            acc = fma(ccw[o], cu, acc);
            acc = fma(-csw[o], su, acc);
        }
        diag[i] = acc + eps[i];
    }
    free(ccw);
}

/* ------------------------------------------------------------------ */
/* Lanczos                                                             */
/* ------------------------------------------------------------------ */
static void spmv(const dqo_system *sys, const double *diag, const cx *x, cx *y) {
    for (int i = 0; i < sys->n; ++i) {
        cx s = cscale(x[i], diag[i]);
        for (int p = sys->rowptr[i]; p < sys->rowptr[i + 1]; ++p) s = cadd(s, cscale(x[sys->col[p]], sys->val[p]));
        y[i] = s;
    }
}

double dqo_lanczos(const dqo_system *sys, const double *diag, const double *q1, double *Qd,
                   double *alpha_d, double *beta_d) {
    int n = sys->n, m = sys->m;
    cx *Q = (cx *)Qd;
    cx *alpha = (cx *)alpha_d, *beta = (cx *)beta_d;
    cx *w = (cx *)malloc(sizeof(cx) * n);
    memset(Q, 0, sizeof(cx) * (size_t)n * (m + 2));
    memset(alpha, 0, sizeof(cx) * (m + 2));
    memset(beta, 0, sizeof(cx) * (m + 2));
    memcpy(Q + n, q1, sizeof(cx) * n);
    for (int j = 1; j <= m; ++j) {
        cx *qj = Q + (size_t)j * n, *qjm = Q + (size_t)(j - 1) * n, *qjp = Q + (size_t)(j + 1) * n;
        spmv(sys, diag, qj, w);
        cx a = {0, 0};
        for (int i = 0; i < n; ++i)
            a = cadd(a, cmul(sys->dot_mode == DQO_DOT_BILINEAR ? qj[i] : cconj(qj[i]), w[i]));
        alpha[j] = a;
        for (int i = 0; i < n; ++i) {
            w[i] = csub(w[i], cmul(a, qj[i]));
            w[i] = csub(w[i], cmul(beta[j - 1], qjm[i]));
        }
        if (sys->reorth) {
            /* full reorthogonalisation: h_k = <q_k, w> for k = 1..j from the
             * same w, then w -= sum_k h_k q_k (classical Gram-Schmidt, once) */
            cx h[64];
            for (int k = 1; k <= j; ++k) {
                const cx *qk = Q + (size_t)k * n;
                cx acc = {0, 0};
                for (int i = 0; i < n; ++i) acc = cadd(acc, cmul(cconj(qk[i]), w[i]));
                h[k] = acc;
            }
            for (int i = 0; i < n; ++i) {
                cx acc = {0, 0};
                for (int k = 1; k <= j; ++k) acc = cadd(acc, cmul(h[k], Q[(size_t)k * n + i]));
                w[i] = csub(w[i], acc);
            }
        }
        double nn = 0.0;
        for (int i = 0; i < n; ++i) nn += cabs2(w[i]);
        double b = sqrt(nn);
        /* lucky breakdown (the reference divides by zero here,
         * gpuSimpleOps.cu:24-28): the Krylov space is invariant; q_{j+1} = 0
         * decouples the rest of T and the step stays exact. */
        if (b <= 1e-12 * (sqrt(cabs2(a)) + (j > 1 ? beta[j - 1].re : 0.0))) b = 0.0;
        beta[j].re = b;
        beta[j].im = 0.0;
        double inv = b > 0.0 ? 1.0 / b : 0.0;
        for (int i = 0; i < n; ++i) qjp[i] = cscale(w[i], inv);
    }
    spmv(sys, diag, Q + (size_t)(m + 1) * n, w);
    double nn = 0.0;
    for (int i = 0; i < n; ++i) nn += cabs2(w[i]);
    free(w);
    return sqrt(nn);
}

/* gpuLanczosHelper.cu:14-60, row-major L x L with L = m+2 */
void dqo_build_tbar(int m, const double *alpha_d, const double *beta_d, double *Td) {
    int L = m + 2;
    const cx *alpha = (const cx *)alpha_d, *beta = (const cx *)beta_d;
    cx *T = (cx *)Td;
    memset(T, 0, sizeof(cx) * L * L);
    for (int i = 0; i < m; ++i) {
        T[i * L + i] = alpha[i + 1];
        if (i + 1 < m) {
            T[i * L + i + 1] = beta[i + 1];
            T[(i + 1) * L + i] = beta[i + 1];
        }
    }
    T[0 * L + m].re = 1.0;
    T[m * L + m + 1].re = 1.0;
}

int dqo_krylov_step(const dqo_system *sys, const double *diag, const double *psi_in, double *psi_out,
                    double *err_est, double *norm_out, int *s_out) {
    return dqo_krylov_step_m(sys, diag, psi_in, psi_out, err_est, norm_out, s_out, NULL);
}

/* EXPOKIT's first error term for a Krylov dimension j: beta_j |E(j-1, j)|,
 * E = exp(tau Tbar_j) of the augmented (j+2) matrix. */
static double err1_at(int j, const double *al, const double *be, cx tau, int norm_mode) {
    const int L = j + 2;
    double *T = (double *)malloc(sizeof(cx) * L * L);
    double *E = (double *)malloc(sizeof(cx) * L * L);
    dqo_build_tbar(j, al, be, T);
    cx *Tc = (cx *)T;
    for (int i = 0; i < L * L; ++i) Tc[i] = cmul(tau, Tc[i]);
    const int s = dqo_pade_exp(L, T, E, norm_mode);
    const cx *Ec = (const cx *)E;
    const double r = s < 0 ? INFINITY : sqrt(cabs2(((const cx *)be)[j])) * sqrt(cabs2(Ec[(j - 1) * L + j]));
    free(T);
    free(E);
    return r;
}

int dqo_krylov_step_m(const dqo_system *sys, const double *diag, const double *psi_in, double *psi_out,
                      double *err_est, double *norm_out, int *s_out, int *m_used) {
    int n = sys->n, mmax = sys->m;
    double *Q = (double *)malloc(sizeof(cx) * (size_t)n * (mmax + 2));
    double *al = (double *)malloc(sizeof(cx) * (mmax + 2));
    double *be = (double *)malloc(sizeof(cx) * (mmax + 2));
    double nrm_av = dqo_lanczos(sys, diag, psi_in, Q, al, be);
    const cx tau0 = {0.0, -sys->dt / sys->hbar};
    int m = mmax;
    if (sys->m_min > 0) {
        /* adaptive dimension: the first checked j whose EXPOKIT err1 meets the tolerance */
        for (int j = sys->m_min; j < mmax; j += DQO_M_CHECK_STRIDE) {
            if (err1_at(j, al, be, tau0, sys->norm_mode) <= sys->m_tol) {
                m = j;
                break;
            }
        }
    }
    if (m_used) *m_used = m;
    const int L = m + 2;
    double *T = (double *)malloc(sizeof(cx) * L * L);
    double *E = (double *)malloc(sizeof(cx) * L * L);
    dqo_build_tbar(m, al, be, T);
    cx tau = {0.0, -sys->dt / sys->hbar};
    cx *Tc = (cx *)T;
    for (int i = 0; i < L * L; ++i) Tc[i] = cmul(tau, Tc[i]);
    int s = dqo_pade_exp(L, T, E, sys->norm_mode);
    if (s_out) *s_out = s;
    if (s < 0) { free(Q); free(al); free(be); free(T); free(E); return s; }
    cx *Ec = (cx *)E, *Qc = (cx *)Q, *out = (cx *)psi_out;
    for (int i = 0; i < n; ++i) {
        cx acc = {0, 0};
        for (int j = 0; j < m; ++j) acc = cadd(acc, cmul(Qc[(size_t)(j + 1) * n + i], Ec[j * L + 0]));
        out[i] = acc;
    }
    double nn = 0.0;
    for (int i = 0; i < n; ++i) nn += cabs2(out[i]);
    double nrm = sqrt(nn);
    if (norm_out) *norm_out = nrm;
    double inv = 1. / nrm;
    for (int i = 0; i < n; ++i) out[i] = cscale(out[i], inv);
    /* EXPOKIT Alg. 3.2 (padeClass.cu:750-782; systemClass.cu:2075-2077); with
     * the adaptive dimension only err1 (||H q_{m+1}|| belongs to the largest m) */
    if (err_est) {
        cx *bec = (cx *)be;
        double hm = sqrt(cabs2(bec[m]));
        double err1 = hm * sqrt(cabs2(Ec[(m - 1) * L + m]));
        double err2 = hm * nrm_av * sqrt(cabs2(Ec[(m - 1) * L + m + 1]));
        double est = (sys->m_min > 0) ? err1 : (err1 > err2) ? err2 / (1 - err2 / err1) : err1;
        if (est < 1.110223e-16) est = 1.110223e-16;
        *err_est = est;
    }
    free(Q); free(al); free(be); free(T); free(E);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Taylor-Krylov (taylorKrylovClass.cu:196-434)                        */
/* ------------------------------------------------------------------ */
int dqo_tk_step(const dqo_system *sys, const double *diag, const double *psi_in, double *psi_out,
                double *err_est, double *norm_out) {
    const int n = sys->n, p = sys->tk_p, mb = sys->tk_m, L = mb + p;
    const cx tau = {0.0, -sys->dt / sys->hbar};
    /* Taylor coefficients tau^k / k! (taylorKrylovClass.cu:200-206) */
    cx ck[DQO_TK_MAX_P];
    cx pw = {1.0, 0.0};
    double fact = 1.0;
    ck[0] = pw;
    for (int k = 1; k < p; ++k) {
        pw = cmul(pw, tau);
        fact *= k;
        ck[k].re = pw.re / fact;
        ck[k].im = pw.im / fact;
    }
    cx *acc = (cx *)malloc(sizeof(cx) * (size_t)n * 3);
    cx *x = acc + n, *y = x + n;
    memcpy(acc, psi_in, sizeof(cx) * n);
    memcpy(x, psi_in, sizeof(cx) * n);
    /* acc = sum_{k<p} c_k A^k psi; x ends as A^p psi (:231-300) */
    for (int k = 1; k <= p; ++k) {
        spmv(sys, diag, x, y);
        if (k < p)
            for (int i = 0; i < n; ++i) acc[i] = cadd(acc[i], cmul(ck[k], y[i]));
        cx *t = x; x = y; y = t;
    }
    /* Krylov part on B from A^p psi (:327-375) */
    double nn = 0.0;
    for (int i = 0; i < n; ++i) nn += cabs2(x[i]);
    const double beta0 = sqrt(nn);
    const double inv0 = beta0 > 0.0 ? 1.0 / beta0 : 0.0;
    for (int i = 0; i < n; ++i) y[i] = cscale(x[i], inv0);
    dqo_system sb = *sys;
    sb.rowptr = sys->tk_rowptr;
    sb.col = sys->tk_col;
    sb.val = sys->tk_val;
    sb.m = mb;
    double *Q = (double *)malloc(sizeof(cx) * (size_t)n * (mb + 2));
    double *al = (double *)malloc(sizeof(cx) * (mb + 2));
    double *be = (double *)malloc(sizeof(cx) * (mb + 2));
    const double nrm_bv = dqo_lanczos(&sb, sys->tk_diag, (const double *)y, Q, al, be);
    /* augmented matrix of size mB + p (gpuLanczosHelper.cu:14-60) */
    cx *T = (cx *)calloc((size_t)L * L, sizeof(cx));
    cx *E = (cx *)malloc(sizeof(cx) * (size_t)L * L);
    const cx *alc = (const cx *)al, *bec = (const cx *)be;
    for (int i = 0; i < mb; ++i) {
        T[i * L + i] = alc[i + 1];
        if (i + 1 < mb) {
            T[i * L + i + 1] = bec[i + 1];
            T[(i + 1) * L + i] = bec[i + 1];
        }
    }
    T[0 * L + mb].re = 1.0;
    for (int k = mb; k + 1 < L; ++k) T[k * L + k + 1].re = 1.0;
    for (int i = 0; i < L * L; ++i) T[i] = cmul(tau, T[i]);
    const int s = dqo_pade_exp(L, (const double *)T, (double *)E, sys->norm_mode);
    int rc = 0;
    if (s < 0) {
        rc = s;
    } else {
        /* out = ||A^p psi|| Q_B phi + taylor part (:345-396) */
        const cx *Qc = (const cx *)Q;
        cx *out = (cx *)psi_out;
        for (int i = 0; i < n; ++i) {
            cx k = {0, 0};
            for (int j = 0; j < mb; ++j) k = cadd(k, cmul(Qc[(size_t)(j + 1) * n + i], E[j * L + L - 1]));
            out[i] = cadd(cscale(k, beta0), acc[i]);
        }
        double on = 0.0;
        for (int i = 0; i < n; ++i) on += cabs2(out[i]);
        const double nrm = sqrt(on);
        if (norm_out) *norm_out = nrm;
        const double inv = 1.0 / nrm;
        for (int i = 0; i < n; ++i) out[i] = cscale(out[i], inv);
        if (err_est) {
            /* padeClass.cu:750-782 on the B part, plus |1 - norm| (:417-434) */
            const double hm = sqrt(cabs2(bec[mb]));
            const double err1 = hm * sqrt(cabs2(E[(mb - 1) * L + mb]));
            const double err2 = hm * nrm_bv * sqrt(cabs2(E[(mb - 1) * L + mb + 1]));
            double est = (err1 > err2) ? err2 / (1 - err2 / err1) : err1;
            est += fabs(1.0 - nrm);
            if (est < 1.110223e-16) est = 1.110223e-16;
            *err_est = est;
        }
    }
    free(acc); free(Q); free(al); free(be); free(T); free(E);
    return rc;
}

/* ------------------------------------------------------------------ */
/* ensemble                                                            */
/* ------------------------------------------------------------------ */
/* 1 / sum_i |psi_i|^4 (systemClass.cu:2209-2253, accumulated in FP64) */
static double ipr_of(int n, const cx *psi) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
        const double a = cabs2(psi[i]);
        s += a * a;
    }
    return 1.0 / s;
}

int dqo_run(const dqo_system *sys, int traj0, int n_traj, int n_steps, const double *psi0d, int pop_every,
            double *pops, double *corr, double *psi_final, double *err_acc, double *ipr, int n_threads) {
    int n = sys->n;
    int n_rec = n_steps / pop_every + 1;
    int nt = 1;
#ifdef _OPENMP
    nt = n_threads > 0 ? n_threads : omp_get_max_threads();
    if (nt > n_traj) nt = n_traj;
    if (nt < 1) nt = 1;
#endif
    double *pacc = (double *)calloc((size_t)nt * n_rec * n, sizeof(double));
    double *cacc = (double *)calloc((size_t)nt * (n_steps + 1) * 2, sizeof(double));
    double *iacc = (double *)calloc((size_t)nt * (n_steps + 1), sizeof(double));
    int status = 0;
    const cx *psi0 = (const cx *)psi0d;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *myp = pacc + (size_t)tid * n_rec * n;
        double *myc = cacc + (size_t)tid * (n_steps + 1) * 2;
        double *myi = iacc + (size_t)tid * (n_steps + 1);
        double *eps = (double *)malloc(sizeof(double) * n * 3);
        double *deps = eps + n, *diag = deps + n;
        float *zzu = sys->noise == DQO_NOISE_ZZ ? (float *)malloc(sizeof(float) * (size_t)sys->n_osc * n) : NULL;
        cx *psi = (cx *)malloc(sizeof(cx) * n * 2);
        cx *tmp = psi + n;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int t = 0; t < n_traj; ++t) {
            int traj = traj0 + t;
            dqo_traj_init(sys, traj, eps, deps);
            if (zzu)
                for (int o = 0; o < sys->n_osc; ++o)
                    for (int i = 0; i < n; ++i)
                        zzu[(size_t)o * n + i] = dqo_zz_phase(sys->seed, (uint32_t)traj, (uint32_t)i, (uint32_t)o);
            memcpy(psi, psi0, sizeof(cx) * n);
            double errsum = 0.0;
            const cx *bra = sys->corr_bra ? (const cx *)sys->corr_bra : psi0;
            cx c = {0, 0};
            if (sys->corr_bra) c.re = 1.0;
            else for (int i = 0; i < n; ++i) c = cadd(c, cmul(cconj(psi0[i]), psi[i]));
            myc[0] += c.re; myc[1] += c.im;
            for (int i = 0; i < n; ++i) myp[i] += cabs2(psi[i]);
            myi[0] += ipr_of(n, psi);
            for (int k = 0; k < n_steps; ++k) {
                if (zzu) dqo_noise_update_zz(sys, k, eps, zzu, diag);
                else dqo_noise_update(sys, traj, k, eps, deps, diag);
                double est;
                int rc = sys->tk_p > 0 ? dqo_tk_step(sys, diag, (const double *)psi, (double *)tmp, &est, NULL)
                                       : dqo_krylov_step(sys, diag, (const double *)psi, (double *)tmp, &est, NULL, NULL);
                if (rc != 0) { status = rc; break; }
                errsum += est;
                memcpy(psi, tmp, sizeof(cx) * n);
                c.re = 0; c.im = 0;
                for (int i = 0; i < n; ++i) c = cadd(c, cmul(cconj(bra[i]), psi[i]));
                myc[2 * (k + 1)] += c.re; myc[2 * (k + 1) + 1] += c.im;
                myi[k + 1] += ipr_of(n, psi);
                if ((k + 1) % pop_every == 0) {
                    double *row = myp + (size_t)((k + 1) / pop_every) * n;
                    for (int i = 0; i < n; ++i) row[i] += cabs2(psi[i]);
                }
            }
            if (psi_final) memcpy(psi_final + (size_t)t * n * 2, psi, sizeof(cx) * n);
            if (err_acc) err_acc[t] = errsum;
        }
        free(eps);
        free(zzu);
        free(psi);
    }
    double inv = 1.0 / n_traj;
    if (pops) {
        for (size_t x = 0; x < (size_t)n_rec * n; ++x) {
            double s = 0.0;
            for (int t = 0; t < nt; ++t) s += pacc[(size_t)t * n_rec * n + x];
            pops[x] = s * inv;
        }
    }
    if (corr) {
        for (int x = 0; x < (n_steps + 1) * 2; ++x) {
            double s = 0.0;
            for (int t = 0; t < nt; ++t) s += cacc[(size_t)t * (n_steps + 1) * 2 + x];
            corr[x] = s * inv;
        }
    }
    if (ipr) {
        for (int k = 0; k <= n_steps; ++k) {
            double s = 0.0;
            for (int t = 0; t < nt; ++t) s += iacc[(size_t)t * (n_steps + 1) + k];
            ipr[k] = s * inv;
        }
    }
    free(pacc);
    free(cacc);
    free(iacc);
    return status;
}

/* ------------------------------------------------------------------ */
/* inverse DFT, cuFFT INVERSE convention: X_k = sum_j x_j e^{+2 pi i jk/n} */
/* ------------------------------------------------------------------ */
void dqo_ifft(int n, double *xd) {
    cx *x = (cx *)xd;
    if (n <= 1) return;
    if ((n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { cx t = x[i]; x[i] = x[j]; x[j] = t; }
        }
        for (int len = 2; len <= n; len <<= 1) {
            double ang = 2.0 * M_PI / len;
            for (int i = 0; i < n; i += len) {
                for (int k = 0; k < len / 2; ++k) {
                    cx w = {cos(ang * k), sin(ang * k)};
                    cx u = x[i + k], v = cmul(x[i + k + len / 2], w);
                    x[i + k] = cadd(u, v);
                    x[i + k + len / 2] = csub(u, v);
                }
            }
        }
    } else {
        cx *y = (cx *)malloc(sizeof(cx) * n);
        for (int k = 0; k < n; ++k) {
            cx s = {0, 0};
            for (int j = 0; j < n; ++j) {
                double ang = 2.0 * M_PI * (double)(((long long)j * k) % n) / n;
                cx w = {cos(ang), sin(ang)};
                s = cadd(s, cmul(x[j], w));
            }
            y[k] = s;
        }
        memcpy(x, y, sizeof(cx) * n);
        free(y);
    }
}

/* ------------------------------------------------------------------ */
/* Spectrum loss and its adjoint gradient (FP64 host reference).       */
/* This capability has no reference counterpart; it restates the        */
/* adjoint of psi(k+1) = exp(tau H_k) psi(k), tau = -i dt/hbar:          */
/*   lambda(T) = s_T,  lambda(k) = s_k + exp(tau H_k)^dagger lambda(k+1) */
/*   dL/dp = Re sum_k int_0^1 <e^{(1-s)A^+}lambda(k+1)| tau dH/dp e^{sA} psi(k)> ds */
/* with both exponentials in their Krylov bases and the s-integral from   */
/* the block-triangular exponential exp([[tau T_W, e1 e1^T],[0, tau T_V]]) */
/* (Van Loan 1978).  Needs the Hermitian Lanczos product.               */
/* ------------------------------------------------------------------ */
static void tridiag_m(int m, const cx *alpha, const cx *beta, cx *T) {
    memset(T, 0, sizeof(cx) * m * m);
    for (int i = 0; i < m; ++i) {
        T[i * m + i] = alpha[i + 1];
        if (i + 1 < m) { T[i * m + i + 1] = beta[i + 1]; T[(i + 1) * m + i] = beta[i + 1]; }
    }
}

double dqo_spectrum_loss_grad(const dqo_system *sys, const double *val_base, const int *cls, int n_classes,
                              int n_traj, int n_steps, const double *psi0d, int len, double scale,
                              const double *target, double *grad, int n_threads) {
    (void)n_threads;
    const int n = sys->n, m = sys->m, T = n_steps;
    const cx *psi0 = (const cx *)psi0d;
    const cx tau = {0.0, -sys->dt / sys->hbar};
    /* forward: store psi(k) and the diagonal of every step */
    cx *psi_all = (cx *)malloc(sizeof(cx) * (size_t)n_traj * (T + 1) * n);
    double *diag_all = (double *)malloc(sizeof(double) * (size_t)n_traj * T * n);
    cx *C = (cx *)calloc((size_t)(T + 1), sizeof(cx));
    double *eps = (double *)malloc(sizeof(double) * n * 2);
    double *deps = eps + n;
    float *zzu = sys->noise == DQO_NOISE_ZZ ? (float *)malloc(sizeof(float) * (size_t)sys->n_osc * n) : NULL;
    for (int b = 0; b < n_traj; ++b) {
        dqo_traj_init(sys, b, eps, deps);
        if (zzu)
            for (int o = 0; o < sys->n_osc; ++o)
                for (int i = 0; i < n; ++i)
                    zzu[(size_t)o * n + i] = dqo_zz_phase(sys->seed, (uint32_t)b, (uint32_t)i, (uint32_t)o);
        cx *ps = psi_all + (size_t)b * (T + 1) * n;
        memcpy(ps, psi0, sizeof(cx) * n);
        for (int k = 0; k < T; ++k) {
            double *d = diag_all + ((size_t)b * T + k) * n;
            if (zzu) dqo_noise_update_zz(sys, k, eps, zzu, d);
            else dqo_noise_update(sys, b, k, eps, deps, d);
            dqo_krylov_step(sys, d, (const double *)(ps + (size_t)k * n), (double *)(ps + (size_t)(k + 1) * n), NULL,
                            NULL, NULL);
        }
        for (int k = 0; k <= T; ++k) {
            cx acc = {0, 0};
            for (int i = 0; i < n; ++i) acc = cadd(acc, cmul(cconj(psi0[i]), ps[(size_t)k * n + i]));
            C[k].re += acc.re / n_traj;
            C[k].im += acc.im / n_traj;
        }
    }
    /* spectrum, loss, G = IDFT(g) */
    cx *S = (cx *)calloc((size_t)len, sizeof(cx));
    for (int k = 0; k <= T && k < len; ++k) S[k] = C[k];
    dqo_ifft(len, (double *)S);
    double loss = 0.0;
    cx *Gv = (cx *)calloc((size_t)len, sizeof(cx));
    for (int j = 0; j < len; ++j) {
        double a = scale * S[j].re - target[j];
        loss += a * a;
        Gv[j].re = 2.0 * scale * a;
    }
    if (!grad) {
        free(psi_all); free(diag_all); free(C); free(eps); free(zzu); free(S); free(Gv);
        return loss;
    }
    dqo_ifft(len, (double *)Gv);
    memset(grad, 0, sizeof(double) * (n + n_classes));
    cx *V = (cx *)malloc(sizeof(cx) * (size_t)n * (m + 2));
    cx *W = (cx *)malloc(sizeof(cx) * (size_t)n * (m + 2));
    cx *aV = (cx *)malloc(sizeof(cx) * (m + 2) * 4);
    cx *bV = aV + (m + 2), *aW = bV + (m + 2), *bW = aW + (m + 2);
    cx *lam = (cx *)malloc(sizeof(cx) * n * 3);
    cx *qw = lam + n, *tvec = lam + 2 * n;
    const int L2 = 2 * m;
    cx *Z = (cx *)malloc(sizeof(cx) * L2 * L2 * 2);
    cx *EZ = Z + L2 * L2;
    cx *TW = (cx *)malloc(sizeof(cx) * m * m * 3);
    cx *TV = TW + m * m, *EW = TV + m * m;
    cx *tb = (cx *)malloc(sizeof(cx) * m);
    for (int b = 0; b < n_traj; ++b) {
        const cx *ps = psi_all + (size_t)b * (T + 1) * n;
        for (int i = 0; i < n; ++i) lam[i] = cscale(cmul(cconj(Gv[T]), psi0[i]), 1.0 / n_traj);
        for (int t = T - 1; t >= 0; --t) {
            const double *d = diag_all + ((size_t)b * T + t) * n;
            dqo_lanczos(sys, d, (const double *)(ps + (size_t)t * n), (double *)V, (double *)aV, (double *)bV);
            double ln = 0.0;
            for (int i = 0; i < n; ++i) ln += cabs2(lam[i]);
            ln = sqrt(ln);
            cx *Ul = tvec;
            memset(Ul, 0, sizeof(cx) * n);
            if (ln > 0.0) {
                for (int i = 0; i < n; ++i) qw[i] = cscale(lam[i], 1.0 / ln);
                dqo_lanczos(sys, d, (const double *)qw, (double *)W, (double *)aW, (double *)bW);
                tridiag_m(m, aW, bW, TW);
                tridiag_m(m, aV, bV, TV);
                /* U^dagger lam = ||lam|| W exp(-tau T_W) e1 */
                const cx mtau = cscale(tau, -1.0);
                for (int x = 0; x < m * m; ++x) EZ[x] = cmul(mtau, TW[x]);
                dqo_pade_exp(m, (const double *)EZ, (double *)EW, DQO_NORM_COMPLEX);
                for (int i = 0; i < n; ++i) {
                    cx acc = {0, 0};
                    for (int a = 0; a < m; ++a) acc = cadd(acc, cmul(W[(size_t)(a + 1) * n + i], EW[a * m]));
                    Ul[i] = cscale(acc, ln);
                }
                /* Van Loan: Z = [[tau T_W, E11], [0, tau T_V]] */
                memset(Z, 0, sizeof(cx) * L2 * L2);
                for (int i = 0; i < m; ++i)
                    for (int j = 0; j < m; ++j) {
                        Z[i * L2 + j] = cmul(tau, TW[i * m + j]);
                        Z[(m + i) * L2 + m + j] = cmul(tau, TV[i * m + j]);
                    }
                Z[0 * L2 + m].re = 1.0;
                dqo_pade_exp(L2, (const double *)Z, (double *)EZ, DQO_NORM_COMPLEX);
                /* rho_ik = tau ||lam|| sum_ab conj(W_ia) N_ab V_kb, N = EZ[0:m, m:2m] */
                cx coef = cscale(tau, ln);
                for (int i = 0; i < n; ++i) {
                    for (int bb = 0; bb < m; ++bb) {
                        cx acc = {0, 0};
                        for (int a = 0; a < m; ++a)
                            acc = cadd(acc, cmul(cconj(W[(size_t)(a + 1) * n + i]), EZ[a * L2 + m + bb]));
                        tb[bb] = cmul(coef, acc);
                    }
                    /* diagonal: site energy i */
                    cx rho = {0, 0};
                    for (int bb = 0; bb < m; ++bb) rho = cadd(rho, cmul(tb[bb], V[(size_t)(bb + 1) * n + i]));
                    grad[i] += rho.re;
                    /* off-diagonal: coupling classes */
                    if (n_classes > 0) {
                        for (int p = sys->rowptr[i]; p < sys->rowptr[i + 1]; ++p) {
                            int k = sys->col[p];
                            cx r2 = {0, 0};
                            for (int bb = 0; bb < m; ++bb) r2 = cadd(r2, cmul(tb[bb], V[(size_t)(bb + 1) * n + k]));
                            grad[n + cls[p]] += val_base[p] * r2.re;
                        }
                    }
                }
            }
            for (int i = 0; i < n; ++i)
                lam[i] = cadd(cscale(cmul(cconj(Gv[t]), psi0[i]), 1.0 / n_traj), Ul[i]);
        }
    }
    free(psi_all); free(diag_all); free(C); free(eps); free(zzu); free(S); free(Gv);
    free(V); free(W); free(aV); free(lam); free(Z); free(TW); free(tb);
    return loss;
}
