/*
 * dq_oracle.h — CPU FP64 restatement of DynaQuant's stochastic-Hamiltonian
 * Krylov step.  TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is
 * compared against.  Nothing in the product library links or calls it; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity pins: Padé c_k and hbar/expCoeff against the reference's captured
 * log (out:76-83), the Padé exponential against scipy.linalg.expm, the full
 * step against dense expm(-i dt H/hbar), Philox against the published
 * Random123 known answers and cuRAND's device generator.  The reference's
 * own trajectories are not reproducible (wall-clock seeds, missing
 * Hamiltonian file), so trajectory-level golden vectors are generated by
 * this oracle with fixed Philox seeds (tests/golden/make_golden.py).
 */
#ifndef DQ_ORACLE_H
#define DQ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Noise models (reference enum simulationType, includeFiles.cu:19-25). */
enum { DQO_NOISE_NONE = 0, DQO_NOISE_GAUSS = 1, DQO_NOISE_OU = 2, DQO_NOISE_ZZ = 3 };
/* Lanczos alpha: reference-exact unconjugated dot (lanczosClass.cu:421,
 * cublasZdotu) or the Hermitian inner product. */
enum { DQO_DOT_BILINEAR = 0, DQO_DOT_HERMITIAN = 1 };
/* Padé scaling norm: reference |Re|-only row sums (gpuPadeHelper.cu:25) or
 * the complex-modulus infinity norm. */
enum { DQO_NORM_REAL_ONLY = 0, DQO_NORM_COMPLEX = 1 };
/* Philox purposes (the fourth counter word's top byte). */
enum { DQO_P_OU = 1, DQO_P_GAUSS = 2, DQO_P_OU_INIT = 3, DQO_P_STATIC = 4, DQO_P_ZZPHASE = 5 };

typedef struct {
    int n;                 /* sites */
    const int *rowptr;     /* off-diagonal CSR, n+1 */
    const int *col;        /* off-diagonal column indices */
    const double *val;     /* off-diagonal couplings (cm^-1), already scaled */
    const double *h0diag;  /* diagonal of the input Hamiltonian (cm^-1), n */
    int m;                 /* Krylov dimension */
    double dt;             /* fs */
    double hbar;           /* cm^-1 fs */
    int dot_mode;
    int norm_mode;
    int noise;             /* DQO_NOISE_* */
    int ka_substeps;       /* OU Euler-Maruyama substeps per step */
    const double *sigma;   /* per-site noise sigma (cm^-1), n (or NULL) */
    const double *tau;     /* per-site OU correlation time (fs), n (or NULL) */
    double sigma_static;   /* static disorder sigma, redrawn per trajectory */
    const double *static_eps; /* optional explicit static energies (n), replaces h0diag+disorder */
    uint64_t seed;
    int reorth;            /* 1: full reorthogonalisation (classical Gram-Schmidt, once) */
    int m_min;             /* adaptive Krylov dimension: first check (0 = fixed m) */
    double m_tol;          /* adaptive: accept the first checked j with beta_j |E(j-1, j)| <= m_tol */
    int n_osc;             /* ZZ real noise: oscillators per site */
    const double *zz_omega; /* ZZ: angular frequencies (rad/fs), n_osc */
    const double *zz_coeff; /* ZZ: amplitudes (cm^-1), n_osc */
    int tk_p;              /* Taylor-Krylov order p (0 = Lanczos mode) */
    int tk_m;              /* Taylor-Krylov: Krylov dimension on the auxiliary matrix B */
    const int *tk_rowptr;  /* B: off-diagonal CSR, n+1 */
    const int *tk_col;
    const double *tk_val;
    const double *tk_diag; /* B: diagonal, n */
    const double *corr_bra; /* optional correlation bra (n complex); M(0) is then 1 (spectraClass.cu:296) */
} dqo_system;

/* Checks of the adaptive Krylov dimension happen at j = m_min, m_min + 4,
 * ... below m; a trajectory that passes none uses m. */
enum { DQO_M_CHECK_STRIDE = 4 };
/* Taylor-Krylov order limit */
enum { DQO_TK_MAX_P = 32 };

/* ---- building blocks ---- */
void dqo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double dqo_log(double x);
void dqo_sincos_2pi(double u, double *s, double *c);
double dqo_normal(uint64_t seed, uint32_t purpose, uint32_t traj, uint32_t step,
                  uint32_t site, uint32_t sub);
double dqo_hbar_reference(void);
void dqo_pade_ck(int p, double *ck);
/* exp of an L x L complex matrix A (row-major interleaved re/im), Padé(6,6)
 * with scaling and squaring; returns s (or -1 when s >= 50). */
int dqo_pade_exp(int L, const double *A, double *E, int norm_mode);

/* ---- one trajectory ---- */
/* Per-trajectory state: static energies eps (n), OU offsets deps (n). */
void dqo_traj_init(const dqo_system *sys, int traj, double *eps, double *deps);
/* Noise update for step `step` (gpuSysHelper.cu:73-128 / :32-66): writes the
 * step's diagonal into diag (n) and advances deps. */
void dqo_noise_update(const dqo_system *sys, int traj, int step, const double *eps,
                      double *deps, double *diag);
/* Lanczos + Padé + combine + renorm for one step. psi_in/psi_out are n complex
 * (interleaved).  Returns 0 on success; err_est gets the EXPOKIT estimate,
 * norm_out the pre-renormalisation norm, s_out the Padé scaling. */
int dqo_krylov_step(const dqo_system *sys, const double *diag, const double *psi_in,
                    double *psi_out, double *err_est, double *norm_out, int *s_out);
/* As dqo_krylov_step, also returning the Krylov dimension used (m, or the
 * adaptive choice when sys->m_min > 0). */
int dqo_krylov_step_m(const dqo_system *sys, const double *diag, const double *psi_in,
                      double *psi_out, double *err_est, double *norm_out, int *s_out, int *m_used);
/* Taylor-Krylov step (taylorKrylovClass.cu:223-434): psi_out = sum_{k<p}
 * tau^k/k! A^k psi_in + ||A^p psi_in|| Q_B [exp(tau Tbar_B)]_{0..mB-1, L-1},
 * Tbar_B the (mB + p) augmented Lanczos matrix of B from A^p psi_in (ones at
 * (0, mB) and (mB+k, mB+k+1)), then renormalised.  err_est = EXPOKIT
 * estimate of the B part + |1 - norm|.  A is H with this step's diagonal. */
int dqo_tk_step(const dqo_system *sys, const double *diag, const double *psi_in, double *psi_out,
                double *err_est, double *norm_out);
/* Lanczos only: Q (m+2) columns of n complex each (column 0 zero), alpha and
 * beta (m+2 complex each), returns ||H q_{m+1}||. */
double dqo_lanczos(const dqo_system *sys, const double *diag, const double *q1,
                   double *Q, double *alpha, double *beta);
void dqo_build_tbar(int m, const double *alpha, const double *beta, double *T);

/* ---- ZZ real noise (gpuSysHelper.cu:134-177, systemClass.cu:1077-1240) ---- */
/* Amplitude and angular frequency of one oscillator of the spectral density:
 * G = J / (1 - exp(-omega / (k_B T))), coeff = sqrt(2) sqrt(G d_omega / pi),
 * omega_fs = omega / 5308.84 (omega, J, d_omega in cm^-1, T in K). */
void dqo_zz_coefficients(int n_osc, const double *omega_invcm, const double *J, double d_omega, double temperature,
                         double *omega_fs, double *coeff);
/* Phase fraction (phi / 2 pi, float) of oscillator osc at site for a
 * trajectory: Philox keyed (seed, ZZPHASE, trajectory pair, osc, site). */
float dqo_zz_phase(uint64_t seed, uint32_t traj, uint32_t site, uint32_t osc);
/* diag_i = eps_i + sum_osc coeff cos(omega t + 2 pi u_osc,i) at t = step dt,
 * summed in oscillator order as two fused multiply-adds per oscillator with
 * the factors of dqo_zz_factors and sin/cos(2 pi u); u is [osc][site]. */
void dqo_noise_update_zz(const dqo_system *sys, int step, const double *eps, const float *u, double *diag);
/* (coeff cos(omega t), coeff sin(omega t)) per oscillator, angle frac(omega t / 2 pi) */
void dqo_zz_factors(const dqo_system *sys, int step, double *ccw, double *csw);

/* ---- ensemble run ---- */
/* Runs trajectories traj0..traj0+n_traj-1 for n_steps from psi0 (n complex).
 * pops: (n_steps/pop_every + 1) x n, ensemble-averaged |psi|^2 at steps
 * 0, pop_every, ...; corr: (n_steps+1) complex, averaged <psi0|psi(t)>;
 * psi_final: n_traj x n complex (may be NULL); err_acc: n_traj (may be NULL);
 * ipr: n_steps + 1, averaged 1 / sum_i |psi_i(k)|^4 (may be NULL,
 * systemClass.cu:2219-2257).  Taylor-Krylov steps when sys->tk_p > 0.
 * Returns 0 or a negative error code. */
int dqo_run(const dqo_system *sys, int traj0, int n_traj, int n_steps, const double *psi0,
            int pop_every, double *pops, double *corr, double *psi_final, double *err_acc,
            double *ipr, int n_threads);

/* ---- spectrum ---- */
/* In-place inverse DFT (sign +1, unnormalised, cuFFT INVERSE convention) of
 * n complex values; radix-2 when n is a power of two, direct sum otherwise. */
void dqo_ifft(int n, double *x);

/* ---- adjoint (no reference counterpart) ---- */
/* Loss L = sum_j (scale * Re(IDFT_len(Cbar)_j) - target_j)^2 with Cbar(k) the
 * trajectory mean of <psi0|psi(k)>, k = 0..n_steps, zero-padded to len.  The
 * site energies are sys->static_eps; val (in sys) must equal sum over classes
 * of scale_c * val_base.  grad (n + n_classes, may be NULL) receives dL/deps_i
 * and dL/dscale_c.  Hermitian dot only.  Returns L. */
double dqo_spectrum_loss_grad(const dqo_system *sys, const double *val_base, const int *cls, int n_classes,
                              int n_traj, int n_steps, const double *psi0, int len, double scale,
                              const double *target, double *grad, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
