/*
 * dq.h — C ABI of dynaquant_b200, a B200 (sm_100a) implementation of
 * DynaQuant's stochastic-Hamiltonian exciton propagator.
 *
 * One time step of the reference is four calls on three objects
 * (propagate.cu:226-248):
 *     lanczosClass::doLanczos(psi_src)      lanczosClass.cu:232
 *     padeClass::doPade()                   padeClass.cu:206
 *     propagateSystem(sys, lan, pade, dest) propStep.cu:10
 *     systemClass::renormalizeAndStoreNorm  systemClass.cu:1771
 * preceded by systemClass::updateHamiltonian(t) (systemClass.cu:1883), and
 * followed by calculateErrorEstimate (systemClass.cu:2057).  dq_prop_step
 * below is that whole sequence as one stream-ordered call; dq_run is the
 * batched ensemble form of propagate.cu's run loop (propagate.cu:167-298).
 *
 * Conventions: every function returns dq_status (0 = DQ_OK);
 * dq_last_error(ctx) gives the message of the last failure.  Host arrays are
 * copied and stay owned by the caller.  A context is single-threaded; work is
 * ordered on the context's stream (dq_get_stream).  Units: energies cm^-1,
 * time fs.
 */
#ifndef DQ_H
#define DQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DQ_API __attribute__((visibility("default")))
#else
#define DQ_API
#endif

typedef struct dq_ctx dq_ctx;
typedef int dq_status;
typedef struct { double re, im; } dq_cdouble;

enum {
    DQ_OK = 0,
    DQ_ERR_ARG = 1,       /* invalid argument or size */
    DQ_ERR_CUDA = 2,      /* CUDA runtime error (allocation, launch) */
    DQ_ERR_BREAKDOWN = 3, /* Lanczos beta_j == 0 (lucky breakdown) */
    DQ_ERR_NAN = 4,       /* non-finite value or norm drift detected */
    DQ_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
    DQ_ERR_SCALING = 6,   /* Padé scaling s >= 50 (padeClass.cu:618-623) */
    DQ_ERR_STATE = 7,     /* call out of order (e.g. backward before forward) */
    DQ_ERR_SINGULAR = 8   /* Padé denominator singular (padeClass.cu:735-738) */
};

/* Noise on the diagonal site energies (includeFiles.cu:19-25). */
enum { DQ_NOISE_NONE = 0, DQ_NOISE_GAUSS = 1 /* SIM_TYPE_HSR */, DQ_NOISE_OU = 2 /* SIM_TYPE_KUBO_ANDERSON */,
       DQ_NOISE_ZZ = 3 /* SIM_TYPE_ZZ_REAL_NOISE */ };
/* Lanczos alpha: DQ_DOT_BILINEAR is the reference's unconjugated cublasZdotu
 * (lanczosClass.cu:421); DQ_DOT_HERMITIAN the Hermitian inner product. */
enum { DQ_DOT_BILINEAR = 0, DQ_DOT_HERMITIAN = 1 };
/* Padé scaling norm: DQ_NORM_REAL_ONLY sums |Re| as gpuPadeHelper.cu:25 does;
 * DQ_NORM_COMPLEX sums |.|. */
enum { DQ_NORM_REAL_ONLY = 0, DQ_NORM_COMPLEX = 1 };
/* Ensemble path precision: complex128 everywhere, or complex64 vectors with
 * FP64 Lanczos scalars and FP64 Padé. */
enum { DQ_PREC_FP64 = 0, DQ_PREC_MIXED = 1 };

typedef struct dq_config {
    int n_sites;            /* N */
    int m;                  /* Krylov dimension (2..32); the maximum when adaptive */
    int n_traj;             /* trajectories held by the context (B) */
    double dt;              /* fs */
    double hbar;            /* cm^-1 fs; <= 0 selects the reference's value (cppUtility.cpp:19-22) */
    int noise_model;        /* DQ_NOISE_* */
    int ka_substeps;        /* OU Euler-Maruyama substeps per step (ka_substeps key) */
    double sigma_static;    /* static disorder sigma (cm^-1), redrawn per trajectory */
    uint64_t seed;          /* Philox key */
    int dot_mode;           /* DQ_DOT_* */
    int norm_mode;          /* DQ_NORM_* */
    int precision;          /* DQ_PREC_*: ensemble path (dq_run) */
    int reorth;             /* 1: full reorthogonalisation (Hermitian dot only) */
    int pop_every;          /* record ensemble populations every k steps */
    int m_min;              /* adaptive Krylov dimension (ensemble path, dq_run): 0 = fixed m; else each
                               trajectory takes the first j = m_min, m_min + 4, ... below m whose
                               EXPOKIT term beta_j |E(j-1, j)| <= m_tol, or m (the plain path keeps m) */
    double m_tol;           /* adaptive Krylov dimension: tolerance (0 selects 1e-7) */
    int max_steps;          /* capacity of the correlation / population records */
    int device;             /* CUDA device ordinal; every call on the context makes it current for
                               its duration and gives the caller's current device back */
} dq_config;

/* Fills defaults: m 16, dt 1, reference hbar, no noise, 1 substep,
 * Hermitian dot, complex norm, mixed precision, pop_every 1, max_steps 1024. */
DQ_API void dq_config_default(dq_config *cfg);

DQ_API dq_status dq_create(const dq_config *cfg, dq_ctx **out);
DQ_API void dq_destroy(dq_ctx *ctx);
DQ_API const char *dq_last_error(const dq_ctx *ctx);
/* cudaStream_t the context orders its work on. */
DQ_API void *dq_get_stream(dq_ctx *ctx);

/* Hamiltonian as CSR including every diagonal entry (the reference requires
 * all diagonals for a fluctuating Hamiltonian, sparseMatrixClasses.cu:173-251).
 * Replaces matCooClass::readInFile + matCsrClass::pointToCooAndConvert +
 * systemClass::prepForNonConstHam (sparseMatrixClasses.cu:75-540,
 * systemClass.cu:810-870).  The diagonal becomes the static site energies;
 * off-diagonal couplings are stored once and shared by all trajectories. */
DQ_API dq_status dq_set_hamiltonian_csr(dq_ctx *ctx, int n, const int *rowptr, const int *col,
                                        const double *val);
/* Optional coupling classes: cls[k] in [0, n_classes) for the k-th
 * OFF-DIAGONAL entry of the CSR given to dq_set_hamiltonian_csr (CSR order,
 * diagonal entries skipped); that coupling is scaled by scales[cls[k]]. */
DQ_API dq_status dq_set_coupling_classes(dq_ctx *ctx, const int *cls, int n_classes, const double *scales);
/* Per-site noise parameters: sigma (cm^-1) and, for OU, tau (fs).
 * Replaces prepForKA / prepForHsr (systemClass.cu:912-1071). */
DQ_API dq_status dq_set_noise_params(dq_ctx *ctx, const double *sigma, const double *tau);
/* ZZ real noise (SIM_TYPE_ZZ_REAL_NOISE; prepForZZReal, systemClass.cu:1077-1207):
 * the spectral density's n_osc points omega (cm^-1) and J (cm^-1), spacing
 * d_omega and temperature (K).  Each site's diagonal at t = step dt is its
 * static energy plus sum_osc c cos(omega_fs t + phi), c = sqrt(2) sqrt(G d_omega
 * / pi), G = J / (1 - exp(-omega / (k_B T))), omega_fs = omega / 5308.84, with
 * phases drawn per trajectory, site and oscillator (Philox; the reference
 * redraws them per run, systemClass.cu:1212-1234). */
DQ_API dq_status dq_set_zz_spectral_density(dq_ctx *ctx, int n_osc, const double *omega, const double *J,
                                            double d_omega, double temperature);
/* Taylor-Krylov propagation (PROP_MODE_TAYLOR_LANCZOS; taylorKrylovClass.cu:
 * 135-434, replaces the taylorKrylovClass constructor and the auxiliary
 * matrix file): each step is psi <- sum_{k<p} tau^k/k! A^k psi +
 * ||A^p psi|| Q_B [exp(tau Tbar_B)]_{:, L-1}, A the step's Hamiltonian,
 * Q_B and Tbar_B (size L = m_b + p, EXPOKIT's phi_p augmentation) from m_b
 * Lanczos iterations on the auxiliary matrix B (full CSR over the N sites,
 * diagonal included) started from A^p psi, then renormalised; the error
 * estimate is EXPOKIT's on the B part plus |1 - norm|.  2 <= p, 1 <= m_b <= 32,
 * m_b + p <= 34; p = 0 returns to Lanczos mode.  Steps run in FP64 on the
 * per-trajectory path (dq_prop_step, dq_run_plain) and, for dq_run, on an
 * ensemble path that advances all trajectories together; groups and the
 * adjoint refuse this mode. */
DQ_API dq_status dq_set_taylor_krylov(dq_ctx *ctx, int p, int m_b, const int *rowptr, const int *col,
                                      const double *val);
/* Inverse participation ratio (print_partic; systemClass.cu:2219-2257):
 * when enabled, every path adds 1 / sum_i |psi_i|^4 of each trajectory's
 * state after every step (and of psi0) into a per-step sum, kept in FP64
 * (the reference rounds sum |psi|^4 to float).  Takes effect at the next
 * reset. */
DQ_API dq_status dq_set_ipr(dq_ctx *ctx, int enable);
/* steps done + 1 values: the ensemble mean of 1 / sum |psi(k)|^4, k = 0.. */
DQ_API dq_status dq_get_ipr(dq_ctx *ctx, double *out, int *n_values);
/* The bra of the correlation M(t) = sum_i conj(bra_i) psi_i(t) (N complex,
 * host), replacing psi0: the CD spectrum's transition-dipole bra with the
 * R x mu initial state (spectraClass.cu:464-496, calcCorrFunc :505-571).  As
 * in the reference, M(0) is then recorded as 1 for every trajectory
 * (spectraClass.cu:296).  NULL returns to <psi0|psi(t)>.  The adjoint refuses
 * a separate bra.  Takes effect at the next reset. */
DQ_API dq_status dq_set_correlation_bra(dq_ctx *ctx, const dq_cdouble *bra);
/* ---- ensembles sharded over processes / GPUs (no reference counterpart;
 * the reference runs numEnsembleRuns one after another, propagate.cu:167-298) ----
 * Index of this context's trajectory 0 in the whole ensemble (even, >= 0):
 * every random draw of local trajectory b is keyed by traj0 + b, so shards
 * [r B, (r+1) B) over ranks r reproduce one ensemble of world x B
 * trajectories.  Takes effect at the next reset. */
DQ_API dq_status dq_set_trajectory_offset(dq_ctx *ctx, int traj0);
/* Raw observable SUMS over this context's trajectories (not divided):
 * populations (steps/pop_every + 1) x N, correlation steps + 1 complex and,
 * when enabled, IPR steps + 1 (each pointer may be NULL). */
DQ_API dq_status dq_get_observable_sums(dq_ctx *ctx, double *pops, dq_cdouble *corr, double *ipr);
/* Replaces the observable sums by ones reduced over all shards (same
 * shapes; ipr may be NULL) standing for n_traj_total trajectories: the
 * getters and file writers then report the whole ensemble.  dq_run refuses
 * to continue until dq_reset. */
DQ_API dq_status dq_set_observable_sums(dq_ctx *ctx, const double *pops, const dq_cdouble *corr, const double *ipr,
                                        int n_traj_total);
/* Explicit static site energies shared by all trajectories (replaces the
 * Hamiltonian diagonal plus static disorder); NULL restores them. */
DQ_API dq_status dq_set_static_energies(dq_ctx *ctx, const double *eps);
/* Initial state (host, N complex); replaces setInitState /
 * initStateAsBasisVector / spectraClass::prepInitState. */
DQ_API dq_status dq_set_initial_state(dq_ctx *ctx, const dq_cdouble *psi0);
/* Initial state from one polarisation direction's transition dipoles (host,
 * N real): psi0 = mu / |mu| (spectraClass.cu:440-458, the absorption run's
 * state; its correlation is then <mu/|mu| | psi(t)>). */
DQ_API dq_status dq_set_initial_dipole(dq_ctx *ctx, const double *mu);
/* Redraws static disorder and OU offsets for every trajectory, sets every
 * trajectory to psi0 and clears the observable records (prepAnalysesForNextRun,
 * systemClass.cu:1554-1608). */
DQ_API dq_status dq_reset(dq_ctx *ctx);

/* ---- plain FP64 per-trajectory form: the drop-in for propStep ---- */
/* One step of trajectory `traj` at step index `step`: noise update of that
 * trajectory's diagonal, m-step Lanczos, Padé exp, psi_out = V exp(tau T) e1,
 * renormalisation.  psi_in/psi_out are DEVICE pointers to N complex128
 * (may not alias).  If err_est is non-NULL the call synchronises and writes
 * the EXPOKIT error estimate there.  Steps of a trajectory must be issued in
 * order (its OU offsets advance with each call). */
DQ_API dq_status dq_prop_step(dq_ctx *ctx, int traj, int step, const dq_cdouble *psi_in_dev,
                              dq_cdouble *psi_out_dev, double *err_est);
/* Runs every trajectory through dq_prop_step's kernels one after another for
 * n_steps, accumulating populations / correlation / error on the device. */
DQ_API dq_status dq_run_plain(dq_ctx *ctx, int n_steps);

/* Allocation-free Krylov step; this entry point has no counterpart in the
 * reference.  For callers that cannot allocate device memory while they step
 * (an application whose own pool owns all device memory and forbids
 * cudaMalloc/cudaFree inside its time loop, or a framework that only hands
 * out buffers it manages): it needs no dq_ctx and allocates nothing.  One
 * step psi_out = exp(-i H dt/hbar) psi_in by m-step Lanczos + Padé + renorm
 * for H = diag + offdiag, where rowptr/col/val is the OFF-DIAGONAL CSR and
 * diag this step's diagonal; every pointer is DEVICE memory owned by the
 * caller (psi_in and psi_out may not alias).  psi_in must have unit norm: it
 * is the first Krylov vector as given, as dq_prop_step and the reference's
 * step take it (psi_out is renormalised to unit norm).  Work is ordered on `stream`
 * (a cudaStream_t, NULL = legacy default stream).  Scratch is one static
 * 16 MiB device array per GPU (held until process exit), so it accepts
 * (m+3)*n*16 bytes + ~70 KB <= 16 MiB (about 55,000 sites at m = 16) and
 * returns DQ_ERR_ARG with the reason in errbuf beyond that.  The first call
 * on a device looks up the array's device address and should come before
 * any stream capture.  All calls on a device share the array (each clears
 * what must start at zero): calls that overlap on the GPU race.  If err_est
 * is non-NULL the call synchronises `stream`, writes the EXPOKIT error
 * estimate and returns the device status (breakdown, non-finite value, Padé
 * scaling).  With err_est == NULL the call does not synchronise and cannot
 * report a device error itself: the error stays recorded in the array and the
 * next call on the device that passes err_est returns it (and clears it).
 * errbuf (may be NULL) receives a message on failure. */
DQ_API dq_status dq_krylov_step_static(int n, const int *rowptr, const int *col, const double *val,
                                       const double *diag, const dq_cdouble *psi_in, dq_cdouble *psi_out, int m,
                                       double dt, double hbar, int dot_mode, int norm_mode, void *stream,
                                       double *err_est, char *errbuf, int errbuf_len);

/* ---- batched ensemble form ---- */
/* Advances all trajectories by n_steps with the configured precision
 * (shared-structure SpMM Lanczos over all trajectories, batched FP64 Padé,
 * fused combine/observables), the step loop captured in a CUDA graph. */
DQ_API dq_status dq_run(dq_ctx *ctx, int n_steps);

/* Tiling of the ensemble kernels: traj_chunk trajectories per CTA column
 * (a power of two dividing n_traj, <= 64), vec 1 or 2 complex values per
 * thread (8- or 16-byte loads; 1 in FP64), about ctas_per_sm CTAs per SM,
 * each owning a contiguous range of sites, and rows_per_block (1, 2, 4 or 8)
 * rows computed together by the SpMM over the union of their neighbour
 * columns.  staged = 1 stages the gathered trajectory rows in a shared-memory
 * window filled by TMA (needs the matrix bandwidth to fit the window; the
 * call fails otherwise), 0 gathers through L1, 2 runs each Lanczos iteration
 * as one fused kernel (TMA-streamed w, r_j, r_{j-1}; r_{j+1} formed in a
 * shared-memory ring and gathered from there; groups must be 1), 3 gathers
 * through L1 with one warp per row block (records fetched 32 at a time;
 * complex64, traj_chunk = 32 vec), 4 is the fused form with warp-owned row
 * blocks (complex64, traj_chunk = 32 vec, ctas_per_sm 1), 5 is the L1 form
 * in 512-thread CTAs (one sliding gather window per CTA), 6 gathers from a
 * TMA-fed shared-memory ring with warp-owned row blocks and 2 trajectories
 * per lane, 7 the same ring with 4 trajectories per lane (both complex64,
 * traj_chunk 32, vec 2, ctas_per_sm 1, rows_per_block <= 3), 8 runs each
 * Lanczos iteration as one L1-gather launch without the axpy pass (it keeps
 * p_j = H q_{j-1} - beta_{j-2} q_{j-2} instead of the residual and gathers
 * that; 512-thread CTAs; groups 1, no reorthogonalisation or adaptive m), 9
 * is form 5 with its gathers issued as asynchronous copies into per-warp
 * shared-memory rings (complex64, traj_chunk 64, vec 2, ctas_per_sm 1,
 * rows_per_block <= 3, at most 128 union entries per block), 10 is form 5
 * with one warp per row block, its records in a per-warp shared buffer and
 * eight gathers in flight per warp (complex64, traj_chunk 64, vec 2,
 * ctas_per_sm 1, rows_per_block <= 3), 11 is form 10 with the axpy in the
 * same launch: a cooperative launch in which each CTA waits (bounded) for its
 * chunk's alpha_j and then forms r_{j+1} for its own rows while w and q_j are
 * still in L2 (no reorthogonalisation or adaptive m), 12 is the L1 form at
 * 32 warps per SM and at most 64 registers a thread (complex64, vec 2,
 * rows_per_block <= 3; ctas_per_sm 1: one 1024-thread CTA per SM, 2: two
 * 512-thread CTAs).  groups splits the trajectory chunks
 * into groups whose m Lanczos iterations run one group after another, so a
 * group's Krylov slabs stay resident in L2 (must divide n_traj / traj_chunk).  Changing it restarts the ensemble at the next dq_run
 * (as dq_reset does). */
DQ_API dq_status dq_set_tiling(dq_ctx *ctx, int traj_chunk, int vec, int ctas_per_sm, int rows_per_block,
                               int staged, int groups);
DQ_API dq_status dq_get_tiling(dq_ctx *ctx, int *traj_chunk, int *vec, int *ctas_per_sm, int *rows_per_block,
                               int *staged, int *groups);
/* Times one Lanczos iteration (SpMM + axpy) of the current system under
 * every valid tiling, keeps the fastest and resets the ensemble.  best_ms
 * (may be NULL) gets its time per iteration. */
DQ_API dq_status dq_autotune(dq_ctx *ctx, int reps, double *best_ms);
/* Mean device time of one Lanczos iteration (SpMM + axpy) under the current
 * tiling, over reps launches; the ensemble restarts at the next dq_run. */
DQ_API dq_status dq_time_iteration(dq_ctx *ctx, int reps, double *ms);
/* Measurement, no reference counterpart: mean device time of one launch of
 * the gathers alone of the current tiling's packed coupling blocks (complex64,
 * vec 2, rows_per_block <= 3): the same row-block walk, record stream and
 * 16-byte gathers of the trajectory rows as the L1-gather SpMM, without its
 * FMAs, diagonal, q_{j-1} term, alpha and all but one store per block, over
 * the chunks of one SpMM launch (one chunk group); the floor that access
 * pattern sets on the GPU.  Overwrites the ensemble's work
 * slab (the ensemble restarts at the next dq_run); DQ_ERR_STATE for other
 * tilings. */
DQ_API dq_status dq_time_gather_floor(dq_ctx *ctx, int reps, double *ms);
/* Test hook, no reference counterpart: sets the budget (SM cycles) of the
 * bounded shared-memory barrier waits of the TMA-fed SpMM forms on the
 * context's device; 0 restores the default (about 2 s).  A negative value
 * makes every CTA of the ring form (staged 6/7) first wait -cycles cycles on
 * a barrier that no copy ever completes: the wait runs out, the kernel
 * records DQ_ERR_TIMEOUT, lets its own copies in flight land (with the
 * default budget) and returns, and dq_run reports the status.  The same
 * budget bounds the per-chunk wait for alpha of the cooperative iteration
 * form (staged 11); a negative value makes that wait look -cycles cycles for
 * a generation that never comes, with the same outcome.  It applies to every
 * context on the device until changed again. */
DQ_API dq_status dq_debug_set_wait_cycles(dq_ctx *ctx, int cycles);

/* Kernel kinds of one ensemble step, for dq_profile_step. */
enum {
    DQ_KIND_NOISE = 0,      /* OU / Gaussian diagonal update */
    DQ_KIND_SPMM = 1,       /* SpMM w = H q_j fused with alpha_j */
    DQ_KIND_AXPY = 2,       /* r_{j+1} = w - alpha q_j - beta q_{j-1}, beta_j */
    DQ_KIND_SPMM_NORM = 3,  /* ||H q_{m+1}|| for the error estimate */
    DQ_KIND_PADE = 4,       /* batched Padé exponential */
    DQ_KIND_COMBINE = 5,    /* psi = V y, norms, correlation */
    DQ_KIND_POP = 6,        /* population record */
    DQ_KIND_FUSED = 7,      /* fused iteration: r_j, SpMM H r_j, beta_{j-1}, alpha_j (staged = 2) */
    DQ_KIND_COUNT = 8
};
/* Advances all trajectories by n_steps exactly like dq_run, but launches the
 * step's kernels eagerly with CUDA events between them; ms_per_launch[k]
 * receives the mean device time of one launch of kind k (n_kinds entries,
 * up to DQ_KIND_COUNT) and launches[k] their count (may be NULL). */
DQ_API dq_status dq_profile_step(dq_ctx *ctx, int n_steps, double *ms_per_launch, int *launches, int n_kinds);

/* ---- observables (host outputs, caller-owned) ---- */
/* Ensemble-averaged populations, records at steps 0, pop_every, ...:
 * (*n_records) x N doubles. Pass out = NULL to query n_records. */
DQ_API dq_status dq_get_populations(dq_ctx *ctx, double *out, int *n_records);
/* Ensemble-averaged <psi0|psi(t_k)> for k = 0..steps done (spectraClass.cu:510-571). */
DQ_API dq_status dq_get_correlation(dq_ctx *ctx, dq_cdouble *out, int *n_points);
/* Current normalised states, n_traj x N complex128. */
DQ_API dq_status dq_get_states(dq_ctx *ctx, dq_cdouble *out);
/* Accumulated EXPOKIT error per trajectory (systemClass.cu:2057-2085). */
DQ_API dq_status dq_get_error_accum(dq_ctx *ctx, double *out);
/* Steps done since dq_reset. */
DQ_API int dq_steps_done(const dq_ctx *ctx);
/* Static energies and OU offsets (FP64, N each) of one trajectory in the
 * path that ran last; the step's diagonal is eps + deps for OU noise.  The
 * counterpart of the reference's debug_diags dump (propagate.cu:214-223).
 * Either pointer may be NULL. */
DQ_API dq_status dq_get_noise_state(dq_ctx *ctx, int traj, double *eps, double *deps);

/* Inverse DFT (cuFFT INVERSE convention, unnormalised) of the first
 * n_in correlation points zero-padded to len (a power of two), on the GPU.
 * Replaces spectraClass::singleSpectraCalc's cufftExecZ2Z (spectraClass.cu:621). */
DQ_API dq_status dq_get_spectrum(dq_ctx *ctx, int len, dq_cdouble *out);
/* Optional Gaussian line-shape dressing (lineShapeDressing /
 * gaussLineshapeWidth; spectraClass.cu:583-600, gpuSpectraHelper.cu:16-42):
 * before every transform (dq_get_spectrum, dq_write_spectrum[_mean]) the
 * ensemble-mean correlation point k < steps is multiplied by
 * exp(-(dt (k + 1) / sigma)^2 / 2), the time offset by one step as in the
 * reference; the correlation file shows the dressed values.  sigma in fs;
 * 0 turns it off. */
DQ_API dq_status dq_set_line_dressing(dq_ctx *ctx, double sigma_fs);

/* ---- the reference's output files ---- */
/* pops.dat of popPrintClass (popPrintClass.cu:160-522): header numsims / dt /
 * totalsteps / numprintedsites (text lines, or int/double/int/int in binary),
 * then for every recorded step s >= 1 ("STEP s" in text) each site's SUM of
 * |psi|^2 over the runs (text "%25.17g (site)").  numsims is the number of
 * trajectories summed.  continuation = 1 adds the sums of the existing file
 * at path (same dt, totalsteps, sites; numsims accumulates); the file is
 * written as temp_<name> beside it and renamed over it.  With pop_every = 1
 * the step lines are the reference's every step. */
DQ_API dq_status dq_write_populations(dq_ctx *ctx, const char *path, int binary, int continuation);
/* folder/_states_<t>.dat of statePrintClass (statePrintClass.cu:82-199) for
 * the current step: float t = dt * steps done, int N, int n_traj, then every
 * trajectory's normalised state (N complex128). */
DQ_API dq_status dq_write_states(dq_ctx *ctx, const char *folder);
/* The correlation and spectrum text files of spectraClass (spectraClass.cu:
 * 621-690) for the ensemble-mean correlation of the steps done: transform
 * length steps + 1, frequency index wrapped above steps/2, rev/fs and cm^-1
 * axes (c = 299792458 m/s), values scaled by `scaling` held as a float (the
 * caller passes mu_tot^2 for absorption or (pi/2) 1e-7 mu_tot RD_tot for CD),
 * the transform also divided by the step count. */
DQ_API dq_status dq_write_spectrum(dq_ctx *ctx, const char *corr_path, const char *spec_path, double scaling);
/* The overall files over polarisation directions (spectraClass.cu:697-744):
 * the mean of n_ctx contexts' scaled correlations and transforms (one
 * context per direction, scalings[k] as for dq_write_spectrum); the contexts
 * must have the same steps done and dt. */
DQ_API dq_status dq_write_spectrum_mean(dq_ctx *const *ctxs, int n_ctx, const double *scalings, const char *corr_path,
                                        const char *spec_path);
/* invParticRat.dat (systemClass.cu:1735-1750): "# Inverse Particle Ratios",
 * "# {timestep} {IPR}}", then "k  IPR_k" (%g) for k = 0..steps-1, IPR_k the
 * ensemble mean from dq_get_ipr.  Needs dq_set_ipr(ctx, 1) before the run. */
DQ_API dq_status dq_write_ipr(dq_ctx *ctx, const char *path);

/* ---- several aggregates together (no reference counterpart) ----
 * A group advances the ensembles of several contexts (aggregates of any
 * size and trajectory count, on one device) by the same number of steps:
 * each group step is one CUDA graph with one concurrent branch per member,
 * so small aggregates run beside large ones.  Members keep their own
 * settings (tiling, adaptive Krylov dimension, noise) and observables. */
typedef struct dq_group dq_group;
DQ_API dq_status dq_group_create(dq_ctx *const *members, int n_members, dq_group **out);
DQ_API void dq_group_destroy(dq_group *group);
DQ_API const char *dq_group_last_error(const dq_group *group);
/* Advances every member by n_steps (as dq_run does for one context). */
DQ_API dq_status dq_group_run(dq_group *group, int n_steps);
/* dq_group_run that also gives the device time of the n_steps graph
 * launches in *device_ms (events on the group's stream; the capture of the
 * step graph is excluded). */
DQ_API dq_status dq_group_run_timed(dq_group *group, int n_steps, double *device_ms);

/* ---- adjoint: gradient of a spectrum-fitting loss ----
 * No counterpart in the reference (it has no gradients).  The loss is
 *   L = sum_j (scale * Re(S_j) - target_j)^2,  j = 0..fft_len-1,
 * with S the unnormalised inverse DFT (dq_get_spectrum's convention) of the
 * ensemble-mean correlation Cbar(k) = <psi0|psi(k)>, k = 0..n_steps,
 * zero-padded to fft_len (a power of two).  The gradient is taken with
 * respect to the site energies (the diagonal of the input Hamiltonian, or the
 * explicit static energies; N values) and the coupling-class scales of
 * dq_set_coupling_classes (one implicit class of scale 1 when none are set).
 * The backward pass runs the adjoint recursion lambda(k) = s_k +
 * exp(-i dt H_k/hbar) lambda(k+1) with its own Lanczos basis per step and the
 * exponential's Fréchet derivative from the block-triangular exponential of
 * the two tridiagonal matrices (Van Loan).  Requires dot_mode
 * DQ_DOT_HERMITIAN, m <= 24, n_traj a multiple of 8, at most 8 coupling
 * classes and a normalised initial state. */
/* Fixes the loss.  target: fft_len host doubles.  checkpoint_every: steps per
 * recomputed segment (0 = automatic: keep every step's state and diagonal
 * resident when they fit in about half of the free device memory, else about
 * sqrt(n_steps)); states at segment starts are kept, the rest is recomputed
 * by the backward pass. */
DQ_API dq_status dq_adjoint_setup(dq_ctx *ctx, int n_steps, int fft_len, double scale, const double *target,
                                  int checkpoint_every);
/* Resets the ensemble and runs the n_steps of dq_adjoint_setup, keeping what
 * the backward pass needs; *loss (may be NULL) receives L.  Populations and
 * correlation are recorded as by dq_run. */
DQ_API dq_status dq_forward(dq_ctx *ctx, double *loss);
/* Gradient of the last dq_forward's loss: grad_sites (N host doubles) and
 * grad_classes (one per coupling class, or one for the implicit class; may
 * be NULL).  Overwrites the
 * ensemble's current states (the next dq_run starts from dq_reset). */
DQ_API dq_status dq_backward(dq_ctx *ctx, double *grad_sites, double *grad_classes);
/* The same gradient for an ensemble sharded over contexts (one per rank,
 * dq_set_trajectory_offset; no reference counterpart).  dq_forward_shard runs
 * this context's trajectories and returns its raw correlation sums (steps + 1
 * complex, host); after the caller sums them over all shards,
 * dq_forward_reduced installs the sums of the whole ensemble of n_traj_total
 * trajectories, computes the loss of its mean (*loss, may be NULL) and
 * prepares dq_backward, whose gradients are then this shard's part: their
 * sum over the shards is the gradient of the whole ensemble's loss. */
DQ_API dq_status dq_forward_shard(dq_ctx *ctx, dq_cdouble *corr_sums);
DQ_API dq_status dq_forward_reduced(dq_ctx *ctx, const dq_cdouble *corr_sums, int n_traj_total, double *loss);

#ifdef __cplusplus
}
#endif
#endif /* DQ_H */
