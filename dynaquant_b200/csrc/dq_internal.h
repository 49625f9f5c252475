// dq_internal.h — the context behind the C ABI (include/dq.h).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/dq.h"
#include "dq_common.cuh"
#include "dq_pade.cuh"

namespace dq {

// Scalars of the plain per-trajectory path (device resident).
struct PlainScalars {
    cd alpha[kMaxL];
    cd beta[kMaxL];
    double sc[kMaxL];     // slab j holds q_j / sc[j] (unnormalised Lanczos residual)
    cd yt[kMaxL];         // y_{j-1} * sc[j]: combine weights
    double nav;           // ||H q_{m+1}||
    double norm;          // ||psi_out|| before renormalisation
    double invnorm;
    double err;           // EXPOKIT estimate of the last step
    int s;                // Padé squarings of the last step
    int status;           // DQ_OK or a DQ_ERR_* code raised on the device
    unsigned int ticket[4];
    cd h[kMaxL];          // full reorthogonalisation: <q_k, r_{j+1}>
    unsigned int ticket_r[2];
    double tk_beta0;      // Taylor-Krylov: ||A^p psi_in||
    double tk_kerr;       // Taylor-Krylov: EXPOKIT estimate of the B part
};

constexpr int kPlainThreads = 256;
constexpr int kMaxPartials = 4096;
constexpr int kMaxZZOsc = 1024;   // oscillators of one ZZ spectral density
constexpr int kIprRowGroups = 296; // row groups of the ensemble IPR reduction (2 per SM)

struct BatchedState;   // dq_batched.cu
struct TkEnsemble;     // dq_tk_ensemble.cu
struct AdjointState;   // dq_adjoint.cu

}  // namespace dq

struct dq_ctx {
    dq_config cfg{};
    std::string err;
    cudaStream_t stream = nullptr;
    double hbar = 0.0;
    double tau_im = 0.0;  // tau = (0, tau_im) = -i dt / hbar

    // host copies of the system
    int n = 0;
    std::vector<int> rowptr, col;          // off-diagonal CSR
    std::vector<double> val_base, val;     // couplings before / after class scaling
    std::vector<int> cls;                  // coupling class per off-diagonal entry
    std::vector<double> scales;
    std::vector<double> h0diag;
    std::vector<double> sigma, tau;
    std::vector<double> static_eps;        // explicit static energies (empty = h0 + disorder)
    std::vector<dq_cdouble> psi0;
    bool have_ham = false, have_noise = false, have_psi0 = false, ready = false;

    // device: shared structure
    int* d_rowptr = nullptr;
    int* d_col = nullptr;
    double* d_val = nullptr;
    double* d_h0 = nullptr;
    double* d_static = nullptr;            // explicit static energies (or null)
    double* d_sigma = nullptr;
    double* d_invtau = nullptr;
    double* d_coeff = nullptr;
    dq::cd* d_psi0 = nullptr;
    dq::cd* d_bra = nullptr;               // correlation bra (null: psi0)
    int nnz_off = 0;
    bool rows_sorted = false;              // every off-diagonal row's columns non-decreasing
    int bw = 0;                            // bandwidth max |col - row| of the off-diagonal CSR
    // ZZ real noise: oscillators (angular frequency rad/fs, amplitude); the
    // phases are Philox draws made where they are used
    int zz_n_osc = 0;
    std::vector<double> zz_omega, zz_coeff;
    double* d_zz_omega = nullptr;
    double* d_zz_coeff = nullptr;

    // plain path: per trajectory state [traj][site], work buffers
    double* d_eps_p = nullptr;
    double* d_deps_p = nullptr;
    double* d_diag = nullptr;
    dq::cd* d_Q = nullptr;        // (m+2) slabs of n
    dq::cd* d_w = nullptr;
    dq::cd* d_psi_a = nullptr;    // ensemble driver ping-pong states
    dq::cd* d_psi_b = nullptr;
    double* d_partial = nullptr;  // kMaxPartials x 2
    dq::PlainScalars* d_ps = nullptr;

    // observables (sums over trajectories; divided by n_traj on read)
    int n_rec_max = 0;
    double* d_pops = nullptr;     // n_rec_max x n
    dq::cd* d_corr = nullptr;     // max_steps + 1
    double* d_erracc = nullptr;   // n_traj
    int steps_done = 0;
    int plain_traj_done = 0;      // trajectories completed by dq_run_plain
    int last_path = 0;            // 0: dq_run_plain, 1: dq_run, 2: reduced sums set, 3: Taylor-Krylov dq_run
    int traj0 = 0;                // index of trajectory 0 in the whole (sharded) ensemble: the Philox key
    int obs_traj = 0;             // trajectories behind the observable sums when set from a reduction
    double dress_sigma = 0.0;     // Gaussian line-shape dressing of M(t) before transforms (fs; 0 = off)

    // Taylor-Krylov mode (tk_p > 0): the auxiliary matrix B (off-diagonal
    // CSR + diagonal), its Krylov basis and the Taylor work vectors
    int tk_p = 0, tk_m = 0;
    int* d_tk_rowptr = nullptr;
    int* d_tk_col = nullptr;
    double* d_tk_val = nullptr;
    double* d_tk_diag = nullptr;
    dq::cd* d_tk_Q = nullptr;     // (tk_m + 2) slabs of n; slab 1 holds A^p psi
    dq::cd* d_tk_x = nullptr;     // 2 slabs: A^k psi ping-pong
    dq::cd* d_tk_acc = nullptr;   // Taylor sum
    std::vector<dq::cd> tk_coef;  // tau^k / k!, k < p

    // inverse participation ratio (sums over trajectories of 1 / sum |psi|^4)
    bool ipr_on = false;
    double* d_ipr = nullptr;            // max_steps + 1
    double* d_ipr_partial = nullptr;    // kIprRowGroups x n_traj
    unsigned int* d_ipr_ticket = nullptr;

    dq::BatchedState* bat = nullptr;
    dq::AdjointState* adj = nullptr;
    dq::TkEnsemble* tke = nullptr;   // ensemble workspace of Taylor-Krylov mode
};

namespace dq {
// The bra of the correlation M(t) = <bra|psi(t)>: psi0 unless one was set.
inline const cd* corr_bra(const dq_ctx* c) { return c->d_bra ? c->d_bra : c->d_psi0; }

// Makes a context's device current for the length of one entry point and gives
// the caller's current device back on return, so contexts on several GPUs can
// be driven from one thread in any order (no synchronisation involved).
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int device) {
        int cur = -1;
        if (device < 0 || cudaGetDevice(&cur) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        if (cur == device) return;
        if (cudaSetDevice(device) == cudaSuccess) prev = cur;
        else cudaGetLastError();
    }
    explicit DeviceScope(const dq_ctx* c) : DeviceScope(c ? c->cfg.device : -1) {}
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Trajectories the observable sums stand for (their divisor for means).
inline int observed_trajectories(const dq_ctx* c) {
    if (c->obs_traj > 0) return c->obs_traj;
    return (c->last_path == 0 && c->plain_traj_done > 0) ? c->plain_traj_done : c->cfg.n_traj;
}

// implemented in dq_plain.cu
dq_status plain_alloc(dq_ctx* c);
void plain_free(dq_ctx* c);
dq_status plain_traj_init(dq_ctx* c);
dq_status plain_step(dq_ctx* c, int traj, int step, const cd* psi_in, cd* psi_out, bool observe, int rec);
dq_status plain_clear_observables(dq_ctx* c);
dq_status plain_observe_initial(dq_ctx* c);
dq_status check_cuda(dq_ctx* c, cudaError_t e, const char* what);
dq_status read_status(dq_ctx* c, int code, const char* what);
// implemented in dq_batched.cu
// default_tiling = false leaves the tiling unset (TC = 0) for a caller that
// sets one at once (batched_set_tiling, or batched_default_tiling)
dq_status batched_alloc(dq_ctx* c, bool default_tiling = true);
dq_status batched_default_tiling(dq_ctx* c);
void batched_free(dq_ctx* c);
dq_status batched_reset(dq_ctx* c);
dq_status batched_run(dq_ctx* c, int n_steps);
dq_status batched_enqueue_step(dq_ctx* c);
dq_status batched_read_status(dq_ctx* c);
dq_status batched_get_states(dq_ctx* c, dq_cdouble* out);
dq_status batched_collect_corr(dq_ctx* c);
dq_status batched_profile(dq_ctx* c, int n_steps, double* ms, int* cnt, int nk);
dq_status batched_set_tiling(dq_ctx* c, int tc, int tpt, int ctas_per_sm, int R, int staged, int groups);
void batched_get_tiling(dq_ctx* c, int* tc, int* tpt, int* cps, int* R, int* staged, int* groups);
dq_status batched_invalidate_blocks(dq_ctx* c);
dq_status batched_time_iteration(dq_ctx* c, int reps, double* ms);
dq_status batched_time_gather_floor(dq_ctx* c, int reps, double* ms);
dq_status batched_set_wait_cycles(dq_ctx* c, int cycles);
void batched_noise_arrays(dq_ctx* c, const double** eps, const double** deps);
// kernels of dq_batched.cu also launched by the Taylor-Krylov ensemble
__global__ void k_traj_init_b(int n, int B, int traj0, uint64_t seed, const double* h0, const double* static_eps,
                              double sigma_static, const double* sigma, int noise, double* eps, double* deps);
// implemented in dq_tk_ensemble.cu
dq_status tk_ensemble_reset(dq_ctx* c);
dq_status tk_ensemble_run(dq_ctx* c, int n_steps);
dq_status tk_ensemble_states(dq_ctx* c, dq_cdouble* out);
void tk_ensemble_free(dq_ctx* c);
// implemented in dq_fft.cu
// M(k) *= exp(-(dt (k + 1) / sigma)^2 / 2) for k < n_dress (spectraClass.cu:583-600)
dq_status dress_correlation(dq_ctx* c, int n_dress, cd* x);
dq_status fft_inverse(dq_ctx* c, int len, const cd* in, int n_in, double scale, cd* out);
// implemented in dq_adjoint.cu
void adjoint_free(dq_ctx* c);
}  // namespace dq
