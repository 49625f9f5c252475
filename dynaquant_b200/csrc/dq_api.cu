// dq_api.cu — the C ABI (include/dq.h): context life cycle, system set-up,
// the plain drop-in step, the ensemble drivers and the observable getters.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <utility>

#include "dq_internal.h"

using namespace dq;

namespace {

double reference_hbar() {
    // cppUtility.cpp:19-22, including the reference's c = 299792548 m/s
    double pi = atan(1.0) * 4.0;
    double lightspeed = 299792548.;
    return (1 / 100.) * (1e15) * 1. / (lightspeed * 2 * pi);
}

dq_status fail(dq_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define DQ_CU(call)                                                     \
    do {                                                                \
        dq_status _s = check_cuda(c, (call), #call);                    \
        if (_s != DQ_OK) return _s;                                     \
    } while (0)

template <typename T>
dq_status upload(dq_ctx* c, T** dptr, const T* host, size_t count) {
    if (*dptr) { cudaFree(*dptr); *dptr = nullptr; }
    if (count == 0) return DQ_OK;
    DQ_CU(cudaMalloc(dptr, sizeof(T) * count));
    DQ_CU(cudaMemcpyAsync(*dptr, host, sizeof(T) * count, cudaMemcpyHostToDevice, c->stream));
    DQ_CU(cudaStreamSynchronize(c->stream));
    return DQ_OK;
}

dq_status upload_couplings(dq_ctx* c) {
    c->val.resize(c->val_base.size());
    for (size_t k = 0; k < c->val_base.size(); ++k) {
        double s = 1.0;
        if (!c->cls.empty()) s = c->scales[c->cls[k]];
        c->val[k] = s * c->val_base[k];
    }
    dq_status st = batched_invalidate_blocks(c);
    if (st) return st;
    return upload(c, &c->d_val, c->val.data(), c->val.size());
}

}  // namespace

extern "C" {

void dq_config_default(dq_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->m = 16;
    cfg->n_traj = 1;
    cfg->dt = 1.0;
    cfg->hbar = 0.0;
    cfg->noise_model = DQ_NOISE_NONE;
    cfg->ka_substeps = 1;
    cfg->dot_mode = DQ_DOT_HERMITIAN;
    cfg->norm_mode = DQ_NORM_COMPLEX;
    cfg->precision = DQ_PREC_MIXED;
    cfg->pop_every = 1;
    cfg->max_steps = 1024;
}

dq_status dq_create(const dq_config* cfg, dq_ctx** out) {
    if (!cfg || !out) return DQ_ERR_ARG;
    *out = nullptr;
    if (cfg->n_sites < 2 || cfg->m < 2 || cfg->m > kMaxM || cfg->n_traj < 1 || !(cfg->dt > 0) ||
        cfg->pop_every < 1 || cfg->max_steps < 1 || cfg->ka_substeps < 0 ||
        cfg->noise_model < DQ_NOISE_NONE || cfg->noise_model > DQ_NOISE_ZZ ||
        (cfg->reorth && cfg->dot_mode != DQ_DOT_HERMITIAN) || cfg->m > cfg->n_sites ||
        cfg->m_min < 0 || cfg->m_min > cfg->m || (cfg->m_min > 0 && cfg->m_min < 2) || cfg->m_tol < 0)
        return DQ_ERR_ARG;
    if ((cfg->n_sites + kPlainThreads - 1) / kPlainThreads > kMaxPartials) return DQ_ERR_ARG;
    dq_ctx* c = new (std::nothrow) dq_ctx();
    if (!c) return DQ_ERR_CUDA;
    c->cfg = *cfg;
    if (c->cfg.ka_substeps == 0) c->cfg.ka_substeps = 1;
    c->n = cfg->n_sites;
    c->hbar = cfg->hbar > 0 ? cfg->hbar : reference_hbar();
    c->tau_im = -cfg->dt / c->hbar;   // propagate.cu:90-93: expCoeff = (0, -dt/hbar)
    dq_status st = DQ_OK;
    int prev_device = -1;
    if (cudaGetDevice(&prev_device) != cudaSuccess) {
        cudaGetLastError();
        prev_device = -1;
    }
    do {
        if ((st = check_cuda(c, cudaSetDevice(cfg->device), "cudaSetDevice"))) break;
        if ((st = check_cuda(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream"))) break;
        c->n_rec_max = cfg->max_steps / cfg->pop_every + 1;
        if ((st = check_cuda(c, cudaMalloc(&c->d_pops, sizeof(double) * (size_t)c->n_rec_max * c->n), "pops"))) break;
        if ((st = check_cuda(c, cudaMalloc(&c->d_corr, sizeof(cd) * (size_t)(cfg->max_steps + 1)), "corr"))) break;
        if ((st = check_cuda(c, cudaMalloc(&c->d_erracc, sizeof(double) * cfg->n_traj), "erracc"))) break;
        if ((st = check_cuda(c, cudaMalloc(&c->d_psi0, sizeof(cd) * c->n), "psi0"))) break;
        if ((st = plain_alloc(c))) break;
        if ((st = plain_clear_observables(c))) break;
    } while (0);
    if (st != DQ_OK) {
        dq_destroy(c);
    } else {
        *out = c;
    }
    // the caller's current device is left as it was
    if (prev_device >= 0 && prev_device != cfg->device) cudaSetDevice(prev_device);
    return st;
}

static void tk_free(dq_ctx* c) {
    tk_ensemble_free(c);
    cudaFree(c->d_tk_rowptr); cudaFree(c->d_tk_col); cudaFree(c->d_tk_val); cudaFree(c->d_tk_diag);
    cudaFree(c->d_tk_Q); cudaFree(c->d_tk_x); cudaFree(c->d_tk_acc);
    c->d_tk_rowptr = c->d_tk_col = nullptr;
    c->d_tk_val = c->d_tk_diag = nullptr;
    c->d_tk_Q = c->d_tk_x = c->d_tk_acc = nullptr;
    c->tk_p = c->tk_m = 0;
    c->tk_coef.clear();
}

void dq_destroy(dq_ctx* c) {
    if (!c) return;
    DeviceScope dev_scope(c);
    if (c->stream) cudaStreamSynchronize(c->stream);
    adjoint_free(c);
    batched_free(c);
    plain_free(c);
    cudaFree(c->d_rowptr); cudaFree(c->d_col); cudaFree(c->d_val); cudaFree(c->d_h0);
    cudaFree(c->d_static); cudaFree(c->d_sigma); cudaFree(c->d_invtau); cudaFree(c->d_coeff);
    cudaFree(c->d_psi0); cudaFree(c->d_bra); cudaFree(c->d_pops); cudaFree(c->d_corr); cudaFree(c->d_erracc);
    cudaFree(c->d_zz_omega); cudaFree(c->d_zz_coeff);
    tk_free(c);
    cudaFree(c->d_ipr); cudaFree(c->d_ipr_partial); cudaFree(c->d_ipr_ticket);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* dq_last_error(const dq_ctx* c) { return c ? c->err.c_str() : "null context"; }

void* dq_get_stream(dq_ctx* c) { return c ? (void*)c->stream : nullptr; }

dq_status dq_set_hamiltonian_csr(dq_ctx* c, int n, const int* rowptr, const int* col, const double* val) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (n != c->n || !rowptr || !col || !val) return fail(c, DQ_ERR_ARG, "hamiltonian: size or null pointer");
    if (rowptr[0] != 0) return fail(c, DQ_ERR_ARG, "hamiltonian: rowptr[0] != 0");
    for (int i = 0; i < n; ++i)
        if (rowptr[i + 1] < rowptr[i]) return fail(c, DQ_ERR_ARG, "hamiltonian: rowptr not monotone");
    const int nnz = rowptr[n];
    std::vector<int> rp(n + 1, 0), cl;
    std::vector<double> vb, h0(n, 0.0);
    cl.reserve(nnz);
    vb.reserve(nnz);
    // besides the split: whether every row's off-diagonal columns are sorted
    // (the device builder of the packed coupling blocks merges sorted rows)
    // and the bandwidth (it sizes the shared-memory windows)
    bool sorted = true;
    int bw = 0;
    for (int i = 0; i < n; ++i) {
        int prev = -1;
        for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
            int j = col[p];
            if (j < 0 || j >= n) return fail(c, DQ_ERR_ARG, "hamiltonian: column index out of range");
            if (!std::isfinite(val[p])) return fail(c, DQ_ERR_ARG, "hamiltonian: non-finite value");
            if (j == i) {
                h0[i] += val[p];
            } else {
                cl.push_back(j);
                vb.push_back(val[p]);
                if (j < prev) sorted = false;
                prev = j;
                bw = std::max(bw, std::abs(j - i));
            }
        }
        rp[i + 1] = (int)cl.size();
    }
    c->rows_sorted = sorted;
    c->bw = bw;
    c->nnz_off = (int)cl.size();
    c->rowptr = std::move(rp);
    c->col = std::move(cl);
    c->val_base = std::move(vb);
    c->h0diag = std::move(h0);
    c->cls.clear();
    c->scales.clear();
    dq_status st;
    if ((st = upload(c, &c->d_rowptr, c->rowptr.data(), c->rowptr.size()))) return st;
    if ((st = upload(c, &c->d_col, c->col.data(), c->col.size()))) return st;
    if ((st = upload(c, &c->d_h0, c->h0diag.data(), c->h0diag.size()))) return st;
    if ((st = upload_couplings(c))) return st;
    if (c->nnz_off == 0) {
        // keep valid (non-null) pointers for kernels
        static const int zi = 0;
        static const double zd = 0.0;
        if ((st = upload(c, &c->d_col, &zi, 1))) return st;
        if ((st = upload(c, &c->d_val, &zd, 1))) return st;
    }
    c->have_ham = true;
    c->ready = false;
    return DQ_OK;
}

dq_status dq_set_coupling_classes(dq_ctx* c, const int* cls, int n_classes, const double* scales) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!c->have_ham) return fail(c, DQ_ERR_STATE, "coupling classes: set the Hamiltonian first");
    if (!cls || !scales || n_classes < 1) return fail(c, DQ_ERR_ARG, "coupling classes: null or empty");
    std::vector<int> off(cls, cls + c->nnz_off);
    for (int v : off)
        if (v < 0 || v >= n_classes) return fail(c, DQ_ERR_ARG, "coupling classes: class out of range");
    c->cls = off;
    c->scales.assign(scales, scales + n_classes);
    return upload_couplings(c);
}

dq_status dq_set_noise_params(dq_ctx* c, const double* sigma, const double* tau) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!sigma) return fail(c, DQ_ERR_ARG, "noise params: sigma is null");
    if (c->cfg.noise_model == DQ_NOISE_OU && !tau) return fail(c, DQ_ERR_ARG, "noise params: OU needs tau");
    const int n = c->n;
    c->sigma.assign(sigma, sigma + n);
    std::vector<double> invtau(n, 0.0), coeff(n, 0.0);
    if (tau) {
        c->tau.assign(tau, tau + n);
        for (int i = 0; i < n; ++i) {
            if (!(tau[i] > 0)) return fail(c, DQ_ERR_ARG, "noise params: tau must be > 0");
            // systemClass.cu:1033-1034
            invtau[i] = 1. / tau[i];
            coeff[i] = sigma[i] * sqrt(2. / tau[i]);
        }
    }
    dq_status st;
    if ((st = upload(c, &c->d_sigma, c->sigma.data(), (size_t)n))) return st;
    if ((st = upload(c, &c->d_invtau, invtau.data(), (size_t)n))) return st;
    if ((st = upload(c, &c->d_coeff, coeff.data(), (size_t)n))) return st;
    c->have_noise = true;
    return DQ_OK;
}

dq_status dq_set_zz_spectral_density(dq_ctx* c, int n_osc, const double* omega, const double* J, double d_omega,
                                     double temperature) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (n_osc < 1 || n_osc > kMaxZZOsc || !omega || !J || !(temperature > 0) || !(d_omega > 0))
        return fail(c, DQ_ERR_ARG, "zz: 1..1024 oscillators, positive spacing and temperature");
    // systemClass.cu:1128-1139: hbar = 1, k_B = 0.695035 cm^-1/K, 1/cm -> 1/fs by 5308.84
    const double pi = 3.14159265358979323846;
    c->zz_omega.resize(n_osc);
    c->zz_coeff.resize(n_osc);
    for (int o = 0; o < n_osc; ++o) {
        const double G = J[o] / (1 - exp(-1. / (0.695035 * temperature) * 1.0 * omega[o]));
        c->zz_coeff[o] = sqrt(2.) * sqrt(G * d_omega / pi);
        c->zz_omega[o] = omega[o] / 5308.84;
        if (!std::isfinite(c->zz_coeff[o])) return fail(c, DQ_ERR_ARG, "zz: non-finite amplitude (omega <= 0?)");
    }
    c->zz_n_osc = n_osc;
    dq_status st;
    if ((st = upload(c, &c->d_zz_omega, c->zz_omega.data(), (size_t)n_osc))) return st;
    if ((st = upload(c, &c->d_zz_coeff, c->zz_coeff.data(), (size_t)n_osc))) return st;
    c->ready = false;
    return DQ_OK;
}

dq_status dq_set_taylor_krylov(dq_ctx* c, int p, int m_b, const int* rowptr, const int* col, const double* val) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (p == 0) {
        tk_free(c);
        c->ready = false;
        return DQ_OK;
    }
    if (p < 2 || m_b < 1 || m_b > kMaxM || m_b + p > kMaxL || !rowptr || !col || !val)
        return fail(c, DQ_ERR_ARG, "taylor_krylov: need 2 <= p, 1 <= m_b <= 32, m_b + p <= 34 and a CSR matrix B");
    if (c->cfg.m_min > 0) return fail(c, DQ_ERR_ARG, "taylor_krylov: needs a fixed Krylov dimension (m_min = 0)");
    const int n = c->n;
    if (rowptr[0] != 0) return fail(c, DQ_ERR_ARG, "taylor_krylov: rowptr[0] != 0");
    for (int i = 0; i < n; ++i)
        if (rowptr[i + 1] < rowptr[i]) return fail(c, DQ_ERR_ARG, "taylor_krylov: rowptr not monotone");
    // split B into its diagonal and off-diagonal CSR like the Hamiltonian
    std::vector<int> rp(n + 1, 0), cl;
    std::vector<double> vb, dg(n, 0.0);
    for (int i = 0; i < n; ++i) {
        for (int q = rowptr[i]; q < rowptr[i + 1]; ++q) {
            const int j = col[q];
            if (j < 0 || j >= n) return fail(c, DQ_ERR_ARG, "taylor_krylov: column index out of range");
            if (!std::isfinite(val[q])) return fail(c, DQ_ERR_ARG, "taylor_krylov: non-finite value");
            if (j == i) dg[i] += val[q];
            else { cl.push_back(j); vb.push_back(val[q]); }
        }
        rp[i + 1] = (int)cl.size();
    }
    if (cl.empty()) { cl.push_back(0); vb.push_back(0.0); }   // valid pointers for the kernels
    tk_free(c);
    dq_status st;
    if ((st = upload(c, &c->d_tk_rowptr, rp.data(), rp.size()))) return st;
    if ((st = upload(c, &c->d_tk_col, cl.data(), cl.size()))) return st;
    if ((st = upload(c, &c->d_tk_val, vb.data(), vb.size()))) return st;
    if ((st = upload(c, &c->d_tk_diag, dg.data(), dg.size()))) return st;
    DQ_CU(cudaMalloc(&c->d_tk_Q, sizeof(cd) * (size_t)n * (m_b + 2)));
    DQ_CU(cudaMemsetAsync(c->d_tk_Q, 0, sizeof(cd) * (size_t)n * (m_b + 2), c->stream));
    DQ_CU(cudaMalloc(&c->d_tk_x, sizeof(cd) * (size_t)n * 2));
    DQ_CU(cudaMalloc(&c->d_tk_acc, sizeof(cd) * (size_t)n));
    // tau^k / k! with tau = -i dt / hbar (taylorKrylovClass.cu:196-206)
    const cd tau = cmk(0.0, c->tau_im);
    cd pw = cmk(1.0, 0.0);
    double fact = 1.0;
    c->tk_coef.assign(p, cmk(0.0, 0.0));
    c->tk_coef[0] = pw;
    for (int k = 1; k < p; ++k) {
        pw = cmk(pw.x * tau.x - pw.y * tau.y, pw.x * tau.y + pw.y * tau.x);
        fact *= k;
        c->tk_coef[k] = cmk(pw.x / fact, pw.y / fact);
    }
    c->tk_p = p;
    c->tk_m = m_b;
    c->ready = false;
    return DQ_OK;
}

dq_status dq_set_ipr(dq_ctx* c, int enable) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (enable && !c->d_ipr) {
        DQ_CU(cudaMalloc(&c->d_ipr, sizeof(double) * (size_t)(c->cfg.max_steps + 1)));
        DQ_CU(cudaMemsetAsync(c->d_ipr, 0, sizeof(double) * (size_t)(c->cfg.max_steps + 1), c->stream));
        DQ_CU(cudaMalloc(&c->d_ipr_partial, sizeof(double) * (size_t)kIprRowGroups * c->cfg.n_traj));
        DQ_CU(cudaMalloc(&c->d_ipr_ticket, sizeof(unsigned int)));
        DQ_CU(cudaMemsetAsync(c->d_ipr_ticket, 0, sizeof(unsigned int), c->stream));
    }
    c->ipr_on = enable != 0;
    c->ready = false;
    return DQ_OK;
}

dq_status dq_get_ipr(dq_ctx* c, double* out, int* n_values) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!c->ipr_on) return fail(c, DQ_ERR_STATE, "get_ipr: the inverse participation ratio is not enabled");
    const int nv = c->steps_done + 1;
    if (n_values) *n_values = nv;
    if (!out) return DQ_OK;
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(out, c->d_ipr, sizeof(double) * nv, cudaMemcpyDeviceToHost));
    const double inv = 1.0 / observed_trajectories(c);
    for (int k = 0; k < nv; ++k) out[k] *= inv;
    return DQ_OK;
}

dq_status dq_set_correlation_bra(dq_ctx* c, const dq_cdouble* bra) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!bra) {
        cudaFree(c->d_bra);
        c->d_bra = nullptr;
    } else {
        for (int i = 0; i < c->n; ++i)
            if (!std::isfinite(bra[i].re) || !std::isfinite(bra[i].im))
                return fail(c, DQ_ERR_ARG, "correlation_bra: non-finite value");
        if (!c->d_bra) DQ_CU(cudaMalloc(&c->d_bra, sizeof(cd) * c->n));
        DQ_CU(cudaMemcpyAsync(c->d_bra, bra, sizeof(cd) * c->n, cudaMemcpyHostToDevice, c->stream));
        DQ_CU(cudaStreamSynchronize(c->stream));
    }
    c->ready = false;
    return DQ_OK;
}

dq_status dq_set_trajectory_offset(dq_ctx* c, int traj0) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (traj0 < 0 || traj0 % 2) return fail(c, DQ_ERR_ARG, "trajectory_offset: must be even and >= 0");
    c->traj0 = traj0;
    c->ready = false;
    return DQ_OK;
}

dq_status dq_get_observable_sums(dq_ctx* c, double* pops, dq_cdouble* corr, double* ipr) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (c->last_path == 1 && c->bat) {
        dq_status st = batched_collect_corr(c);
        if (st) return st;
    }
    const int nrec = c->steps_done / c->cfg.pop_every + 1, np = c->steps_done + 1;
    DQ_CU(cudaStreamSynchronize(c->stream));
    if (pops) DQ_CU(cudaMemcpy(pops, c->d_pops, sizeof(double) * (size_t)nrec * c->n, cudaMemcpyDeviceToHost));
    if (corr) DQ_CU(cudaMemcpy(corr, c->d_corr, sizeof(cd) * np, cudaMemcpyDeviceToHost));
    if (ipr) {
        if (!c->ipr_on) return fail(c, DQ_ERR_STATE, "observable_sums: the inverse participation ratio is off");
        DQ_CU(cudaMemcpy(ipr, c->d_ipr, sizeof(double) * np, cudaMemcpyDeviceToHost));
    }
    return DQ_OK;
}

dq_status dq_set_observable_sums(dq_ctx* c, const double* pops, const dq_cdouble* corr, const double* ipr,
                                 int n_traj_total) {
    DeviceScope dev_scope(c);
    if (!c || !pops || !corr || n_traj_total < 1) return DQ_ERR_ARG;
    if (ipr && !c->ipr_on) return fail(c, DQ_ERR_STATE, "observable_sums: the inverse participation ratio is off");
    const int nrec = c->steps_done / c->cfg.pop_every + 1, np = c->steps_done + 1;
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(c->d_pops, pops, sizeof(double) * (size_t)nrec * c->n, cudaMemcpyHostToDevice));
    DQ_CU(cudaMemcpy(c->d_corr, corr, sizeof(cd) * np, cudaMemcpyHostToDevice));
    if (ipr) DQ_CU(cudaMemcpy(c->d_ipr, ipr, sizeof(double) * np, cudaMemcpyHostToDevice));
    c->obs_traj = n_traj_total;
    c->last_path = 2;
    return DQ_OK;
}

dq_status dq_set_static_energies(dq_ctx* c, const double* eps) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!eps) {
        c->static_eps.clear();
        cudaFree(c->d_static);
        c->d_static = nullptr;
        return DQ_OK;
    }
    c->static_eps.assign(eps, eps + c->n);
    return upload(c, &c->d_static, c->static_eps.data(), (size_t)c->n);
}

dq_status dq_set_initial_state(dq_ctx* c, const dq_cdouble* psi0) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!psi0) return fail(c, DQ_ERR_ARG, "initial state is null");
    c->psi0.assign(psi0, psi0 + c->n);
    DQ_CU(cudaMemcpyAsync(c->d_psi0, psi0, sizeof(cd) * c->n, cudaMemcpyHostToDevice, c->stream));
    DQ_CU(cudaStreamSynchronize(c->stream));
    c->have_psi0 = true;
    c->ready = false;   // the next run starts every trajectory from it
    return DQ_OK;
}

// spectraClass.cu:440-458: psi0 = mu / |mu| for one polarisation direction
dq_status dq_set_initial_dipole(dq_ctx* c, const double* mu) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (!mu) return fail(c, DQ_ERR_ARG, "initial dipole is null");
    double s = 0.0;
    for (int i = 0; i < c->n; ++i) s += mu[i] * mu[i];
    const double nrm = sqrt(s);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) return fail(c, DQ_ERR_ARG, "initial dipole: zero or non-finite norm");
    std::vector<dq_cdouble> psi0(c->n);
    for (int i = 0; i < c->n; ++i) {
        psi0[i].re = mu[i] / nrm;
        psi0[i].im = 0.0;
    }
    return dq_set_initial_state(c, psi0.data());
}

static dq_status check_ready(dq_ctx* c) {
    if (!c->have_ham) return fail(c, DQ_ERR_STATE, "no Hamiltonian set");
    if ((c->cfg.noise_model == DQ_NOISE_GAUSS || c->cfg.noise_model == DQ_NOISE_OU) && !c->have_noise)
        return fail(c, DQ_ERR_STATE, "no noise parameters set");
    if (c->cfg.noise_model == DQ_NOISE_ZZ && c->zz_n_osc == 0) return fail(c, DQ_ERR_STATE, "no ZZ spectral density set");
    if (!c->have_psi0) return fail(c, DQ_ERR_STATE, "no initial state set");
    return DQ_OK;
}

dq_status dq_reset(dq_ctx* c) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    dq_status st;
    if ((st = check_ready(c))) return st;
    if ((st = plain_traj_init(c))) return st;
    if ((st = plain_clear_observables(c))) return st;
    c->steps_done = 0;
    c->plain_traj_done = 0;
    c->obs_traj = 0;
    if (c->last_path == 2) c->last_path = 0;
    if (c->tk_p > 0 && c->tke) {
        if ((st = tk_ensemble_reset(c))) return st;
    } else if (c->bat) {
        if ((st = batched_reset(c))) return st;
    }
    c->ready = true;
    return DQ_OK;
}

dq_status dq_prop_step(dq_ctx* c, int traj, int step, const dq_cdouble* psi_in, dq_cdouble* psi_out, double* err_est) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (traj < 0 || traj >= c->cfg.n_traj || step < 0 || !psi_in || !psi_out || psi_in == psi_out)
        return fail(c, DQ_ERR_ARG, "prop_step: bad trajectory, step or pointers");
    dq_status st;
    if (!c->ready) {
        if ((st = dq_reset(c))) return st;
    }
    if ((st = plain_step(c, traj, step, reinterpret_cast<const cd*>(psi_in), reinterpret_cast<cd*>(psi_out), false, -1)))
        return st;
    if (err_est) {
        DQ_CU(cudaStreamSynchronize(c->stream));
        PlainScalars h;
        DQ_CU(cudaMemcpy(&h, c->d_ps, sizeof(h), cudaMemcpyDeviceToHost));
        *err_est = h.err;
        if (h.status) {
            int code = h.status;
            cudaMemsetAsync(&c->d_ps->status, 0, sizeof(int), c->stream);
            return read_status(c, code, "prop_step");
        }
    }
    return DQ_OK;
}

dq_status dq_run_plain(dq_ctx* c, int n_steps) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (n_steps < 0 || n_steps > c->cfg.max_steps) return fail(c, DQ_ERR_ARG, "run_plain: n_steps out of range");
    dq_status st;
    if ((st = dq_reset(c))) return st;
    // the ensemble's initial record (added at its reset) belongs to dq_run
    if ((st = plain_clear_observables(c))) return st;
    const int n = c->n, pe = c->cfg.pop_every;
    for (int t = 0; t < c->cfg.n_traj; ++t) {
        if ((st = plain_observe_initial(c))) return st;
        cd* src = c->d_psi_a;
        cd* dst = c->d_psi_b;
        DQ_CU(cudaMemcpyAsync(src, c->d_psi0, sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->stream));
        for (int k = 0; k < n_steps; ++k) {
            int rec = ((k + 1) % pe == 0) ? (k + 1) / pe : -1;
            if ((st = plain_step(c, t, k, src, dst, true, rec))) return st;
            std::swap(src, dst);
        }
    }
    DQ_CU(cudaStreamSynchronize(c->stream));
    PlainScalars h;
    DQ_CU(cudaMemcpy(&h, c->d_ps, sizeof(h), cudaMemcpyDeviceToHost));
    if (h.status) return read_status(c, h.status, "run_plain");
    c->steps_done = n_steps;
    c->plain_traj_done = c->cfg.n_traj;
    c->last_path = 0;
    c->ready = false;   // the ensemble form restarts from dq_reset
    return DQ_OK;
}

dq_status dq_run(dq_ctx* c, int n_steps) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (n_steps < 0 || c->steps_done + n_steps > c->cfg.max_steps)
        return fail(c, DQ_ERR_ARG, "run: steps exceed max_steps");
    if (c->obs_traj > 0)
        return fail(c, DQ_ERR_STATE, "run: the observables hold reduced ensemble sums; dq_reset first");
    dq_status st;
    if (c->tk_p > 0) {
        // Taylor-Krylov mode: the FP64 ensemble of dq_tk_ensemble.cu
        if (c->cfg.reorth) return fail(c, DQ_ERR_ARG, "run: Taylor-Krylov ensemble without reorthogonalisation");
        if (!c->tke) {
            if ((st = check_ready(c))) return st;
            if ((st = tk_ensemble_reset(c))) return st;
            c->ready = false;
        }
        if (!c->ready || c->last_path != 3) {
            if ((st = dq_reset(c))) return st;
        }
        c->last_path = 3;
        return tk_ensemble_run(c, n_steps);
    }
    if (!c->bat) {
        if ((st = batched_alloc(c))) return st;
        c->ready = false;
    }
    if (!c->ready) {
        if ((st = dq_reset(c))) return st;
    }
    c->last_path = 1;
    return batched_run(c, n_steps);
}

dq_status dq_get_populations(dq_ctx* c, double* out, int* n_records) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    int nrec = c->steps_done / c->cfg.pop_every + 1;
    if (n_records) *n_records = nrec;
    if (!out) return DQ_OK;
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(out, c->d_pops, sizeof(double) * (size_t)nrec * c->n, cudaMemcpyDeviceToHost));
    const double inv = 1.0 / observed_trajectories(c);
    for (size_t x = 0; x < (size_t)nrec * c->n; ++x) out[x] *= inv;
    return DQ_OK;
}

dq_status dq_get_correlation(dq_ctx* c, dq_cdouble* out, int* n_points) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    int np = c->steps_done + 1;
    if (n_points) *n_points = np;
    if (!out) return DQ_OK;
    if (c->last_path == 1 && c->bat) {
        dq_status st = batched_collect_corr(c);
        if (st) return st;
    }
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(out, c->d_corr, sizeof(cd) * np, cudaMemcpyDeviceToHost));
    const double inv = 1.0 / observed_trajectories(c);
    for (int k = 0; k < np; ++k) { out[k].re *= inv; out[k].im *= inv; }
    return DQ_OK;
}

dq_status dq_get_states(dq_ctx* c, dq_cdouble* out) {
    DeviceScope dev_scope(c);
    if (!c || !out) return DQ_ERR_ARG;
    if (c->last_path == 3 && c->tke) return tk_ensemble_states(c, out);
    if (!c->bat) return fail(c, DQ_ERR_STATE, "get_states: no ensemble state (run dq_run first)");
    return batched_get_states(c, out);
}

dq_status dq_get_error_accum(dq_ctx* c, double* out) {
    DeviceScope dev_scope(c);
    if (!c || !out) return DQ_ERR_ARG;
    DQ_CU(cudaStreamSynchronize(c->stream));
    DQ_CU(cudaMemcpy(out, c->d_erracc, sizeof(double) * c->cfg.n_traj, cudaMemcpyDeviceToHost));
    return DQ_OK;
}

int dq_steps_done(const dq_ctx* c) { return c ? c->steps_done : -1; }

}  // extern "C"

extern "C" dq_status dq_get_noise_state(dq_ctx* c, int traj, double* eps, double* deps) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (traj < 0 || traj >= c->cfg.n_traj) return fail(c, DQ_ERR_ARG, "noise_state: bad trajectory");
    const int n = c->n;
    DQ_CU(cudaStreamSynchronize(c->stream));
    if (c->last_path == 1 && c->bat) {
        const double* e = nullptr;
        const double* d = nullptr;
        batched_noise_arrays(c, &e, &d);
        const size_t pitch = sizeof(double) * c->cfg.n_traj;
        if (eps) DQ_CU(cudaMemcpy2D(eps, sizeof(double), e + traj, pitch, sizeof(double), n, cudaMemcpyDeviceToHost));
        if (deps) DQ_CU(cudaMemcpy2D(deps, sizeof(double), d + traj, pitch, sizeof(double), n, cudaMemcpyDeviceToHost));
    } else {
        if (eps) DQ_CU(cudaMemcpy(eps, c->d_eps_p + (size_t)traj * n, sizeof(double) * n, cudaMemcpyDeviceToHost));
        if (deps) DQ_CU(cudaMemcpy(deps, c->d_deps_p + (size_t)traj * n, sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    return DQ_OK;
}

extern "C" dq_status dq_profile_step(dq_ctx* c, int n_steps, double* ms_per_launch, int* launches, int n_kinds) {
    DeviceScope dev_scope(c);
    if (!c || !ms_per_launch || n_kinds < 1) return DQ_ERR_ARG;
    if (n_steps < 1 || c->steps_done + n_steps > c->cfg.max_steps)
        return fail(c, DQ_ERR_ARG, "profile_step: steps exceed max_steps");
    dq_status st;
    if (!c->bat) {
        if ((st = batched_alloc(c))) return st;
        c->ready = false;
    }
    if (!c->ready) {
        if ((st = dq_reset(c))) return st;
    }
    c->last_path = 1;
    const int nk = n_kinds < DQ_KIND_COUNT ? n_kinds : DQ_KIND_COUNT;
    std::vector<double> ms(DQ_KIND_COUNT, 0.0);
    std::vector<int> cnt(DQ_KIND_COUNT, 0);
    if ((st = batched_profile(c, n_steps, ms.data(), cnt.data(), DQ_KIND_COUNT))) return st;
    for (int k = 0; k < nk; ++k) {
        ms_per_launch[k] = cnt[k] ? ms[k] / cnt[k] : 0.0;
        if (launches) launches[k] = cnt[k];
    }
    return DQ_OK;
}

static dq_status ensure_batched(dq_ctx* c) {
    dq_status st;
    if (!c->bat) {
        if ((st = check_ready(c))) return st;
        if ((st = batched_alloc(c))) return st;
        c->ready = false;
    }
    return DQ_OK;
}

extern "C" dq_status dq_set_tiling(dq_ctx* c, int traj_chunk, int vec, int ctas_per_sm, int rows_per_block,
                                   int staged, int groups) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    dq_status st;
    if (!c->bat) {
        // a new workspace gets the requested tiling directly (no default blocks built first)
        if ((st = check_ready(c))) return st;
        if ((st = batched_alloc(c, false))) return st;
        c->ready = false;
        if ((st = batched_set_tiling(c, traj_chunk, vec, ctas_per_sm, rows_per_block, staged, groups))) {
            dq_status st2 = batched_default_tiling(c);
            if (st2) return st2;
            return fail(c, st, "set_tiling: invalid tiling for this system");
        }
        return DQ_OK;
    }
    if ((st = batched_set_tiling(c, traj_chunk, vec, ctas_per_sm, rows_per_block, staged, groups)))
        return fail(c, st, "set_tiling: invalid tiling for this system");
    c->ready = false;
    return DQ_OK;
}

extern "C" dq_status dq_get_tiling(dq_ctx* c, int* traj_chunk, int* vec, int* ctas_per_sm, int* rows_per_block,
                                   int* staged, int* groups) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    dq_status st;
    if ((st = ensure_batched(c))) return st;
    batched_get_tiling(c, traj_chunk, vec, ctas_per_sm, rows_per_block, staged, groups);
    return DQ_OK;
}

extern "C" dq_status dq_autotune(dq_ctx* c, int reps, double* best_ms) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    if (reps < 1) reps = 5;
    dq_status st;
    if ((st = ensure_batched(c))) return st;
    if ((st = dq_reset(c))) return st;
    int b_tc = 0, b_vec = 0, b_cps = 0, b_r = 0, b_st = 0, b_g = 1;
    double best = 1e30;
    const int vecs[2] = {2, 1};
    for (int groups = 1; groups <= 8; groups <<= 1)
        for (int staged = 0; staged <= 12; ++staged)
            for (int vi = 0; vi < 2; ++vi)
                for (int tc = 4; tc <= 64; tc <<= 1)
                    for (int cps = 1; cps <= 8; cps <<= 1)
                        for (int R : {1, 2, 3, 4, 8}) {
                            if (batched_set_tiling(c, tc, vecs[vi], cps, R, staged, groups) != DQ_OK) continue;
                            double ms = 0.0;
                            if ((st = batched_time_iteration(c, reps, &ms))) return st;
                            if (ms < best) {
                                best = ms; b_tc = tc; b_vec = vecs[vi]; b_cps = cps; b_r = R; b_st = staged;
                                b_g = groups;
                            }
                        }
    if (!b_tc) return fail(c, DQ_ERR_ARG, "autotune: no valid tiling");
    if ((st = batched_set_tiling(c, b_tc, b_vec, b_cps, b_r, b_st, b_g))) return st;
    if (best_ms) *best_ms = best;
    c->ready = false;
    return dq_reset(c);
}

extern "C" dq_status dq_time_iteration(dq_ctx* c, int reps, double* ms) {
    DeviceScope dev_scope(c);
    if (!c || !ms) return DQ_ERR_ARG;
    if (reps < 1) reps = 5;
    dq_status st;
    if ((st = ensure_batched(c))) return st;
    if ((st = dq_reset(c))) return st;
    if ((st = batched_time_iteration(c, reps, ms))) return st;
    c->ready = false;
    return DQ_OK;
}

extern "C" dq_status dq_time_gather_floor(dq_ctx* c, int reps, double* ms) {
    DeviceScope dev_scope(c);
    if (!c || !ms) return DQ_ERR_ARG;
    if (reps < 1) reps = 5;
    dq_status st;
    if ((st = ensure_batched(c))) return st;
    if ((st = dq_reset(c))) return st;
    if ((st = batched_time_gather_floor(c, reps, ms))) return st;
    c->ready = false;
    return DQ_OK;
}

extern "C" dq_status dq_debug_set_wait_cycles(dq_ctx* c, int cycles) {
    DeviceScope dev_scope(c);
    if (!c) return DQ_ERR_ARG;
    return batched_set_wait_cycles(c, cycles);
}
