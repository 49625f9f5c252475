// dq_output.cu — the reference's output files written from the ensemble's
// device observables:
//   pops.dat              popPrintClass.cu:160-522 (text or binary, sums over
//                         runs, continuation through temp_pops.dat + rename)
//   _states_<t>.dat       statePrintClass.cu:82-199 (binary: float stamp,
//                         int N, int runs, then every run's complex128 state)
//   correlation/spectrum  spectraClass.cu:621-690 (text; transform length
//                         steps + 1, the reference's frequency axes and
//                         scaling constant)
// Formatting follows the reference's iostream settings: setprecision(17)
// setw(25) for populations ("%25.17g"), the stream default ("%g", 6
// significant digits) elsewhere.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "dq_internal.h"

namespace dq {

// X_k = sum_j x_j exp(+2 pi i jk / n) for any n (the spectrum's length is
// steps + 1); one thread per output, the angle reduced exactly as jk mod n.
__global__ void k_idft_direct(int n, const cd* __restrict__ x, double scale, cd* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double sr = 0.0, si = 0.0;
        long long jk = 0;
        for (int j = 0; j < n; ++j) {
            double s, c;
            sincospi(2.0 * (double)jk / (double)n, &s, &c);
            const cd v = x[j];
            sr += v.x * c - v.y * s;
            si += v.x * s + v.y * c;
            jk += k;
            if (jk >= n) jk -= n;
        }
        out[k] = cmk(sr * scale, si * scale);
    }
}

}  // namespace dq

using namespace dq;

namespace {
dq_status ofail(dq_ctx* c, int code, const std::string& msg) {
    c->err = msg;
    return code;
}

// The ensemble's population records (sums over trajectories) on the host.
dq_status host_pop_sums(dq_ctx* c, std::vector<double>& sums, int* nrec) {
    if (c->last_path == 1 && c->bat) {
        dq_status st = batched_collect_corr(c);
        if (st) return st;
    }
    *nrec = c->steps_done / c->cfg.pop_every + 1;
    sums.resize((size_t)*nrec * c->n);
    dq_status st = check_cuda(c, cudaStreamSynchronize(c->stream), "output sync");
    if (st) return st;
    return check_cuda(c, cudaMemcpy(sums.data(), c->d_pops, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost),
                      "population copy");
}

bool read_text_header(FILE* f, int* numsims, double* dt, int* steps, int* sites) {
    char key[64];
    if (fscanf(f, "%63s %d", key, numsims) != 2 || std::string(key) != "numsims") return false;
    if (fscanf(f, "%63s %lf", key, dt) != 2 || std::string(key) != "dt") return false;
    if (fscanf(f, "%63s %d", key, steps) != 2 || std::string(key) != "totalsteps") return false;
    if (fscanf(f, "%63s %d", key, sites) != 2 || std::string(key) != "numprintedsites") return false;
    return true;
}
}  // namespace

extern "C" {

dq_status dq_write_populations(dq_ctx* c, const char* path, int binary, int continuation) {
    DeviceScope dev_scope(c);
    if (!c || !path) return DQ_ERR_ARG;
    std::vector<double> sums;
    int nrec = 0;
    dq_status st = host_pop_sums(c, sums, &nrec);
    if (st) return st;
    const int n = c->n, T = c->steps_done, pe = c->cfg.pop_every;
    const int nsteps_out = nrec - 1;   // records at pop_every, 2 pop_every, ... (step 0 is not printed)
    const double dt = c->cfg.dt;
    int numsims = observed_trajectories(c);
    std::vector<double> prev;
    if (continuation) {
        // add the sums of an earlier file with the same dt, steps and sites
        FILE* f = fopen(path, binary ? "rb" : "r");
        if (!f) return ofail(c, DQ_ERR_ARG, "write_populations: continuation file missing");
        int pn = 0, ps = 0, pz = 0;
        double pdt = 0;
        bool ok;
        if (binary) {
            ok = fread(&pn, sizeof(int), 1, f) == 1 && fread(&pdt, sizeof(double), 1, f) == 1 &&
                 fread(&ps, sizeof(int), 1, f) == 1 && fread(&pz, sizeof(int), 1, f) == 1;
        } else {
            ok = read_text_header(f, &pn, &pdt, &ps, &pz);
        }
        if (!ok || pdt != dt || ps != T || pz != n) {
            fclose(f);
            return ofail(c, DQ_ERR_ARG, "write_populations: previous file's dt, totalsteps or sites differ");
        }
        prev.resize((size_t)nsteps_out * n);
        for (int r = 0; r < nsteps_out && ok; ++r) {
            if (binary) {
                ok = fread(prev.data() + (size_t)r * n, sizeof(double), n, f) == (size_t)n;
            } else {
                char key[64];
                int stp = 0;
                ok = fscanf(f, "%63s %d", key, &stp) == 2 && std::string(key) == "STEP";
                for (int i = 0; i < n && ok; ++i) {
                    int site = -1;
                    ok = fscanf(f, "%lf (%d)", &prev[(size_t)r * n + i], &site) == 2 && site == i;
                }
            }
        }
        fclose(f);
        if (!ok) return ofail(c, DQ_ERR_ARG, "write_populations: previous file is truncated or malformed");
        numsims += pn;
    }
    // temp file beside the target, then rename (popPrintClass.cu:496-519)
    std::string p(path);
    const size_t slash = p.find_last_of('/');
    const std::string tmp = (slash == std::string::npos) ? "temp_" + p : p.substr(0, slash + 1) + "temp_" + p.substr(slash + 1);
    FILE* f = fopen(tmp.c_str(), binary ? "wb" : "w");
    if (!f) return ofail(c, DQ_ERR_ARG, "write_populations: cannot create " + tmp);
    bool ok = true;
    if (binary) {
        ok = fwrite(&numsims, sizeof(int), 1, f) == 1 && fwrite(&dt, sizeof(double), 1, f) == 1 &&
             fwrite(&T, sizeof(int), 1, f) == 1 && fwrite(&n, sizeof(int), 1, f) == 1;
    } else {
        ok = fprintf(f, "numsims %d\ndt %g\ntotalsteps %d\nnumprintedsites %d\n", numsims, dt, T, n) > 0;
    }
    std::vector<double> row(n);
    for (int r = 1; r <= nsteps_out && ok; ++r) {
        for (int i = 0; i < n; ++i) row[i] = sums[(size_t)r * n + i] + (prev.empty() ? 0.0 : prev[(size_t)(r - 1) * n + i]);
        if (binary) {
            ok = fwrite(row.data(), sizeof(double), n, f) == (size_t)n;
        } else {
            ok = fprintf(f, "STEP %d\n", r * pe) > 0;
            for (int i = 0; i < n && ok; ++i) ok = fprintf(f, "%25.17g (%d)\n", row[i], i) > 0;
        }
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) return ofail(c, DQ_ERR_ARG, "write_populations: write failed");
    if (rename(tmp.c_str(), path) != 0) return ofail(c, DQ_ERR_ARG, "write_populations: rename failed");
    return DQ_OK;
}

dq_status dq_write_states(dq_ctx* c, const char* folder) {
    DeviceScope dev_scope(c);
    if (!c || !folder) return DQ_ERR_ARG;
    if (!c->bat && !c->tke) return ofail(c, DQ_ERR_STATE, "write_states: no ensemble state (run dq_run first)");
    const int n = c->n, nr = c->cfg.n_traj;
    std::vector<dq_cdouble> st_host((size_t)nr * n);
    dq_status st = dq_get_states(c, st_host.data());
    if (st) return st;
    // statePrintClass.cu:112-127: stamp = dt * step as a float, printed by the stream default
    const float stamp = (float)(c->cfg.dt * c->steps_done);
    char name[64];
    snprintf(name, sizeof name, "/_states_%g.dat", (double)stamp);
    const std::string path = std::string(folder) + name;
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return ofail(c, DQ_ERR_ARG, "write_states: cannot create " + path);
    bool ok = fwrite(&stamp, sizeof(float), 1, f) == 1 && fwrite(&n, sizeof(int), 1, f) == 1 &&
              fwrite(&nr, sizeof(int), 1, f) == 1 &&
              fwrite(st_host.data(), sizeof(dq_cdouble), st_host.size(), f) == st_host.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? DQ_OK : ofail(c, DQ_ERR_ARG, "write_states: write failed");
}

// invParticRat.dat (systemClass.cu:1735-1750): a two-line header, then one
// line "k  IPR_k" per step k = 0..steps-1 with the ensemble mean of
// 1 / sum_i |psi_i(k)|^4 printed like an ostream at its default precision.
dq_status dq_write_ipr(dq_ctx* c, const char* path) {
    DeviceScope dev_scope(c);
    if (!c || !path) return DQ_ERR_ARG;
    int nv = 0;
    dq_status st = dq_get_ipr(c, nullptr, &nv);
    if (st) return st;
    std::vector<double> v(nv);
    if ((st = dq_get_ipr(c, v.data(), &nv))) return st;
    FILE* f = fopen(path, "w");
    if (!f) return ofail(c, DQ_ERR_ARG, std::string("write_ipr: cannot open ") + path);
    fprintf(f, "# Inverse Particle Ratios\n# {timestep} {IPR}}\n");
    for (int k = 0; k + 1 < nv; ++k) fprintf(f, "%d  %g\n", k, v[k]);
    fclose(f);
    return DQ_OK;
}

// The ensemble-mean correlation and its inverse DFT of length steps + 1
// (spectraClass.cu:108, :621-626), scaled as spectraClass.cu:640-687 does
// before printing: M(t) by the scaling constant (held in a float), the
// transform by that constant over the step count.
static dq_status scaled_spectrum(dq_ctx* c, double scaling, std::vector<cd>& corr, std::vector<cd>& spec) {
    if (c->last_path == 1 && c->bat) {
        dq_status st = batched_collect_corr(c);
        if (st) return st;
    }
    const int T = c->steps_done, len = T + 1;
    cd* d = nullptr;
    dq_status st = check_cuda(c, cudaMalloc(&d, sizeof(cd) * 2 * (size_t)len), "spectrum alloc");
    if (st) return st;
    corr.assign(len, cd{0.0, 0.0});
    spec.assign(len, cd{0.0, 0.0});
    st = check_cuda(c, cudaMemcpyAsync(d, c->d_corr, sizeof(cd) * len, cudaMemcpyDeviceToDevice, c->stream), "copy");
    // optional Gaussian dressing of M(t) before the transform; the file shows the dressed M(t)
    if (!st) st = dress_correlation(c, T, d);
    if (!st) {
        const int blocks = std::max(1, std::min(148 * 4, (len + 127) / 128));
        k_idft_direct<<<blocks, 128, 0, c->stream>>>(len, d, 1.0 / observed_trajectories(c), d + len);
        st = check_cuda(c, cudaGetLastError(), "inverse DFT");
    }
    if (!st) st = check_cuda(c, cudaMemcpyAsync(corr.data(), d, sizeof(cd) * len, cudaMemcpyDeviceToHost, c->stream),
                             "copy");
    if (!st) st = check_cuda(c, cudaMemcpyAsync(spec.data(), d + len, sizeof(cd) * len, cudaMemcpyDeviceToHost,
                                                c->stream), "copy");
    if (!st) st = check_cuda(c, cudaStreamSynchronize(c->stream), "sync");
    cudaFree(d);
    if (st) return st;
    // the reference keeps the scaling constant in a float (spectraClass.cu:643-651)
    const float sc = (float)scaling;
    const double inv_traj = 1.0 / observed_trajectories(c);
    for (int i = 0; i < len; ++i) {
        corr[i].x = corr[i].x * inv_traj * sc;
        corr[i].y = corr[i].y * inv_traj * sc;
        spec[i].x = spec[i].x * (sc / T);
        spec[i].y = spec[i].y * (sc / T);
    }
    return DQ_OK;
}

static dq_status write_spectrum_files(dq_ctx* c, int T, double dt, const std::vector<cd>& corr,
                                      const std::vector<cd>& spec, const char* corr_path, const char* spec_path) {
    const int len = T + 1;
    FILE* f = fopen(corr_path, "w");
    if (!f) return ofail(c, DQ_ERR_ARG, std::string("write_spectrum: cannot create ") + corr_path);
    bool ok = fprintf(f, "{timestep #} {timestamp fs} {M(t) real imag}: \n") > 0;
    for (int i = 0; i < len && ok; ++i) ok = fprintf(f, "%6d%14g%14g%14g\n", i, i * dt, corr[i].x, corr[i].y) > 0;
    ok = (fclose(f) == 0) && ok;
    if (!ok) return ofail(c, DQ_ERR_ARG, "write_spectrum: correlation write failed");
    // 1 / (c[m/s] 100 [cm/m] 1e-15 [s/fs]) with c = 299792458 (spectraClass.cu:151-154)
    const double inv_fs_to_inv_cm = 1. / (299792458. * 100. * 1.e-15);
    f = fopen(spec_path, "w");
    if (!f) return ofail(c, DQ_ERR_ARG, std::string("write_spectrum: cannot create ") + spec_path);
    ok = fprintf(f, "{k #} {freq rev/fs} {freq cm^-1} {Transform real imag}: \n") > 0;
    for (int id = 0; id < len && ok; ++id) {
        const int k = id > T / 2 ? -T + id : id;
        ok = fprintf(f, "%6d%14g%14g%14g%14g\n", k, (double)k / (T * dt), inv_fs_to_inv_cm * k / (dt * T), spec[id].x,
                     spec[id].y) > 0;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? DQ_OK : ofail(c, DQ_ERR_ARG, "write_spectrum: spectrum write failed");
}

dq_status dq_write_spectrum(dq_ctx* c, const char* corr_path, const char* spec_path, double scaling) {
    DeviceScope dev_scope(c);
    if (!c || !corr_path || !spec_path) return DQ_ERR_ARG;
    std::vector<cd> corr, spec;
    dq_status st = scaled_spectrum(c, scaling, corr, spec);
    if (st) return st;
    return write_spectrum_files(c, c->steps_done, c->cfg.dt, corr, spec, corr_path, spec_path);
}

// The overall spectrum files over the polarisation directions (spectraClass.cu:
// 697-744): the mean of the directions' scaled correlations and transforms.
dq_status dq_write_spectrum_mean(dq_ctx* const* ctxs, int n_ctx, const double* scalings, const char* corr_path,
                                 const char* spec_path) {
    if (!ctxs || n_ctx < 1 || !scalings || !corr_path || !spec_path) return DQ_ERR_ARG;
    dq_ctx* c0 = ctxs[0];
    if (!c0) return DQ_ERR_ARG;
    const int T = c0->steps_done;
    std::vector<cd> corr(T + 1, cd{0.0, 0.0}), spec(T + 1, cd{0.0, 0.0}), ci, si;
    for (int k = 0; k < n_ctx; ++k) {
        dq_ctx* c = ctxs[k];
        if (!c) return DQ_ERR_ARG;
        if (c->steps_done != T || c->cfg.dt != c0->cfg.dt)
            return ofail(c0, DQ_ERR_ARG, "write_spectrum_mean: the contexts differ in steps done or dt");
        dq_status st;
        {
            DeviceScope dev_scope(c);
            st = scaled_spectrum(c, scalings[k], ci, si);
        }
        if (st) {
            if (c != c0) c0->err = c->err;
            return st;
        }
        for (int i = 0; i <= T; ++i) {
            corr[i].x += ci[i].x;
            corr[i].y += ci[i].y;
            spec[i].x += si[i].x;
            spec[i].y += si[i].y;
        }
    }
    for (int i = 0; i <= T; ++i) {
        corr[i].x /= n_ctx;
        corr[i].y /= n_ctx;
        spec[i].x /= n_ctx;
        spec[i].y /= n_ctx;
    }
    return write_spectrum_files(c0, T, c0->cfg.dt, corr, spec, corr_path, spec_path);
}

}  // extern "C"
