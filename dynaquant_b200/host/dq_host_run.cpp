// dq_host_run.cpp — the run driver of an input file: the reference's main
// (propagate.cu:29-298) over the C ABI of include/dq.h.
//
// The reference runs its ensemble one run after another, each run a fresh
// realisation of the noise, and adds every run's populations into pops.dat
// (popPrintClass) and its correlation into the spectrum.  Here the runs of one
// initial condition are the trajectories of one batched ensemble (dq_run), and
// the files are written from the ensemble's sums, so they hold what the
// reference's files hold after its last run.  Lanczos steps use the
// reference's conventions: the unconjugated alpha (cublasZdotu,
// lanczosClass.cu:421) and |Re|-only Padé row sums (gpuPadeHelper.cu:25).
#include <sys/stat.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/dq_host.h"
#include "dq_host_internal.h"

using namespace dqh;

namespace {

std::string resolve(const char* base, const char* p) {
    std::string s(p);
    if (s.empty() || s[0] == '/' || !base || !*base) return s;
    std::string b(base);
    if (b.back() != '/') b += '/';
    return b + s;
}

struct Ctx {
    dq_ctx* h = nullptr;
    ~Ctx() { if (h) dq_destroy(h); }
};

// One polarisation direction of a spectrum run (spectraClass.cu:356-496).
struct Direction {
    std::vector<dq_cdouble> psi0;
    std::vector<dq_cdouble> bra;   // CD only
    double scaling = 1.0;
};

float as_float(double x) { return (float)x; }

}  // namespace

extern "C" dq_status dq_infile_run(const dq_infile* in, const char* base_dir, int device, char* errbuf,
                                   int errbuf_len) {
    auto bad = [&](int code, const std::string& msg) {
        put_err(errbuf, errbuf_len, msg);
        return code;
    };
    if (!in) return bad(DQ_ERR_ARG, "infile_run: null input");
    if (!in->hamfile[0]) return bad(DQ_ERR_ARG, "infile_run: no hamfile");
    if (in->totalsteps < 1) return bad(DQ_ERR_ARG, "infile_run: totalsteps must be positive");
    if (!(in->dt > 0)) return bad(DQ_ERR_ARG, "infile_run: dt must be positive");
    if (in->simtype == DQ_SIM_ZZ_REAL_NOISE && !(in->temperature > 0))
        return bad(DQ_ERR_ARG, "ERROR. temperature must be positive for SIM_TYPE_ZZ_REAL_NOISE. Aborting.");
    std::string err;
    Csr H;
    if (!read_hamiltonian(resolve(base_dir, in->hamfile), H, err)) return bad(DQ_ERR_ARG, err);
    const int n = H.n;
    const std::string out_dir = resolve(base_dir, in->outfolder);
    struct stat sb;
    if (stat(out_dir.c_str(), &sb) == -1) mkdir(out_dir.c_str(), 0700);   // systemClass.cu:652-656

    // noise model and its per-site parameters
    int noise = DQ_NOISE_NONE;
    std::vector<double> sigma, tau, zz_om, zz_J;
    double zz_dom = 0.0;
    if (in->simtype == DQ_SIM_KUBO_ANDERSON) {
        noise = DQ_NOISE_OU;
        if (!read_ka_params(resolve(base_dir, in->ka_paramsfile), n, sigma, tau, err)) return bad(DQ_ERR_ARG, err);
    } else if (in->simtype == DQ_SIM_HSR) {
        noise = DQ_NOISE_GAUSS;
        if (!read_hsr_stddev(resolve(base_dir, in->hsr_stddevfile), n, sigma, err)) return bad(DQ_ERR_ARG, err);
    } else if (in->simtype == DQ_SIM_ZZ_REAL_NOISE) {
        noise = DQ_NOISE_ZZ;
        if (!read_spectral_density(resolve(base_dir, in->zz_specd_file), zz_dom, zz_om, zz_J, err))
            return bad(DQ_ERR_ARG, err);
    }
    // SIM_TYPE_ZZ_COMPLEX_NOISE is parsed by the reference but its Hamiltonian
    // update does nothing for it (systemClass.cu:1883-1897): a constant Hamiltonian

    // initial conditions: one state, or the three polarisation directions
    std::vector<Direction> dirs;
    const bool spec = in->absorbspec || in->cdspec;
    if (spec) {
        std::vector<double> mu, R;
        if (!read_vectors3(resolve(base_dir, in->dipolefile), n, mu, err)) return bad(DQ_ERR_ARG, err);
        if (in->cdspec && !read_vectors3(resolve(base_dir, in->posfile), n, R, err)) return bad(DQ_ERR_ARG, err);
        std::vector<double> rd;
        if (in->cdspec) {
            rd.resize((size_t)3 * n);
            for (int i = 0; i < n; ++i) {
                const double* m = &mu[(size_t)3 * i];
                const double* r = &R[(size_t)3 * i];
                rd[(size_t)3 * i] = r[1] * m[2] - r[2] * m[1];
                rd[(size_t)3 * i + 1] = r[2] * m[0] - r[0] * m[2];
                rd[(size_t)3 * i + 2] = r[0] * m[1] - r[1] * m[0];
            }
        }
        for (int d = 0; d < 3; ++d) {
            double mt = 0.0, rt = 0.0;
            for (int i = 0; i < n; ++i) mt += mu[(size_t)3 * i + d] * mu[(size_t)3 * i + d];
            mt = std::sqrt(mt);
            if (in->cdspec) {
                for (int i = 0; i < n; ++i) rt += rd[(size_t)3 * i + d] * rd[(size_t)3 * i + d];
                rt = std::sqrt(rt);
            }
            Direction D;
            D.psi0.resize(n);
            if (in->absorbspec) {
                if (!(mt > 0)) return bad(DQ_ERR_ARG, "infile_run: a dipole direction has zero norm");
                for (int i = 0; i < n; ++i) D.psi0[i] = dq_cdouble{mu[(size_t)3 * i + d] / mt, 0.0};
                D.scaling = (double)as_float(mt * mt);   // held in a float (spectraClass.cu:640-651)
            } else {
                if (!(mt > 0) || !(rt > 0)) return bad(DQ_ERR_ARG, "infile_run: a CD direction has zero norm");
                D.bra.resize(n);
                for (int i = 0; i < n; ++i) {
                    D.psi0[i] = dq_cdouble{rd[(size_t)3 * i + d] / rt, 0.0};
                    D.bra[i] = dq_cdouble{mu[(size_t)3 * i + d] / mt, 0.0};
                }
                const float pi_half = as_float(3.1415926535f / 2.0f);
                float sc = as_float((double)pi_half * 1e-7);
                sc = as_float((double)sc * (mt * rt));
                D.scaling = (double)sc;
            }
            dirs.push_back(std::move(D));
        }
    } else {
        Direction D;
        D.psi0.assign(n, dq_cdouble{0.0, 0.0});
        if (in->initfromfile) {
            std::vector<double> re;
            if (!read_initial_state(resolve(base_dir, in->initstatefile), n, re, err)) return bad(DQ_ERR_ARG, err);
            for (int i = 0; i < n; ++i) D.psi0[i].re = re[i];
        } else {
            if (in->initstate < 0 || in->initstate >= n) return bad(DQ_ERR_ARG, "infile_run: initstate outside the system");
            D.psi0[in->initstate].re = 1.0;
        }
        dirs.push_back(std::move(D));
    }

    Csr Bm;
    if (in->propmode == DQ_PROP_TAYLOR_LANCZOS) {
        if (!read_hamiltonian(resolve(base_dir, in->tkmatfile), Bm, err)) return bad(DQ_ERR_ARG, err);
        if (Bm.n != n) return bad(DQ_ERR_ARG, "infile_run: tkmatfile size differs from hamfile");
    }

    const int runs = in->ensembleavgmode == DQ_ENS_AVG_NONE ? 1 : std::max(1, in->ensembleruns);
    std::vector<Ctx> ctxs(dirs.size());
    for (size_t d = 0; d < dirs.size(); ++d) {
        dq_config cfg;
        dq_config_default(&cfg);
        cfg.n_sites = n;
        cfg.m = in->m;
        cfg.n_traj = runs;
        cfg.dt = in->dt;
        cfg.noise_model = noise;
        cfg.ka_substeps = in->ka_substeps > 0 ? in->ka_substeps : 1;
        cfg.sigma_static = in->staticdis ? in->sigmastatdis : 0.0;
        cfg.seed = in->seed;
        cfg.dot_mode = DQ_DOT_BILINEAR;
        cfg.norm_mode = DQ_NORM_REAL_ONLY;
        cfg.precision = in->precision;
        cfg.pop_every = in->pop_every > 0 ? in->pop_every : 1;
        cfg.max_steps = in->totalsteps;
        cfg.device = device;
        dq_status st = dq_create(&cfg, &ctxs[d].h);
        if (st) return bad(st, "infile_run: dq_create failed (configuration or CUDA)");
        dq_ctx* c = ctxs[d].h;
        auto chk = [&](dq_status s, const char* what) {
            if (s) put_err(errbuf, errbuf_len, std::string(what) + ": " + dq_last_error(c));
            return s;
        };
        if ((st = chk(dq_set_hamiltonian_csr(c, n, H.rowptr.data(), H.col.data(), H.val.data()), "hamfile")))
            return st;
        if (noise == DQ_NOISE_OU || noise == DQ_NOISE_GAUSS) {
            if ((st = chk(dq_set_noise_params(c, sigma.data(), noise == DQ_NOISE_OU ? tau.data() : nullptr),
                          "noise parameters")))
                return st;
        } else if (noise == DQ_NOISE_ZZ) {
            if ((st = chk(dq_set_zz_spectral_density(c, (int)zz_om.size(), zz_om.data(), zz_J.data(), zz_dom,
                                                     in->temperature),
                          "spectral density")))
                return st;
        }
        if ((st = chk(dq_set_initial_state(c, dirs[d].psi0.data()), "initial state"))) return st;
        if (!dirs[d].bra.empty() && (st = chk(dq_set_correlation_bra(c, dirs[d].bra.data()), "CD bra"))) return st;
        if (spec && in->lineshapedress && (st = chk(dq_set_line_dressing(c, in->gausswidth), "line dressing")))
            return st;
        if (in->print_partic && (st = chk(dq_set_ipr(c, 1), "IPR"))) return st;
        if (in->propmode == DQ_PROP_TAYLOR_LANCZOS &&
            (st = chk(dq_set_taylor_krylov(c, in->tk_p, in->tk_m_aux, Bm.rowptr.data(), Bm.col.data(), Bm.val.data()),
                      "Taylor-Krylov")))
            return st;
        // every direction's runs are fresh realisations of the noise
        if ((st = chk(dq_set_trajectory_offset(c, (int)d * ((runs + 1) & ~1)), "trajectory offset"))) return st;
        // the steps, with the state files every writeoutstates steps (statePrintClass)
        const int every = in->writeoutstates > 0 ? in->writeoutstates : in->totalsteps;
        for (int done = 0; done < in->totalsteps;) {
            const int k = std::min(every, in->totalsteps - done);
            if ((st = chk(dq_run(c, k), "run"))) return st;
            done += k;
            if (in->writeoutstates > 0 && done % in->writeoutstates == 0 &&
                (st = chk(dq_write_states(c, out_dir.c_str()), "states")))
                return st;
        }
        // pops.dat holds the sums over every run of every initial condition
        // (popPrintClass turns continuation on after the first run)
        if (in->writeoutpops && in->printallpops) {
            const int cont = (d > 0 || in->ensembleavgmode == DQ_ENS_AVG_CONTINUATION) ? 1 : 0;
            if ((st = chk(dq_write_populations(c, (out_dir + "/pops.dat").c_str(), in->writebinarypops, cont),
                          "pops.dat")))
                return st;
        }
        if (in->print_partic &&
            (st = chk(dq_write_ipr(c, resolve(base_dir, "invParticRat.dat").c_str()), "invParticRat.dat")))
            return st;
    }
    if (spec) {
        const char* tag = in->absorbspec ? "abs" : "CD";
        std::vector<dq_ctx*> hs;
        std::vector<double> scal;
        for (size_t d = 0; d < dirs.size(); ++d) {
            const std::string cp = out_dir + "/" + tag + "CorrFuncDir" + std::to_string(d) + ".dat";
            const std::string sp = out_dir + "/" + tag + "Dir" + std::to_string(d) + ".dat";
            dq_status st = dq_write_spectrum(ctxs[d].h, cp.c_str(), sp.c_str(), dirs[d].scaling);
            if (st) return bad(st, std::string("spectrum: ") + dq_last_error(ctxs[d].h));
            hs.push_back(ctxs[d].h);
            scal.push_back(dirs[d].scaling);
        }
        const std::string cp = out_dir + "/" + tag + "CorrFunc.dat";
        const std::string sp = out_dir + (in->absorbspec ? "/absorption.dat" : "/CD.dat");
        dq_status st = dq_write_spectrum_mean(hs.data(), (int)hs.size(), scal.data(), cp.c_str(), sp.c_str());
        if (st) return bad(st, std::string("spectrum mean: ") + dq_last_error(hs[0]));
    }
    return DQ_OK;
}
