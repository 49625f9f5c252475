// dq_host_parse.cpp — the reference's `key = value` input file
// (systemClass::parseInFile, systemClass.cu:184-735; stringSplit and
// stringTrim, cppUtility.cpp:82-106), read into a dq_infile.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "../../include/dq_host.h"
#include "dq_host_internal.h"

namespace dqh {

void put_err(char* buf, int len, const std::string& msg) {
    if (buf && len > 0) snprintf(buf, (size_t)len, "%s", msg.c_str());
}

// The key is what precedes the first '='; the value starts two characters
// after it (the reference assumes "key = value" with one blank after '=').
// Where that start lies past the end the value is empty (the reference's
// substr would throw there).
void split_line(const std::string& line, std::string& key, std::string& val) {
    const size_t pos = line.find('=');
    key = line.substr(0, pos);
    val = (pos + 2 <= line.size()) ? line.substr(pos + 2) : std::string();
}

// Leading and trailing tabs are removed first, then leading and trailing
// spaces: one pass of each, in that order, so a blank before a tab survives.
void trim_tabs_then_spaces(std::string& s) {
    for (char ch : {'\t', ' '}) {
        const size_t a = s.find_first_not_of(ch), b = s.find_last_not_of(ch);
        if (a == std::string::npos) s.clear();
        else s = s.substr(a, b - a + 1);
    }
}

}  // namespace dqh

using namespace dqh;

namespace {

bool flag01(const std::string& key, const std::string& val, int* out, std::string& err) {
    const int v = atoi(val.c_str());
    if (v != 0 && v != 1) {
        err = "ERROR. " + key + " must be 0 or 1. Aborting.";
        return false;
    }
    *out = v;
    return true;
}

void put_str(char* dst, const std::string& v) {
    snprintf(dst, DQ_HOST_PATH_MAX, "%s", v.c_str());
}

}  // namespace

extern "C" {

void dq_infile_defaults(dq_infile* in) {
    if (!in) return;
    std::memset(in, 0, sizeof(*in));
    // systemClass.cu:30-80
    in->simtype = DQ_SIM_CONST_HAM;
    in->propmode = DQ_PROP_LANCZOS;
    in->initstate = 0;
    in->ensembleavgmode = DQ_ENS_AVG_NONE;
    in->temperature = -1.0;
    in->tk_p = 10;
    in->tk_m_aux = 24;
    put_str(in->outfolder, "outFolderDefault");
    for (int i = 0; i < 10; ++i) in->printpop[i] = -1;
    // left unset by the reference (so every run file names them); these keep a context valid
    in->dt = 1.0;
    in->m = 16;
    in->ka_substeps = 1;
    in->ensembleruns = 1;
    in->gausswidth = 1.0;
    in->stepsperloop = 0;
    // this build's keys
    in->precision = DQ_PREC_FP64;
    in->seed = 0;
    in->pop_every = 1;
}

int dq_infile_split_line(const char* line, char* key, int key_len, char* value, int value_len) {
    if (!line) return 0;
    const std::string s(line);
    if (s.find('=') == std::string::npos) return 0;
    std::string k, v;
    split_line(s, k, v);
    trim_tabs_then_spaces(k);
    trim_tabs_then_spaces(v);
    if (k.find('!') != std::string::npos) return 2;
    if (key && key_len > 0) snprintf(key, (size_t)key_len, "%s", k.c_str());
    if (value && value_len > 0) snprintf(value, (size_t)value_len, "%s", v.c_str());
    return 1;
}

dq_status dq_infile_parse(const char* path, dq_infile* out, char* errbuf, int errbuf_len) {
    if (!path || !out) {
        put_err(errbuf, errbuf_len, "infile_parse: null argument");
        return DQ_ERR_ARG;
    }
    dq_infile in;
    dq_infile_defaults(&in);
    std::ifstream f(path);
    if (!f.is_open()) {
        put_err(errbuf, errbuf_len, std::string("ERROR. inFile failed to open: ") + path);
        return DQ_ERR_ARG;
    }
    std::string line, err;
    auto bad = [&](const std::string& msg) {
        put_err(errbuf, errbuf_len, msg);
        return DQ_ERR_ARG;
    };
    while (std::getline(f, line)) {
        if (line.find('=') == std::string::npos) continue;
        std::string k, v;
        split_line(line, k, v);
        trim_tabs_then_spaces(k);
        trim_tabs_then_spaces(v);
        if (k.find('!') != std::string::npos) continue;
        in.n_assignments++;
        const char* cv = v.c_str();
        if (k == "dt") in.dt = atof(cv);
        else if (k == "temperature") in.temperature = atof(cv);
        else if (k == "debug_diags") { if (!flag01(k, v, &in.debug_diags, err)) return bad(err); }
        else if (k.size() == 9 && k.compare(0, 8, "printpop") == 0 && k[8] >= '0' && k[8] <= '9')
            in.printpop[k[8] - '0'] = atoi(cv);
        else if (k == "print_partic") { if (!flag01(k, v, &in.print_partic, err)) return bad(err); }
        else if (k == "totalsteps") in.totalsteps = atoi(cv);
        else if (k == "ensembleavgmode") {
            // an unknown name falls back to ENS_AVG_MODE_NONE (systemClass.cu:322-331)
            if (v == "ENS_AVG_MODE_FIRST") in.ensembleavgmode = DQ_ENS_AVG_FIRST;
            else if (v == "ENS_AVG_MODE_CONTINUATION") in.ensembleavgmode = DQ_ENS_AVG_CONTINUATION;
            else in.ensembleavgmode = DQ_ENS_AVG_NONE;
        }
        else if (k == "ensembleruns") in.ensembleruns = atoi(cv);
        else if (k == "m") in.m = atoi(cv);
        else if (k == "ka_substeps") in.ka_substeps = atoi(cv);
        else if (k == "dostatelooping") { if (!flag01(k, v, &in.dostatelooping, err)) return bad(err); }
        else if (k == "writeoutpops") { if (!flag01(k, v, &in.writeoutpops, err)) return bad(err); }
        else if (k == "writebinarypops") { if (!flag01(k, v, &in.writebinarypops, err)) return bad(err); }
        else if (k == "printallpops") { if (!flag01(k, v, &in.printallpops, err)) return bad(err); }
        else if (k == "writeoutstates") {
            // a period in steps; the reference writes states when it is positive
            in.writeoutstates = atoi(cv);
        }
        else if (k == "stepsperloop") in.stepsperloop = atoi(cv);
        else if (k == "outfolder") put_str(in.outfolder, v);
        else if (k == "hamfile") put_str(in.hamfile, v);
        else if (k == "statefile") put_str(in.statefile, v);
        else if (k == "outfile") put_str(in.outfile, v);
        else if (k == "tkmatfile") put_str(in.tkmatfile, v);
        else if (k == "tk_p") in.tk_p = atoi(cv);
        else if (k == "tk_m_aux") in.tk_m_aux = atoi(cv);
        else if (k == "simtype") {
            if (v == "SIM_TYPE_CONST_HAM") in.simtype = DQ_SIM_CONST_HAM;
            else if (v == "SIM_TYPE_HSR") in.simtype = DQ_SIM_HSR;
            else if (v == "SIM_TYPE_KUBO_ANDERSON") in.simtype = DQ_SIM_KUBO_ANDERSON;
            else if (v == "SIM_TYPE_ZZ_REAL_NOISE") in.simtype = DQ_SIM_ZZ_REAL_NOISE;
            else if (v == "SIM_TYPE_ZZ_COMPLEX_NOISE") in.simtype = DQ_SIM_ZZ_COMPLEX_NOISE;
            else return bad("ERROR. Unknown simtype '" + v + "'. Aborting.");
        }
        else if (k == "propmode") {
            if (v == "PROP_MODE_LANCZOS") in.propmode = DQ_PROP_LANCZOS;
            else if (v == "PROP_MODE_TAYLOR_LANCZOS") in.propmode = DQ_PROP_TAYLOR_LANCZOS;
            else return bad("ERROR. Unknown propmode '" + v + "'. Aborting.");
        }
        else if (k == "staticdis") { if (!flag01(k, v, &in.staticdis, err)) return bad(err); }
        else if (k == "sigmastatdis") in.sigmastatdis = atof(cv);
        else if (k == "hsr_stddevfile") put_str(in.hsr_stddevfile, v);
        else if (k == "ka_paramsfile") put_str(in.ka_paramsfile, v);
        else if (k == "zz_specd_file") put_str(in.zz_specd_file, v);
        else if (k == "absorbspec") {
            if (!flag01(k, v, &in.absorbspec, err)) return bad(err);
            if (in.absorbspec && in.cdspec) return bad("ERROR. Cannot do both absorbspec and cdspec. Aborting.");
        }
        else if (k == "cdspec") {
            if (!flag01(k, v, &in.cdspec, err)) return bad(err);
            if (in.absorbspec && in.cdspec) return bad("ERROR. Cannot do both absorbspec and cdspec. Aborting.");
        }
        else if (k == "lineshapedress") { if (!flag01(k, v, &in.lineshapedress, err)) return bad(err); }
        else if (k == "gausswidth") in.gausswidth = atof(cv);
        else if (k == "dipolefile") put_str(in.dipolefile, v);
        else if (k == "posfile") put_str(in.posfile, v);
        else if (k == "initstate") in.initstate = atoi(cv);
        else if (k == "initfromfile") { if (!flag01(k, v, &in.initfromfile, err)) return bad(err); }
        else if (k == "initstatefile") put_str(in.initstatefile, v);
        // this build's keys
        else if (k == "precision") {
            if (v == "PREC_FP64") in.precision = DQ_PREC_FP64;
            else if (v == "PREC_MIXED") in.precision = DQ_PREC_MIXED;
            else return bad("ERROR. precision must be PREC_FP64 or PREC_MIXED. Aborting.");
        }
        else if (k == "seed") in.seed = strtoull(cv, nullptr, 10);
        else if (k == "pop_every") in.pop_every = atoi(cv);
        else in.n_unknown++;   // the reference's empty default branch
    }
    *out = in;
    return DQ_OK;
}

}  // extern "C"
