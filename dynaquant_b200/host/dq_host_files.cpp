// dq_host_files.cpp — readers of the reference's data files, in its formats:
//   hamfile         matCooClass::readInFile (sparseMatrixClasses.cu:75-230)
//   ka_paramsfile   prepForKA (systemClass.cu:982-1071): "relaxTime stdDev" per site
//   hsr_stddevfile  prepForHsr (systemClass.cu:912-975): one standard deviation per line
//   initstatefile   initStateFromFile (systemClass.cu:1385-1481)
//   dipolefile / posfile  prepForAbsorb / prepForCD (spectraClass.cu:300-430)
//   zz_specd_file   prepForZZReal (systemClass.cu:1077-1207): "dOmega nOsc", then "omega J"
#include <algorithm>
#include <cmath>
#include <fstream>
#include <numeric>
#include <sstream>

#include "dq_host_internal.h"

namespace dqh {

bool read_hamiltonian(const std::string& path, Csr& out, std::string& err) {
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "ERROR. Matrix file '" + path + "' failed to open.";
        return false;
    }
    std::string line, w0, w1, w2, value_type, kind;
    std::getline(f, line);
    {
        std::istringstream ss(line);
        ss >> w0 >> w1 >> w2 >> value_type >> kind;
    }
    if (kind != "general" && kind != "symmetric" && kind != "hermitian") {
        err = path + ": unknown matrix type '" + kind + "'";
        return false;
    }
    std::getline(f, line);
    int base;
    if (line == "BASE_ZERO") base = 0;
    else if (line == "BASE_ONE") base = 1;
    else {
        err = path + ": the second line must be BASE_ZERO or BASE_ONE";
        return false;
    }
    int n = 0, n2 = 0;
    long long nnz = 0;
    std::getline(f, line);
    {
        std::istringstream ss(line);
        ss >> n >> n2 >> nnz;
    }
    if (n <= 0 || nnz <= 0) {
        err = path + ": N and nnz must be positive";
        return false;
    }
    struct E { int i, j; double v; };
    std::vector<E> e;
    e.reserve((size_t)nnz * (kind == "general" ? 1 : 2));
    long long counter = 0;
    while (std::getline(f, line)) {
        // lines beyond nnz are ignored with a warning in the reference
        if (counter++ >= nnz) continue;
        std::istringstream ss(line);
        int i, j;
        double v = 0.0;
        if (!(ss >> i >> j)) continue;
        ss >> v;   // the value is the real part; Hamiltonians are real
        i -= base;
        j -= base;
        if (i < 0 || i >= n || j < 0 || j >= n) {
            err = path + ": index outside the matrix";
            return false;
        }
        if (kind == "general") {
            e.push_back({i, j, v});
        } else if (i >= j) {
            // symmetric/hermitian: the lower triangle, mirrored (cuSPARSE's
            // FILL_MODE_LOWER view of the matrix the reference hands it)
            e.push_back({i, j, v});
            if (i != j) e.push_back({j, i, v});
        }
    }
    std::stable_sort(e.begin(), e.end(), [](const E& a, const E& b) { return a.i != b.i ? a.i < b.i : a.j < b.j; });
    out.n = n;
    out.rowptr.assign(n + 1, 0);
    out.col.resize(e.size());
    out.val.resize(e.size());
    for (size_t k = 0; k < e.size(); ++k) {
        out.rowptr[e[k].i + 1]++;
        out.col[k] = e[k].j;
        out.val[k] = e[k].v;
    }
    std::partial_sum(out.rowptr.begin(), out.rowptr.end(), out.rowptr.begin());
    return true;
}

bool read_ka_params(const std::string& path, int n, std::vector<double>& sigma, std::vector<double>& tau,
                    std::string& err) {
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "ERROR. KA parameter file '" + path + "' failed to open.";
        return false;
    }
    // a site without a line keeps no noise (zero standard deviation), as the
    // reference's zero-initialised arrays leave it
    sigma.assign(n, 0.0);
    tau.assign(n, 1.0);
    int counter = 0;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        double t, s;
        if (!(ss >> t >> s)) continue;
        if (counter < n) {
            tau[counter] = t;
            sigma[counter] = s;
        }
        counter++;
    }
    if (counter < n - 1) {
        err = path + ": fewer lines than sites";
        return false;
    }
    return true;
}

bool read_hsr_stddev(const std::string& path, int n, std::vector<double>& sigma, std::string& err) {
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "ERROR. HSR file '" + path + "' failed to open.";
        return false;
    }
    sigma.assign(n, 0.0);
    int counter = 0;
    std::string line;
    while (std::getline(f, line)) {
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
        if (counter < n) sigma[counter] = atof(line.c_str());
        counter++;
    }
    if (counter < n - 1) {
        err = path + ": fewer lines than sites";
        return false;
    }
    return true;
}

bool read_initial_state(const std::string& path, int n, std::vector<double>& re, std::string& err) {
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "ERROR. State file '" + path + "' failed to open.";
        return false;
    }
    std::string line;
    std::getline(f, line);
    int off;
    if (line == "BASE_ZERO") off = 0;
    else if (line == "BASE_ONE") off = 1;
    else {
        err = path + ": the first line must be BASE_ZERO or BASE_ONE";
        return false;
    }
    std::getline(f, line);   // comment line
    re.assign(n, 0.0);
    while (std::getline(f, line)) {
        if (line.find("END") != std::string::npos) break;
        std::istringstream ss(line);
        int i;
        float coeff;   // the reference reads the amplitude into a float
        if (!(ss >> i >> coeff)) continue;
        i -= off;
        if (i < 0 || i >= n) {
            err = path + ": site outside the system";
            return false;
        }
        re[i] = (double)coeff;
    }
    double s = 0.0;
    for (double v : re) s += v * v;
    if (!(s > 0.0)) {
        err = path + ": the state is zero";
        return false;
    }
    const double inv = 1.0 / std::sqrt(s);
    for (double& v : re) v *= inv;
    return true;
}

bool read_vectors3(const std::string& path, int n, std::vector<double>& xyz, std::string& err) {
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "ERROR. File '" + path + "' failed to open.";
        return false;
    }
    xyz.assign((size_t)3 * n, 0.0);
    int counter = 0;
    std::string line;
    while (std::getline(f, line) && counter < n) {
        std::istringstream ss(line);
        double a, b, c;
        if (!(ss >> a >> b >> c)) continue;
        xyz[(size_t)3 * counter] = a;
        xyz[(size_t)3 * counter + 1] = b;
        xyz[(size_t)3 * counter + 2] = c;
        counter++;
    }
    if (counter < n) {
        err = path + ": fewer lines than sites";
        return false;
    }
    return true;
}

bool read_spectral_density(const std::string& path, double& d_omega, std::vector<double>& omega,
                           std::vector<double>& J, std::string& err) {
    std::ifstream f(path);
    if (!f.is_open()) {
        err = "ERROR. Spectral density file '" + path + "' failed to open.";
        return false;
    }
    std::string line;
    std::getline(f, line);
    int n_osc = 0;
    {
        std::istringstream ss(line);
        ss >> d_omega >> n_osc;
    }
    if (n_osc <= 0) {
        err = path + ": no oscillators";
        return false;
    }
    omega.clear();
    J.clear();
    while (std::getline(f, line) && (int)omega.size() < n_osc) {
        std::istringstream ss(line);
        double w, j;
        if (!(ss >> w >> j)) continue;
        omega.push_back(w);
        J.push_back(j);
    }
    if ((int)omega.size() < n_osc) {
        err = path + ": fewer oscillator lines than its header states";
        return false;
    }
    return true;
}

}  // namespace dqh
