// dq_host_internal.h — shared pieces of the C++ host (parser, file readers,
// driver); nothing here is part of the C ABI.
#pragma once
#include <string>
#include <vector>

namespace dqh {

void put_err(char* buf, int len, const std::string& msg);
void split_line(const std::string& line, std::string& key, std::string& val);
void trim_tabs_then_spaces(std::string& s);

// A Hamiltonian file as the propagator takes it: full CSR, diagonal included.
struct Csr {
    int n = 0;
    std::vector<int> rowptr, col;
    std::vector<double> val;
};

// Each reader returns false and sets err on a malformed file.
bool read_hamiltonian(const std::string& path, Csr& out, std::string& err);
bool read_ka_params(const std::string& path, int n, std::vector<double>& sigma, std::vector<double>& tau,
                    std::string& err);
bool read_hsr_stddev(const std::string& path, int n, std::vector<double>& sigma, std::string& err);
bool read_initial_state(const std::string& path, int n, std::vector<double>& re, std::string& err);
bool read_vectors3(const std::string& path, int n, std::vector<double>& xyz, std::string& err);
bool read_spectral_density(const std::string& path, double& d_omega, std::vector<double>& omega,
                           std::vector<double>& J, std::string& err);

}  // namespace dqh
