// TEST INFRASTRUCTURE.  C entry points over the reference's own input-line
// functions stringSplit and stringTrim (cppUtility.cpp:82-106), compiled from
// the reference's source into oracle/_ref/libref_infile.so, so that the
// tests can check this build's input-file parser against the reference's code
// line by line.  It repeats the loop body of systemClass::parseInFile
// (systemClass.cu:239-250): lines with '=' are split and trimmed, keys with
// '!' are skipped.
#include <cstdio>
#include <stdexcept>
#include <cuComplex.h>
#include <string>

void stringSplit(std::string& str, std::string& str1, std::string& str2, char chrSplit);
void stringTrim(std::string& str);

extern "C" int ref_parse_line(const char* line, char* key, int klen, char* val, int vlen) {
    std::string s(line), k, v;
    if (s.find('=') == std::string::npos) return 0;   // not an assignment
    try {
        stringSplit(s, k, v, '=');
    } catch (const std::out_of_range&) {
        return -1;   // the reference's substr throws (a line ending in '=')
    }
    stringTrim(k);
    stringTrim(v);
    if (k.find('!') != std::string::npos) return 2;   // skipped key
    snprintf(key, (size_t)klen, "%s", k.c_str());
    snprintf(val, (size_t)vlen, "%s", v.c_str());
    return 1;
}

// The reference's exponent coefficient and Taylor coefficients, from its own
// functions (cppUtility.cpp:10-37, 39-72, 76-79; used at propagate.cu:92-93 and
// taylorKrylovClass.cu:202-206): expCoeff = (0, -dt/hbar), c_k = expCoeff^k / k!.
cuDoubleComplex get_neg_inv_hbar_imag();
cuDoubleComplex powComplex(cuDoubleComplex inVal, int n);
int helperFactorial(int n);

extern "C" void ref_exp_coeff(double dt, double* re, double* im) {
    cuDoubleComplex e = get_neg_inv_hbar_imag();
    e.y = e.y * dt;
    *re = e.x;
    *im = e.y;
}

extern "C" void ref_taylor_coeff(double dt, int k, double* re, double* im) {
    cuDoubleComplex e = get_neg_inv_hbar_imag();
    e.y = e.y * dt;
    cuDoubleComplex c = powComplex(e, k);
    c.x /= helperFactorial(k);
    c.y /= helperFactorial(k);
    *re = c.x;
    *im = c.y;
}
