// TEST INFRASTRUCTURE.  A C entry point over the reference's own input-line
// functions stringSplit and stringTrim (cppUtility.cpp:82-106), compiled from
// the reference's source into oracle/_ref/libref_infile.so, so that the
// tests can check this build's input-file parser against the reference's code
// line by line.  It repeats the loop body of systemClass::parseInFile
// (systemClass.cu:239-250): lines with '=' are split and trimmed, keys with
// '!' are skipped.
#include <cstdio>
#include <stdexcept>
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
