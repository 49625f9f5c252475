// Declarations cppUtility.cpp expects from the reference's includeFiles.cu,
// which pulls in the standard headers and the CUDA complex type before it
// (includeFiles.cu:1-70).  Used only to compile that file as it lies in the
// reference tree into oracle/_ref/libref_infile.so (test infrastructure).
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <string>
#include <cuComplex.h>
using namespace std;
