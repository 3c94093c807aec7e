// oracle/ref_pga_harness.cpp -- TEST INFRASTRUCTURE (the oracle), not product.
//
// Compiles the reference's own src/autofocus/cpu/autofocus_cpu.cpp where it
// lies (oracle/Makefile, REF) and exports its PGA routine
//     template <typename T> void autofocus(Complex<T> *data, int numSamples,
//                                          int numRange, int numIterations)
// (autofocus_cpu.cpp:250-474) with C linkage, so that the oracle's
// restatement of that routine (oracle.pga_cpp_reference) and the GPU PGA in
// the same semantics are checked against the reference's compiled code.
// Stand-in headers under oracle/standin/ declare the Eigen and matio names the
// file mentions (neither library is installed); its main() is renamed and
// never called, and the matio functions it would call are failing stubs.
#include <cstdio>

#define main reference_autofocus_cpu_main
#include "src/autofocus/cpu/autofocus_cpu.cpp"
#undef main

// defined in the reference's MAT reader source (not compiled here); only the
// renamed main() refers to them
void initialize_GOTCHA_MATRead(std::unordered_map<std::string, matvar_t *> &) {}
void initialize_Sandia_SPHRead(std::unordered_map<std::string, matvar_t *> &) {}

extern "C" {
mat_t *Mat_Open(const char *, int) { return nullptr; }
int Mat_Close(mat_t *) { return -1; }
matvar_t *Mat_VarReadNext(mat_t *) { return nullptr; }
void Mat_VarFree(matvar_t *) {}
unsigned Mat_VarGetNumberOfFields(matvar_t *) { return 0; }
matvar_t *Mat_VarGetStructFieldByIndex(matvar_t *, size_t, size_t) { return nullptr; }
void Mat_VarPrint(matvar_t *, int) {}
int Mat_VarReadDataAll(mat_t *, matvar_t *) { return -1; }

// data: complex64 [numSamples][numRange] (column-major numRange x numSamples:
// range fastest, as the routine indexes rangeIndex + pulseIndex * numRange),
// corrected in place.  The routine prints its rms per iteration on stdout.
int ref_pga_f32(float *data, int numSamples, int numRange, int numIterations) {
    if (!data || numSamples < 2 || numRange < 1 || numIterations < 0) return -1;
    autofocus<float>(reinterpret_cast<Complex<float> *>(data), numSamples, numRange, numIterations);
    std::fflush(stdout);
    return 0;
}
}
