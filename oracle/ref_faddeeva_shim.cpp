// Test infrastructure only (oracle side): a C-linkage wrapper around the
// reference's vendored Faddeeva package, compiled from the reference's own
// src/Faddeeva.cpp into oracle/_ref/libfaddeeva_ref.so by oracle/Makefile.
//
// The reference calls Faddeeva::w at Bunch.cpp:147 and Bunch.cpp:150 (inside
// Bunch::BassettiErskine1, Bunch.cpp:119-170).  This wrapper exposes exactly
// that function over plain arrays so that the Python tests can compare the
// CPU oracle and the GPU kernels against the reference's own w(z).
#include <complex>
#include <cstdint>
#include "Faddeeva.h"

extern "C" {

// w(z) for n points; relerr = 0 (the default used by Bunch.cpp:147/150).
void ref_faddeeva_w(const double* zr, const double* zi, double* wr, double* wi,
                    int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    std::complex<double> w = Faddeeva::w(std::complex<double>(zr[i], zi[i]));
    wr[i] = w.real();
    wi[i] = w.imag();
  }
}

}  // extern "C"
