/*
 * oracle/shim/compat.h -- test infrastructure only; force-included (-include) by
 * oracle/Makefile into every reference translation unit.
 *
 * rlm/matrix_coefficients.cpp:11 multiplies complex<double> by float values
 * (expf(...) and 1.0f/n_phi) in the -DDP build.  The Intel compiler the reference was
 * built with accepted this; libstdc++'s operator* templates do not deduce a common
 * type for it under g++.  These two overloads give the only meaningful reading: the
 * float operand is promoted to double, so the single-precision expf result and the
 * float reciprocal enter the double-precision table unchanged, exactly as written.
 */
#ifndef RLMB_ORACLE_COMPAT_H
#define RLMB_ORACLE_COMPAT_H
#include <complex>
static inline std::complex<double> operator*(const std::complex<double>& a, float b) {
    return a * (double)b;
}
static inline std::complex<double> operator*(float b, const std::complex<double>& a) {
    return (double)b * a;
}
#endif
