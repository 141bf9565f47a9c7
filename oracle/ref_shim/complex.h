/* Build-only stand-in for <complex.h> so the reference's C99-complex host
 * code compiles as C++ under nvcc (g++ accepts `_Complex` as a GNU
 * extension).  Only the names the reference uses are provided.  This file
 * is test infrastructure for building the reference binary under
 * oracle/_ref; the product never includes it. */
#ifndef FDTD_REF_SHIM_COMPLEX_H
#define FDTD_REF_SHIM_COMPLEX_H
#define complex _Complex
#ifdef __cplusplus
extern "C" {
#endif
double _Complex cexp(double _Complex);
double creal(double _Complex);
double cimag(double _Complex);
double cabs(double _Complex);
float crealf(float _Complex);
#ifdef __cplusplus
}
#endif
static inline double _Complex fdtd_ref_shim_imag_unit(void) {
  double _Complex z;
  __real__ z = 0.0;
  __imag__ z = 1.0;
  return z;
}
#define I (fdtd_ref_shim_imag_unit())
#endif
