/* Force-included (nvcc -include) ahead of every reference .cu file.
 * nvcc's host front end rejects glibc's imaginary-unit literal behind the C99
 * macro I.  The reference's VERTEX struct (include/FAME_Internal_Common.h) has a
 * member named I, so that header is pulled in first with I undefined, and only
 * then is I redefined as an expression that builds 0+1i without the literal. */
#ifndef FAME_REF_PRELUDE_H
#define FAME_REF_PRELUDE_H
#include "FAME_Internal_Common.h"
#include <complex.h>
static inline double _Complex fame_ref_imag_unit(void) {
  double _Complex z;
  reinterpret_cast<double*>(&z)[0] = 0.0;
  reinterpret_cast<double*>(&z)[1] = 1.0;
  return z;
}
#undef I
#define I (fame_ref_imag_unit())
#endif
