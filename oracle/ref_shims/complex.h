/*
 * TEST INFRASTRUCTURE (oracle build only) -- never linked into the product.
 *
 * Stand-in for <complex.h> used when the reference C++ sources are compiled
 * by g++ in C++ mode.  The reference uses C99 `double complex`, `I`, `creal`,
 * `cimag`, `conj` and `cabs` inside C++ translation units (common_pspw.h:13,
 * 30-32), which C++ does not provide.  This header maps them onto GNU
 * `_Complex` so the reference compiles unmodified.
 */
#ifndef PSPW_ORACLE_COMPLEX_SHIM_H
#define PSPW_ORACLE_COMPLEX_SHIM_H

#include <math.h>

#define complex _Complex
#ifndef I
#define I (__extension__ 1.0i)
#endif

static inline double creal(double _Complex z) { return __real__ z; }
static inline double cimag(double _Complex z) { return __imag__ z; }
static inline double _Complex conj(double _Complex z) { return ~z; }
static inline double cabs(double _Complex z) { return hypot(__real__ z, __imag__ z); }

#endif
