/* Test infrastructure only: a project-written stand-in for the GNU GSL complex
 * API, written from GSL's public documentation (names and signatures only).
 * It exists so that the reference's own sun.cpp / sunmat.h / structs.h /
 * measurements4d.cpp compile unchanged into the oracle harness; GSL itself is
 * not installed in this image.  Only the handful of calls the reference makes
 * are provided. */
#ifndef ASKJA_SHIM_GSL_COMPLEX_MATH_H
#define ASKJA_SHIM_GSL_COMPLEX_MATH_H

#include <math.h>

typedef struct {
  double dat[2];
} gsl_complex;

typedef double* gsl_complex_packed_array;

#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
#define GSL_SET_COMPLEX(zp, x, y) \
  do {                            \
    (zp)->dat[0] = (x);           \
    (zp)->dat[1] = (y);           \
  } while (0)

static inline gsl_complex gsl_complex_rect(double x, double y) {
  gsl_complex z;
  z.dat[0] = x;
  z.dat[1] = y;
  return z;
}

static inline gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b) {
  return gsl_complex_rect(a.dat[0] + b.dat[0], a.dat[1] + b.dat[1]);
}

static inline gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b) {
  return gsl_complex_rect(a.dat[0] - b.dat[0], a.dat[1] - b.dat[1]);
}

static inline gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b) {
  return gsl_complex_rect(a.dat[0] * b.dat[0] - a.dat[1] * b.dat[1],
                          a.dat[0] * b.dat[1] + a.dat[1] * b.dat[0]);
}

static inline gsl_complex gsl_complex_conjugate(gsl_complex a) {
  return gsl_complex_rect(a.dat[0], -a.dat[1]);
}

static inline double gsl_complex_abs(gsl_complex a) { return hypot(a.dat[0], a.dat[1]); }

#endif
