/* Test infrastructure only: project-written stand-in for gsl_ran_gaussian.
 * Gaussian deviates by the Box-Muller transform of two uniforms from the
 * stand-in generator (not GSL's own sampling method). */
#ifndef ASKJA_SHIM_GSL_RANDIST_H
#define ASKJA_SHIM_GSL_RANDIST_H

#include <math.h>

#include "gsl_rng.h"

static inline double gsl_ran_gaussian(const gsl_rng* r, const double sigma) {
  double u1 = gsl_rng_uniform_pos(r);
  double u2 = gsl_rng_uniform(r);
  return sigma * sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

#endif
