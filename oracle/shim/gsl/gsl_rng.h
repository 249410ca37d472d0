/* Test infrastructure only: project-written stand-in for the GSL random number
 * API the reference calls (gsl_rng_env_setup / _alloc / _set / _uniform /
 * _free, gsl_rng_default).  The generator is the C++ standard library's
 * std::mt19937 seeded with the given seed; it is NOT bit-compatible with GSL's
 * mt19937 stream, so runs of the shim-built reference reproduce the
 * reference's algorithm but not its exact random numbers. */
#ifndef ASKJA_SHIM_GSL_RNG_H
#define ASKJA_SHIM_GSL_RNG_H

#include <random>
#include <stdint.h>

typedef struct {
  const char* name;
} gsl_rng_type;

typedef struct {
  const gsl_rng_type* type;
  std::mt19937* state;
} gsl_rng;

static const gsl_rng_type askja_shim_mt19937_type = {"mt19937 (std::mt19937 stand-in)"};
static const gsl_rng_type* gsl_rng_default = &askja_shim_mt19937_type;

static inline const gsl_rng_type* gsl_rng_env_setup(void) { return gsl_rng_default; }

static inline gsl_rng* gsl_rng_alloc(const gsl_rng_type* T) {
  gsl_rng* r = new gsl_rng;
  r->type = T;
  r->state = new std::mt19937(5489u);
  return r;
}

static inline void gsl_rng_set(const gsl_rng* r, unsigned long seed) {
  r->state->seed((uint32_t)(seed & 0xffffffffUL));
}

static inline void gsl_rng_free(gsl_rng* r) {
  if (!r) return;
  delete r->state;
  delete r;
}

/* uniform in [0,1) with 32 random bits */
static inline double gsl_rng_uniform(const gsl_rng* r) { return (double)(*r->state)() / 4294967296.0; }

/* uniform in (0,1) */
static inline double gsl_rng_uniform_pos(const gsl_rng* r) {
  double u;
  do {
    u = gsl_rng_uniform(r);
  } while (u == 0.0);
  return u;
}

#endif
