/* Test infrastructure only: project-written stand-in for the GSL complex FFT
 * calls that the reference's (never called) FourierTrafo makes.  A direct
 * O(n^2) inverse DFT: x_j = (1/n) sum_k z_k exp(+2 pi i j k / n). */
#ifndef ASKJA_SHIM_GSL_FFT_COMPLEX_H
#define ASKJA_SHIM_GSL_FFT_COMPLEX_H

#include <math.h>
#include <stdlib.h>

#include "gsl_complex_math.h"

typedef struct {
  size_t n;
} gsl_fft_complex_wavetable;
typedef struct {
  size_t n;
  double* scratch;
} gsl_fft_complex_workspace;

static inline gsl_fft_complex_wavetable* gsl_fft_complex_wavetable_alloc(size_t n) {
  gsl_fft_complex_wavetable* w = (gsl_fft_complex_wavetable*)malloc(sizeof(gsl_fft_complex_wavetable));
  w->n = n;
  return w;
}
static inline void gsl_fft_complex_wavetable_free(gsl_fft_complex_wavetable* w) { free(w); }
static inline gsl_fft_complex_workspace* gsl_fft_complex_workspace_alloc(size_t n) {
  gsl_fft_complex_workspace* w = (gsl_fft_complex_workspace*)malloc(sizeof(gsl_fft_complex_workspace));
  w->n = n;
  w->scratch = (double*)malloc(2 * n * sizeof(double));
  return w;
}
static inline void gsl_fft_complex_workspace_free(gsl_fft_complex_workspace* w) {
  if (!w) return;
  free(w->scratch);
  free(w);
}

static inline int gsl_fft_complex_inverse(gsl_complex_packed_array data, size_t stride, size_t n,
                                          const gsl_fft_complex_wavetable* wt, gsl_fft_complex_workspace* ws) {
  (void)wt;
  double* s = ws->scratch;
  for (size_t j = 0; j < n; j++) {
    double re = 0, im = 0;
    for (size_t k = 0; k < n; k++) {
      double ph = 2.0 * M_PI * (double)((j * k) % n) / (double)n;
      double zr = data[2 * stride * k], zi = data[2 * stride * k + 1];
      re += zr * cos(ph) - zi * sin(ph);
      im += zr * sin(ph) + zi * cos(ph);
    }
    s[2 * j] = re / (double)n;
    s[2 * j + 1] = im / (double)n;
  }
  for (size_t j = 0; j < n; j++) {
    data[2 * stride * j] = s[2 * j];
    data[2 * stride * j + 1] = s[2 * j + 1];
  }
  return 0;
}

#endif
