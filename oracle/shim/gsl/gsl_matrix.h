/* Test infrastructure only: project-written stand-in for the GSL complex
 * matrix API (public names/signatures from GSL's documentation).  Storage is
 * contiguous row-major (re,im) doubles with tda == size2, which is what the
 * reference's U-conf files contain when gsl_matrix_complex_fwrite writes a
 * freshly allocated matrix: size1*size2 complex numbers in native byte order. */
#ifndef ASKJA_SHIM_GSL_MATRIX_H
#define ASKJA_SHIM_GSL_MATRIX_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl_complex_math.h"

typedef struct {
  size_t size1;
  size_t size2;
  size_t tda;
  double* data;
  void* block;
  int owner;
} gsl_matrix_complex;

/* One allocation holds the header and the data, so the reference's many
 * temporaries cost one calloc/free each. */
static inline gsl_matrix_complex* gsl_matrix_complex_calloc(size_t n1, size_t n2) {
  size_t bytes = sizeof(gsl_matrix_complex) + 2 * n1 * n2 * sizeof(double);
  gsl_matrix_complex* m = (gsl_matrix_complex*)calloc(1, bytes);
  if (!m) return NULL;
  m->size1 = n1;
  m->size2 = n2;
  m->tda = n2;
  m->data = (double*)(m + 1);
  m->block = NULL;
  m->owner = 1;
  return m;
}

static inline gsl_matrix_complex* gsl_matrix_complex_alloc(size_t n1, size_t n2) {
  return gsl_matrix_complex_calloc(n1, n2);
}

static inline void gsl_matrix_complex_free(gsl_matrix_complex* m) { free(m); }

static inline gsl_complex gsl_matrix_complex_get(const gsl_matrix_complex* m, size_t i, size_t j) {
  const double* p = m->data + 2 * (i * m->tda + j);
  return gsl_complex_rect(p[0], p[1]);
}

static inline void gsl_matrix_complex_set(gsl_matrix_complex* m, size_t i, size_t j, gsl_complex z) {
  double* p = m->data + 2 * (i * m->tda + j);
  p[0] = z.dat[0];
  p[1] = z.dat[1];
}

static inline int gsl_matrix_complex_memcpy(gsl_matrix_complex* dest, const gsl_matrix_complex* src) {
  if (dest->size1 != src->size1 || dest->size2 != src->size2) {
    fprintf(stderr, "gsl shim: matrix size mismatch in memcpy\n");
    abort();
  }
  for (size_t i = 0; i < src->size1; i++)
    memcpy(dest->data + 2 * i * dest->tda, src->data + 2 * i * src->tda, 2 * src->size2 * sizeof(double));
  return 0;
}

static inline int gsl_matrix_complex_scale(gsl_matrix_complex* a, const gsl_complex x) {
  for (size_t i = 0; i < a->size1; i++)
    for (size_t j = 0; j < a->size2; j++) {
      double* p = a->data + 2 * (i * a->tda + j);
      double re = p[0] * x.dat[0] - p[1] * x.dat[1];
      double im = p[0] * x.dat[1] + p[1] * x.dat[0];
      p[0] = re;
      p[1] = im;
    }
  return 0;
}

static inline void gsl_matrix_complex_set_zero(gsl_matrix_complex* m) {
  for (size_t i = 0; i < m->size1; i++) memset(m->data + 2 * i * m->tda, 0, 2 * m->size2 * sizeof(double));
}

static inline void gsl_matrix_complex_set_identity(gsl_matrix_complex* m) {
  gsl_matrix_complex_set_zero(m);
  size_t n = m->size1 < m->size2 ? m->size1 : m->size2;
  for (size_t i = 0; i < n; i++) m->data[2 * (i * m->tda + i)] = 1.0;
}

static inline int gsl_matrix_complex_fwrite(FILE* stream, const gsl_matrix_complex* m) {
  for (size_t i = 0; i < m->size1; i++) {
    size_t w = fwrite(m->data + 2 * i * m->tda, sizeof(double), 2 * m->size2, stream);
    if (w != 2 * m->size2) return 1;
  }
  return 0;
}

static inline int gsl_matrix_complex_fread(FILE* stream, gsl_matrix_complex* m) {
  for (size_t i = 0; i < m->size1; i++) {
    size_t r = fread(m->data + 2 * i * m->tda, sizeof(double), 2 * m->size2, stream);
    if (r != 2 * m->size2) return 1;
  }
  return 0;
}

#endif
