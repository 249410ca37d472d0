/* Test infrastructure only: project-written stand-in for gsl_blas_zgemm
 * (C = alpha*op(A)*op(B) + beta*C), plain loops, k summed in ascending order
 * for each output element.  Only the NoTrans/NoTrans form the reference uses
 * is supported; any other form aborts. */
#ifndef ASKJA_SHIM_GSL_BLAS_H
#define ASKJA_SHIM_GSL_BLAS_H

#include "gsl_matrix.h"

enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;

static inline int gsl_blas_zgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB, const gsl_complex alpha,
                                 const gsl_matrix_complex* A, const gsl_matrix_complex* B, const gsl_complex beta,
                                 gsl_matrix_complex* C) {
  if (TransA != CblasNoTrans || TransB != CblasNoTrans || A->size2 != B->size1 || C->size1 != A->size1 ||
      C->size2 != B->size2) {
    fprintf(stderr, "gsl shim: unsupported zgemm form\n");
    abort();
  }
  const size_t M = A->size1, N = B->size2, K = A->size2;
  for (size_t i = 0; i < M; i++)
    for (size_t j = 0; j < N; j++) {
      double* c = C->data + 2 * (i * C->tda + j);
      double sr = c[0] * beta.dat[0] - c[1] * beta.dat[1];
      double si = c[0] * beta.dat[1] + c[1] * beta.dat[0];
      for (size_t k = 0; k < K; k++) {
        const double* a = A->data + 2 * (i * A->tda + k);
        const double* b = B->data + 2 * (k * B->tda + j);
        double ar = a[0] * alpha.dat[0] - a[1] * alpha.dat[1];
        double ai = a[0] * alpha.dat[1] + a[1] * alpha.dat[0];
        sr += ar * b[0] - ai * b[1];
        si += ar * b[1] + ai * b[0];
      }
      c[0] = sr;
      c[1] = si;
    }
  return 0;
}

#endif
