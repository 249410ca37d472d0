// Test infrastructure only (never part of the product path).
//
// Harness around the reference's own measurement routines: #includes the
// reference's measurements4d.cpp (found through -I at build time, never copied
// into this repository) with `main` renamed and exports:
//   PolyakovLoop        measurements4d.cpp:410-466
//   WilsonLoop(dir)     measurements4d.cpp:311-355
//   PlaqExp             measurements4d.cpp:885-927
//   scalarLoopcorr      measurements4d.cpp:357-408
// on a configuration injected in U-conf layout.
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include <algorithm>
#include <complex>
#include <fstream>
#include <random>
#include <vector>

#include <Eigen/Eigenvalues>
#include <gsl/gsl_blas.h>
#include <gsl/gsl_complex_math.h>
#include <gsl/gsl_fft_complex.h>
#include <gsl/gsl_matrix.h>

#define main askja_ref_measure_main
#include <measurements4d.cpp>
#undef main

#define EXPORT extern "C" __attribute__((visibility("default")))

static bool refm_ready = false;

EXPORT int refm_init(int nc, int dim, const int* n, double beta) {
  if (nc < 1 || dim < 1 || dim > 16) return -1;
  if (refm_ready) {
    free_memory();
    refm_ready = false;
  }
  NC = nc;
  DIM = dim;
  BETA = beta;
  struct coord g;
  g.d = dim;
  g.allocate();
  for (int i = 0; i < dim; i++) g.x[i] = n[i];
  xygrid.init(g);
  allocate_memory();
  refm_ready = true;
  return 0;
}

EXPORT int refm_set_u(const double* src) {
  if (!refm_ready) return -1;
  size_t nn = (size_t)NC * NC * 2;
  for (long i = 0; i < xygrid.SIZE; i++)
    for (int j = 0; j < DIM; j++) memcpy(u[i].M[j].M->data, src + ((size_t)i * DIM + j) * nn, nn * sizeof(double));
  return 0;
}

EXPORT double refm_PolyakovLoop() {
  std::vector<double> evs(NC + 1, 0.0);
  PolyakovLoop(evs.data());
  return evs[0];
}

EXPORT double refm_WilsonLoop(int dir) {
  std::vector<double> evs(NC + 1, 0.0);
  WilsonLoop(evs.data(), dir);
  return evs[0];
}

EXPORT void refm_PlaqExp(double* temporal, double* spatial) { PlaqExp(temporal, spatial); }

EXPORT void refm_scalarLoopcorr(double* out) { scalarLoopcorr(out); }
