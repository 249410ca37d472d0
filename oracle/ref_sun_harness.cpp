// Test infrastructure only (never part of the product path).
//
// Harness around the reference's own HMC routines: this translation unit
// #includes the reference's sun.cpp (found through -I at build time, never
// copied into this repository) with its `main` renamed and `time()` made
// deterministic, and exports a C ABI that injects U / pi / Pi in U-conf layout
// ([site][dir][row][col][re,im], doubles) and calls the reference's seam
// functions:
//   updateE              sun.cpp:672-723
//   updateUandcopyDown   sun.cpp:774-790
//   copyDown             sun.cpp:792-801
//   EnergyMag            sun.cpp:507-537
//   simpleenergyEl       sun.cpp:540-548
//   EnergyEl             sun.cpp:560-567
//   TotalEnergy          sun.cpp:571-576
//   GaussLaw             sun.cpp:415-438
//   UViol                sun.cpp:441-471
//   WilsonLoop           sun.cpp:307-362
//   generators           sun.cpp:142-189
//   mexpi / Adjoint      sunmat.h:200-248, 355-371
//   getplus / getminus   structs.h:169-218
//   Tab, FourierTrafo    sun.cpp:580-670, 365-411 (never called by the reference)
// GSL and Eigen are replaced by the project-written shim under oracle/shim.
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include <complex>
#include <fstream>
#include <random>
#include <vector>

#include <Eigen/Eigenvalues>
#include <gsl/gsl_blas.h>
#include <gsl/gsl_complex_math.h>
#include <gsl/gsl_fft_complex.h>
#include <gsl/gsl_matrix.h>
#include <gsl/gsl_randist.h>
#include <gsl/gsl_rng.h>

static unsigned long askja_ref_clock = 1000;
static time_t askja_ref_fake_time(time_t*) { return (time_t)(askja_ref_clock++); }

#define time(x) askja_ref_fake_time(x)
#define main askja_ref_main
#include <sun.cpp>
#undef main
#undef time

#define EXPORT extern "C" __attribute__((visibility("default")))

static sunfield* ref_field(int which) {
  switch (which) {
    case 0: return u;
    case 1: return U;
    case 2: return pi;
    case 3: return Pi;
    case 4: return uconf;
  }
  return nullptr;
}

static bool ref_ready = false;

EXPORT int ref_init(int nc, int dim, const int* n, double beta, int level) {
  if (nc < 1 || dim < 1 || dim > 16) return -1;
  if (ref_ready) {
    free_memory();
    delete[] gens;
    ref_ready = false;
  }
  NC = nc;
  DIM = dim;
  BETA = beta;
  LEVEL = level;
  VERBOSE = 0;
  struct coord g;
  g.d = dim;
  g.allocate();
  for (int i = 0; i < dim; i++) g.x[i] = n[i];
  xygrid.init(g);
  gens = new SUNmatrix[NC * NC - 1];
  for (int i = 0; i < NC * NC - 1; i++) gens[i].SUNmatrix_init(NC);
  generators(gens);
  allocate_memory();
  ref_ready = true;
  return 0;
}

EXPORT long ref_volume() { return xygrid.SIZE; }

EXPORT int ref_set_field(int which, const double* src) {
  sunfield* f = ref_field(which);
  if (!f || !ref_ready) return -1;
  size_t nn = (size_t)NC * NC * 2;
  for (long i = 0; i < xygrid.SIZE; i++)
    for (int j = 0; j < DIM; j++) memcpy(f[i].M[j].M->data, src + ((size_t)i * DIM + j) * nn, nn * sizeof(double));
  return 0;
}

EXPORT int ref_get_field(int which, double* dst) {
  sunfield* f = ref_field(which);
  if (!f || !ref_ready) return -1;
  size_t nn = (size_t)NC * NC * 2;
  for (long i = 0; i < xygrid.SIZE; i++)
    for (int j = 0; j < DIM; j++) memcpy(dst + ((size_t)i * DIM + j) * nn, f[i].M[j].M->data, nn * sizeof(double));
  return 0;
}

EXPORT void ref_set_threads(int n) { omp_set_num_threads(n); }
EXPORT void ref_updateE(double eps) { updateE(eps); }
EXPORT void ref_updateUandcopyDown(double eps) { updateUandcopyDown(eps); }
EXPORT void ref_copyDown() { copyDown(); }
EXPORT void ref_initializeU() { initializeU(); }
EXPORT void ref_initializeE(unsigned long seed) { initializeE(seed); }
EXPORT void ref_takeconfiguration() { takeconfiguration(); }
EXPORT void ref_loadconfiguration() { loadconfiguration(); }
EXPORT double ref_EnergyMag() { return EnergyMag(); }
EXPORT double ref_simpleenergyEl(int which) { return simpleenergyEl(ref_field(which)); }
EXPORT double ref_EnergyEl() { return EnergyEl(); }
EXPORT double ref_TotalEnergy() { return TotalEnergy(); }
EXPORT double ref_GaussLaw() { return GaussLaw(); }
EXPORT double ref_UViol() { return UViol(); }
EXPORT double ref_WilsonLoop() {
  std::vector<double> evs(NC + 1, 0.0);
  WilsonLoop(evs.data());
  return evs[0];
}
EXPORT long ref_getplus(long ind, int dir) { return xygrid.getplus(ind, dir); }
EXPORT long ref_getminus(long ind, int dir) { return xygrid.getminus(ind, dir); }

EXPORT void ref_generators(double* out) {
  size_t nn = (size_t)NC * NC * 2;
  for (int a = 0; a < NC * NC - 1; a++) memcpy(out + a * nn, gens[a].M->data, nn * sizeof(double));
}

EXPORT void ref_mexpi(const double* a, int level, double* out) {
  SUNmatrix m(NC);
  memcpy(m.M->data, a, (size_t)NC * NC * 2 * sizeof(double));
  SUNmatrix r(NC);
  r = mexpi(m, level);
  memcpy(out, r.M->data, (size_t)NC * NC * 2 * sizeof(double));
}

EXPORT void ref_Adjoint(const double* a, double* out) {
  SUNmatrix m(NC);
  memcpy(m.M->data, a, (size_t)NC * NC * 2 * sizeof(double));
  SUNmatrix r(NC);
  r = Adjoint(m);
  memcpy(out, r.M->data, (size_t)NC * NC * 2 * sizeof(double));
}

EXPORT void ref_Tab(long i, double* mdata, int npt) { Tab(i, mdata, npt); }
EXPORT void ref_FourierTrafo(double* coefficients) { FourierTrafo(coefficients); }
