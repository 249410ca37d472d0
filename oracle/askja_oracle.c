/*
 * askja oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, single-file restatement of the reference's HMC path
 * (paro8929/askja: sun.cpp, sunmat.h, structs.h, measurements4d.cpp).  Only
 * tests, the smoke check and the bench's CPU-baseline leg may load it, and
 * only as the checker; the product (askja_b200) never calls it.
 *
 * Parity of this restatement is pinned against the reference's own routines
 * compiled unchanged (oracle/Makefile -> oracle/_ref/libref_sun.so and
 * libref_measure4d.so, built against the project-written GSL shim) and against
 * the golden fixtures in tests/golden/ that those produced.
 *
 * Data layout everywhere is the reference's U-conf order: link (site, dir) at
 * offset (site*dim + dir)*nc*nc complex numbers, each matrix row-major, each
 * complex (re, im) as two doubles (sun.cpp:289-302 storeconf loop order).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

typedef struct {
  int nc, dim;
  long n[16];
  long stride[16]; /* helparr: structs.h:130-136, x0 slowest */
  long vol;
} geom_t;

static int geom_init(geom_t* g, int nc, int dim, const int* n) {
  if (nc < 1 || dim < 1 || dim > 16) return -1;
  g->nc = nc;
  g->dim = dim;
  g->vol = 1;
  for (int i = 0; i < dim; i++) {
    if (n[i] < 1) return -1;
    g->n[i] = n[i];
    g->vol *= n[i];
  }
  for (int i = 0; i < dim; i++) {
    g->stride[i] = 1;
    for (int j = i + 1; j < dim; j++) g->stride[i] *= n[j];
  }
  return 0;
}

/* structs.h:169-191 getplus / 194-218 getminus: decode one coordinate, step it
 * periodically, re-encode. */
static long coord_of(const geom_t* g, long ind, int dir) {
  if (dir == 0) return ind / g->stride[0];
  return (ind % g->stride[dir - 1]) / g->stride[dir];
}
static long getplus(const geom_t* g, long ind, int dir) {
  long c = coord_of(g, ind, dir);
  long nb = (c + 1) % g->n[dir];
  return ind + (nb - c) * g->stride[dir];
}
static long getminus(const geom_t* g, long ind, int dir) {
  long c = coord_of(g, ind, dir);
  long nb = (c - 1) % g->n[dir];
  if (nb < 0) nb += g->n[dir];
  return ind + (nb - c) * g->stride[dir];
}

EXPORT long or_getplus(int dim, const int* n, long ind, int dir) {
  geom_t g;
  if (geom_init(&g, 1, dim, n)) return -1;
  return getplus(&g, ind, dir);
}
EXPORT long or_getminus(int dim, const int* n, long ind, int dir) {
  geom_t g;
  if (geom_init(&g, 1, dim, n)) return -1;
  return getminus(&g, ind, dir);
}

/* ---- dense complex N x N helpers (sunmat.h semantics, row-major re/im) ---- */

#define MAXN 128

static inline const double* LNK(const geom_t* g, const double* f, long site, int dir) {
  return f + ((size_t)site * g->dim + dir) * (size_t)g->nc * g->nc * 2;
}
static inline double* LNKW(const geom_t* g, double* f, long site, int dir) {
  return f + ((size_t)site * g->dim + dir) * (size_t)g->nc * g->nc * 2;
}

/* c = a * b (zgemm NoTrans/NoTrans into a zeroed c, k ascending: sunmat.h:81-114) */
static void mm(int n, const double* a, const double* b, double* c) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double sr = 0, si = 0;
      for (int k = 0; k < n; k++) {
        const double* x = a + 2 * (i * n + k);
        const double* y = b + 2 * (k * n + j);
        sr += x[0] * y[0] - x[1] * y[1];
        si += x[0] * y[1] + x[1] * y[0];
      }
      c[2 * (i * n + j)] = sr;
      c[2 * (i * n + j) + 1] = si;
    }
}

/* conjugate transpose: sunmat.h:251-264 Hermitian */
static void dag(int n, const double* a, double* out) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      out[2 * (j * n + i)] = a[2 * (i * n + j)];
      out[2 * (j * n + i) + 1] = -a[2 * (i * n + j) + 1];
    }
}

static double trR(int n, const double* a) {
  double s = 0;
  for (int i = 0; i < n; i++) s += a[2 * (i * n + i)];
  return s;
}

/* sunmat.h:331-338 tr2(A) = Re Tr(A*A) */
static double tr2(int n, const double* a, double* tmp) {
  mm(n, a, a, tmp);
  return trR(n, tmp);
}

/* a*b*c^dag*d^dag with left-to-right products, as written in sun.cpp:712 */
static void prod4(int n, const double* a, const double* b, const double* c, int dagc, const double* d, int dagd,
                  double* out, double* t1, double* t2, double* t3) {
  mm(n, a, b, t1);
  const double* cc = c;
  if (dagc) {
    dag(n, c, t3);
    cc = t3;
  }
  mm(n, t1, cc, t2);
  const double* dd = d;
  if (dagd) {
    dag(n, d, t3);
    dd = t3;
  }
  mm(n, t2, dd, out);
}

/* sunmat.h:355-371 Adjoint(A) = -i/2 [ (A - A^dag) - Tr(A - A^dag)/n * 1 ] */
EXPORT void or_adjoint(int n, const double* a, double* out) {
  double trr = 0, tri = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double dr = a[2 * (i * n + j)] - a[2 * (j * n + i)];
      double di = a[2 * (i * n + j) + 1] + a[2 * (j * n + i) + 1];
      out[2 * (i * n + j)] = dr;
      out[2 * (i * n + j) + 1] = di;
      if (i == j) {
        trr += dr;
        tri += di;
      }
    }
  for (int i = 0; i < n; i++) {
    out[2 * (i * n + i)] -= trr / n;
    out[2 * (i * n + i) + 1] -= tri / n;
  }
  for (int k = 0; k < n * n; k++) {
    double re = out[2 * k] * 0.5, im = out[2 * k + 1] * 0.5;
    /* times (-i): (re + i im)(-i) = im - i re */
    out[2 * k] = im;
    out[2 * k + 1] = -re;
  }
}

/* sunmat.h:200-248 mexpi(A, L) = sum_{k<=L} (iA)^k/k!, Horner-nested
 * 1 + X(1 + X/2(1 + X/3(...(1 + X/L)))), X = iA; L outside 0..8 acts as 8. */
EXPORT void or_mexpi(int n, const double* a, int level, double* out) {
  int L = (level >= 0 && level <= 8) ? level : 8;
  double x[2 * MAXN * MAXN], t[2 * MAXN * MAXN], p[2 * MAXN * MAXN];
  for (int k = 0; k < n * n; k++) {
    x[2 * k] = -a[2 * k + 1];
    x[2 * k + 1] = a[2 * k];
  }
  memset(out, 0, sizeof(double) * 2 * n * n);
  for (int i = 0; i < n; i++) out[2 * (i * n + i)] = 1.0;
  if (L == 0) return;
  /* innermost: 1 + X/L */
  for (int k = 0; k < n * n; k++) {
    t[2 * k] = x[2 * k] * (1.0 / L);
    t[2 * k + 1] = x[2 * k + 1] * (1.0 / L);
  }
  for (int i = 0; i < n; i++) t[2 * (i * n + i)] += 1.0;
  for (int m = L - 1; m >= 1; m--) {
    double s[2 * MAXN * MAXN];
    for (int k = 0; k < n * n; k++) {
      s[2 * k] = x[2 * k] * (1.0 / m);
      s[2 * k + 1] = x[2 * k + 1] * (1.0 / m);
    }
    mm(n, s, t, p);
    for (int i = 0; i < n; i++) p[2 * (i * n + i)] += 1.0;
    memcpy(t, p, sizeof(double) * 2 * n * n);
  }
  memcpy(out, t, sizeof(double) * 2 * n * n);
}

/* sun.cpp:672-723 updateE: Pi = pi - eps * Adjoint(sum_{k!=j} upper + lower staples) */
EXPORT int or_updateE(int nc, int dim, const int* n, const double* u, const double* pi, double eps, double* Pi) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return -1;
  const int nn2 = 2 * nc * nc;
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < g.vol; i++) {
    double *st = malloc(sizeof(double) * nn2 * 7), *tmp = st + nn2, *t1 = st + 2 * nn2, *t2 = st + 3 * nn2,
           *t3 = st + 4 * nn2, *ad = st + 5 * nn2;
    for (int j = 0; j < dim; j++) {
      long njplus = getplus(&g, i, j);
      memset(st, 0, sizeof(double) * nn2);
      for (int k = 0; k < dim; k++) {
        if (k == j) continue;
        long nkplus = getplus(&g, i, k);
        long nkminus = getminus(&g, i, k);
        long njkminus = getminus(&g, njplus, k);
        prod4(nc, LNK(&g, u, i, j), LNK(&g, u, njplus, k), LNK(&g, u, nkplus, j), 1, LNK(&g, u, i, k), 1, tmp, t1,
              t2, t3);
        for (int e = 0; e < nn2; e++) st[e] += tmp[e];
        /* U_j(x) U_k^dag(x+j-k) U_j^dag(x-k) U_k(x-k) */
        dag(nc, LNK(&g, u, njkminus, k), t3);
        mm(nc, LNK(&g, u, i, j), t3, t1);
        dag(nc, LNK(&g, u, nkminus, j), t3);
        mm(nc, t1, t3, t2);
        mm(nc, t2, LNK(&g, u, nkminus, k), tmp);
        for (int e = 0; e < nn2; e++) st[e] += tmp[e];
      }
      or_adjoint(nc, st, ad);
      const double* p = LNK(&g, pi, i, j);
      double* q = LNKW(&g, Pi, i, j);
      for (int e = 0; e < nn2; e++) q[e] = p[e] - ad[e] * eps;
    }
    free(st);
  }
  return 0;
}

/* sun.cpp:774-790 updateUandcopyDown: U = mexpi(eps*Pi, L) * u; u = U (pi = Pi is the caller's) */
EXPORT int or_updateU(int nc, int dim, const int* n, const double* u, const double* Pi, double eps, int level,
                      double* uout) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return -1;
  const int nn2 = 2 * nc * nc;
  const long nl = g.vol * dim;
#pragma omp parallel for schedule(dynamic, 64)
  for (long l = 0; l < nl; l++) {
    double a[2 * MAXN * MAXN], e[2 * MAXN * MAXN], r[2 * MAXN * MAXN];
    const double* p = Pi + (size_t)l * nn2;
    for (int k = 0; k < nn2; k++) a[k] = p[k] * eps;
    or_mexpi(nc, a, level, e);
    mm(nc, e, u + (size_t)l * nn2, r);
    memcpy(uout + (size_t)l * nn2, r, sizeof(double) * nn2);
  }
  return 0;
}

static void plaq(const geom_t* g, const double* u, long i, int j, int k, double* out, double* t1, double* t2,
                 double* t3) {
  long njplus = getplus(g, i, j);
  long nkplus = getplus(g, i, k);
  prod4(g->nc, LNK(g, u, i, j), LNK(g, u, njplus, k), LNK(g, u, nkplus, j), 1, LNK(g, u, i, k), 1, out, t1, t2, t3);
}

/* sun.cpp:507-537 EnergyMag = sum_x sum_{j<k} (1 - ReTr P_jk(x)/NC) */
EXPORT double or_EnergyMag(int nc, int dim, const int* n, const double* u) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return NAN;
  double res = 0;
  double *buf = malloc(sizeof(double) * 2 * nc * nc * 4), *p = buf, *t1 = buf + 2 * nc * nc,
         *t2 = buf + 4 * nc * nc, *t3 = buf + 6 * nc * nc;
  for (long i = 0; i < g.vol; i++)
    for (int j = 0; j < dim; j++)
      for (int k = j + 1; k < dim; k++) {
        plaq(&g, u, i, j, k, p, t1, t2, t3);
        res += 1 - trR(nc, p) / nc;
      }
  free(buf);
  return res;
}

/* measurements4d.cpp:885-927 PlaqExp: temporal = planes (0,k), spatial = planes (j,k), 1<=j<k */
EXPORT int or_PlaqExp(int nc, int dim, const int* n, const double* u, double* temporal, double* spatial) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return -1;
  double t = 0, s = 0;
  double *buf = malloc(sizeof(double) * 2 * nc * nc * 4), *p = buf, *t1 = buf + 2 * nc * nc,
         *t2 = buf + 4 * nc * nc, *t3 = buf + 6 * nc * nc;
  for (long i = 0; i < g.vol; i++) {
    for (int j = 1; j < dim; j++)
      for (int k = j + 1; k < dim; k++) {
        plaq(&g, u, i, j, k, p, t1, t2, t3);
        s += 1 - trR(nc, p) / nc;
      }
    for (int k = 1; k < dim; k++) {
      plaq(&g, u, i, 0, k, p, t1, t2, t3);
      t += 1 - trR(nc, p) / nc;
    }
  }
  free(buf);
  *temporal = t;
  *spatial = s;
  return 0;
}

/* sun.cpp:540-548 simpleenergyEl(p) = sum tr2(p) */
EXPORT double or_simpleenergyEl(int nc, int dim, const int* n, const double* p) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return NAN;
  double res = 0;
  double* tmp = malloc(sizeof(double) * 2 * nc * nc);
  for (long l = 0; l < g.vol * dim; l++) res += tr2(nc, p + (size_t)l * 2 * nc * nc, tmp);
  free(tmp);
  return res;
}

/* sun.cpp:560-567 EnergyEl = sum 1/4 tr2(pi + Pi) */
EXPORT double or_EnergyEl(int nc, int dim, const int* n, const double* pi, const double* Pi) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return NAN;
  double res = 0;
  const int nn2 = 2 * nc * nc;
  double *s = malloc(sizeof(double) * nn2 * 2), *tmp = s + nn2;
  for (long l = 0; l < g.vol * dim; l++) {
    for (int e = 0; e < nn2; e++) s[e] = pi[(size_t)l * nn2 + e] + Pi[(size_t)l * nn2 + e];
    res += 0.25 * tr2(nc, s, tmp);
  }
  free(s);
  return res;
}

/* sun.cpp:415-438 GaussLaw = tr2( sum_x sum_j [Pi_j(x) - U_j^dag(x-j) Pi_j(x-j) U_j(x-j)] ) */
EXPORT double or_GaussLaw(int nc, int dim, const int* n, const double* u, const double* Pi) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return NAN;
  const int nn2 = 2 * nc * nc;
  double *acc = calloc(nn2 * 4, sizeof(double)), *t1 = acc + nn2, *t2 = acc + 2 * nn2, *t3 = acc + 3 * nn2;
  for (long i = 0; i < g.vol; i++)
    for (int j = 0; j < dim; j++) {
      long m = getminus(&g, i, j);
      dag(nc, LNK(&g, u, m, j), t3);
      mm(nc, t3, LNK(&g, Pi, m, j), t1);
      mm(nc, t1, LNK(&g, u, m, j), t2);
      const double* p = LNK(&g, Pi, i, j);
      for (int e = 0; e < nn2; e++) acc[e] = (acc[e] + p[e]) - t2[e];
    }
  double r = tr2(nc, acc, t1);
  free(acc);
  return r;
}

/* sun.cpp:441-471 UViol = sum tr2(U U^dag - 1) */
EXPORT double or_UViol(int nc, int dim, const int* n, const double* u) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return NAN;
  const int nn2 = 2 * nc * nc;
  double *t1 = malloc(sizeof(double) * nn2 * 3), *t2 = t1 + nn2, *t3 = t1 + 2 * nn2;
  double res = 0;
  for (long l = 0; l < g.vol * dim; l++) {
    dag(nc, u + (size_t)l * nn2, t3);
    mm(nc, u + (size_t)l * nn2, t3, t1);
    for (int i = 0; i < nc; i++) t1[2 * (i * nc + i)] -= 1.0;
    res += tr2(nc, t1, t2);
  }
  free(t1);
  return res;
}

/* ordered product of the links along `dir` starting at `start`, closing the
 * periodic line after n[dir] links; returns |Tr W| / NC */
static double line_trace(const geom_t* g, const double* u, long start, int dir, double* w, double* t) {
  const int nc = g->nc, nn2 = 2 * nc * nc;
  long pos = start;
  memcpy(w, LNK(g, u, pos, dir), sizeof(double) * nn2);
  for (long s = 0; s < g->n[dir] - 1; s++) {
    pos = getplus(g, pos, dir);
    mm(nc, w, LNK(g, u, pos, dir), t);
    memcpy(w, t, sizeof(double) * nn2);
  }
  double tr = 0, ti = 0;
  for (int i = 0; i < nc; i++) {
    tr += w[2 * (i * nc + i)];
    ti += w[2 * (i * nc + i) + 1];
  }
  return hypot(tr, ti) / nc;
}

/* sun.cpp:307-362 WilsonLoop: line along dir 0 from site 0 */
EXPORT double or_WilsonLoop_sun(int nc, int dim, const int* n, const double* u) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return NAN;
  double* w = malloc(sizeof(double) * 4 * nc * nc);
  double r = line_trace(&g, u, 0, 0, w, w + 2 * nc * nc);
  free(w);
  return r;
}

/* measurements4d.cpp:410-466 PolyakovLoop: mean over x1 of the closed line in
 * dir 0 through (0, x1, 0, ...).  (The reference starts each line after the
 * first at x0 = N0-1; the trace of a closed periodic line is the same.) */
EXPORT double or_PolyakovLoop(int nc, int dim, const int* n, const double* u) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN || dim < 2) return NAN;
  double* w = malloc(sizeof(double) * 4 * nc * nc);
  double s = 0;
  for (long x1 = 0; x1 < g.n[1]; x1++) s += line_trace(&g, u, x1 * g.stride[1], 0, w, w + 2 * nc * nc);
  free(w);
  return s / g.n[1];
}

/* measurements4d.cpp:311-355 WilsonLoop(dir): mean over x0 of the closed line in
 * dir `dir` (>=1) through (x0, 0, ..., 0). */
EXPORT double or_WilsonLoopDir(int nc, int dim, const int* n, const double* u, int dir) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN || dir < 1 || dir >= dim) return NAN;
  double* w = malloc(sizeof(double) * 4 * nc * nc);
  double s = 0;
  for (long x0 = 0; x0 < g.n[0]; x0++) s += line_trace(&g, u, x0 * g.stride[0], dir, w, w + 2 * nc * nc);
  free(w);
  return s / g.n[0];
}

/* measurements4d.cpp:357-408 scalarLoopcorr: per x0 slice, mean of ReTr U_{D-1}/NC */
EXPORT int or_scalarLoopcorr(int nc, int dim, const int* n, const double* u, double* out) {
  geom_t g;
  if (geom_init(&g, nc, dim, n) || nc > MAXN) return -1;
  long slice = g.stride[0];
  for (long x0 = 0; x0 < g.n[0]; x0++) {
    double s = 0;
    for (long sl = x0 * slice; sl < (x0 + 1) * slice; sl++) s += trR(nc, LNK(&g, u, sl, dim - 1)) / nc;
    out[x0] = s / slice;
  }
  return 0;
}

/* sun.cpp:142-189 generators: off-diagonal (sym, antisym) pairs for i<j, then
 * diagonal ones, normalised to Tr(T_a T_a) = 1/2.  out: (nc^2-1) matrices. */
EXPORT void or_generators(int nc, double* out) {
  const int nn2 = 2 * nc * nc;
  memset(out, 0, sizeof(double) * nn2 * (nc * nc - 1));
  int num = 0;
  for (int i = 0; i < nc; i++)
    for (int j = i + 1; j < nc; j++) {
      double* a = out + (size_t)num * nn2;
      double* b = out + (size_t)(num + 1) * nn2;
      a[2 * (i * nc + j)] = 0.5;
      a[2 * (j * nc + i)] = 0.5;
      b[2 * (i * nc + j) + 1] = -0.5;
      b[2 * (j * nc + i) + 1] = 0.5;
      num += 2;
    }
  for (int m = 0; m < nc - 1; m++) {
    double* a = out + (size_t)num * nn2;
    double norm = sqrt(0.5 / ((double)(m + 1) * (m + 2)));
    for (int j = 0; j <= m; j++) a[2 * (j * nc + j)] = norm;
    a[2 * ((m + 1) * nc + m + 1)] = -(m + 1) * norm;
    num++;
  }
}

/* sun.cpp:230-247: P = sqrt(2 NC / beta) * sum_a xi_a T_a for each link;
 * xi holds (nc^2-1) normals per link in link order. */
EXPORT int or_momenta_from_normals(int nc, long nlinks, double beta, const double* xi, double* p) {
  const int na = nc * nc - 1, nn2 = 2 * nc * nc;
  double* gens = malloc(sizeof(double) * nn2 * na);
  or_generators(nc, gens);
  double s = sqrt(2.0 * nc / beta);
  for (long l = 0; l < nlinks; l++) {
    double* q = p + (size_t)l * nn2;
    memset(q, 0, sizeof(double) * nn2);
    for (int a = 0; a < na; a++) {
      double x = xi[(size_t)l * na + a];
      for (int e = 0; e < nn2; e++) q[e] += gens[(size_t)a * nn2 + e] * x;
    }
    for (int e = 0; e < nn2; e++) q[e] *= s;
  }
  free(gens);
  return 0;
}

/* ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ---- */
static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

EXPORT void or_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Momentum-refresh normals of the GPU engine: for link l (U-conf order
 * l = site*dim + dir) and generator a, block j = a/4 of Philox with
 * counter (j, l_lo, l_hi, traj) and key (seed_lo, seed_hi); the four 32-bit
 * words become uniforms u = (w + 0.5) * 2^-32 and two Box-Muller pairs
 * (u0,u1) -> (r cos 2pi u1, r sin 2pi u1), r = sqrt(-2 ln u0), likewise (u2,u3). */
EXPORT void or_engine_normals(int nc, long nlinks, uint64_t seed, uint64_t traj, double* xi) {
  const int na = nc * nc - 1;
  const int nblk = (na + 3) / 4;
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (long l = 0; l < nlinks; l++)
    for (int j = 0; j < nblk; j++) {
      uint32_t ctr[4] = {(uint32_t)j, (uint32_t)l, (uint32_t)((uint64_t)l >> 32), (uint32_t)traj}, w[4];
      or_philox4x32_10(ctr, key, w);
      double u[4];
      for (int q = 0; q < 4; q++) u[q] = ((double)w[q] + 0.5) * (1.0 / 4294967296.0);
      double g4[4];
      double r0 = sqrt(-2.0 * log(u[0])), r1 = sqrt(-2.0 * log(u[2]));
      g4[0] = r0 * cos(2.0 * M_PI * u[1]);
      g4[1] = r0 * sin(2.0 * M_PI * u[1]);
      g4[2] = r1 * cos(2.0 * M_PI * u[3]);
      g4[3] = r1 * sin(2.0 * M_PI * u[3]);
      for (int q = 0; q < 4; q++) {
        int a = 4 * j + q;
        if (a < na) xi[(size_t)l * na + a] = g4[q];
      }
    }
}

/* Reunitarisation used by the FP32 path: Gram-Schmidt orthonormalisation of
 * the rows (modified, in row order), then the last row multiplied by
 * conj(det)/|det| so that det = 1.  (Not in the reference, which never
 * reunitarises.) */
static void cdet(int n, const double* a, double* dr, double* di) {
  double m[2 * MAXN * MAXN];
  memcpy(m, a, sizeof(double) * 2 * n * n);
  double rr = 1, ri = 0;
  for (int c = 0; c < n; c++) {
    int piv = c;
    double best = -1;
    for (int r = c; r < n; r++) {
      double v = hypot(m[2 * (r * n + c)], m[2 * (r * n + c) + 1]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (piv != c) {
      for (int k = 0; k < n; k++) {
        double t0 = m[2 * (c * n + k)], t1 = m[2 * (c * n + k) + 1];
        m[2 * (c * n + k)] = m[2 * (piv * n + k)];
        m[2 * (c * n + k) + 1] = m[2 * (piv * n + k) + 1];
        m[2 * (piv * n + k)] = t0;
        m[2 * (piv * n + k) + 1] = t1;
      }
      rr = -rr;
      ri = -ri;
    }
    double pr = m[2 * (c * n + c)], pi_ = m[2 * (c * n + c) + 1];
    double nr = rr * pr - ri * pi_, ni = rr * pi_ + ri * pr;
    rr = nr;
    ri = ni;
    double den = pr * pr + pi_ * pi_;
    if (den == 0) {
      *dr = 0;
      *di = 0;
      return;
    }
    for (int r = c + 1; r < n; r++) {
      double ar = m[2 * (r * n + c)], ai = m[2 * (r * n + c) + 1];
      double fr = (ar * pr + ai * pi_) / den, fi = (ai * pr - ar * pi_) / den;
      for (int k = c; k < n; k++) {
        double br = m[2 * (c * n + k)], bi = m[2 * (c * n + k) + 1];
        m[2 * (r * n + k)] -= fr * br - fi * bi;
        m[2 * (r * n + k) + 1] -= fr * bi + fi * br;
      }
    }
  }
  *dr = rr;
  *di = ri;
}

EXPORT void or_reunitarise(int n, double* a) {
  for (int r = 0; r < n; r++) {
    double* row = a + 2 * r * n;
    for (int q = 0; q < r; q++) {
      const double* pr = a + 2 * q * n;
      double sr = 0, si = 0; /* <pr, row> = sum conj(pr) row */
      for (int k = 0; k < n; k++) {
        sr += pr[2 * k] * row[2 * k] + pr[2 * k + 1] * row[2 * k + 1];
        si += pr[2 * k] * row[2 * k + 1] - pr[2 * k + 1] * row[2 * k];
      }
      for (int k = 0; k < n; k++) {
        row[2 * k] -= sr * pr[2 * k] - si * pr[2 * k + 1];
        row[2 * k + 1] -= sr * pr[2 * k + 1] + si * pr[2 * k];
      }
    }
    double nrm = 0;
    for (int k = 0; k < n; k++) nrm += row[2 * k] * row[2 * k] + row[2 * k + 1] * row[2 * k + 1];
    nrm = 1.0 / sqrt(nrm);
    for (int k = 0; k < 2 * n; k++) row[k] *= nrm;
  }
  double dr, di;
  cdet(n, a, &dr, &di);
  double dn = hypot(dr, di);
  double cr = dr / dn, ci = -di / dn; /* conj(det)/|det| */
  double* row = a + 2 * (n - 1) * n;
  for (int k = 0; k < n; k++) {
    double xr = row[2 * k], xi = row[2 * k + 1];
    row[2 * k] = xr * cr - xi * ci;
    row[2 * k + 1] = xr * ci + xi * cr;
  }
}

EXPORT void or_det(int n, const double* a, double* out2) { cdet(n, a, &out2[0], &out2[1]); }
