// Residual-plane FP32 mode (NC <= 4, thread per link): FP32 arithmetic on
// FP32 fields that each carry a bfloat16 residual plane.
//
// Why.  In an FP32-only HMC the energy difference dH of a trajectory differs
// from the FP64 one by the storage rounding of every link and momentum at
// every MD step: an unbiased random walk, ~1e-4 per trajectory on SU(3) 8^4
// and ~16x that on 32^4 (it grows as sqrt(links)), plus a systematic part from
// the per-update FP32 projection onto SU(N).  Carrying each stored value as
// hi + lo (hi the FP32 value, lo its residual in bfloat16) gives ~32
// significant bits at 1.5x the bytes of the links and 2/3 of the bytes of
// full FP32 momentum matrices, while every product, the staple sum, the force
// and the exponential stay in FP32 from hi alone.
//
// What changes against the FP32-only kernels (small.cuh):
//  * links: hi = the usual float2 field, lo = one uint32 per complex element
//    (bfloat16 residual of re in the low half, of im in the high half), same
//    blocked index as hi;
//  * momenta: the N^2-1 real coordinates of the Hermitian traceless matrix
//    instead of N^2 complex entries -- k = 2p, 2p+1: Re, Im of the p-th upper
//    off-diagonal entry (i < j, row-major), k = N(N-1) + m: the diagonal entry
//    m < N-1 (the last one is minus their sum, so P stays traceless exactly);
//    hi floats at ((d*B + s/32)*NCOEF + k)*32 + s%32 and lo bfloat16 pairs
//    (coordinates 2w, 2w+1 in word w) at ((d*B + s/32)*NLOW + w)*32 + s%32;
//  * the kick and the link update are accumulated into (hi, lo) exactly
//    (TwoSum, then a renormalising Fast2Sum): P += -eps F, U += (E - 1) U with
//    E - 1 formed directly (never as E minus the identity);
//  * no per-update projection: links are projected onto SU(N) in FP64 from
//    hi + lo once per trajectory (k_reunit), which keeps the norms exact to
//    ~1e-10 instead of scattering them by the FP32 rounding of a projection;
//  * every reduction (action, kinetic energy) reads hi + lo in FP64.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "misc.cuh"
#include "small.cuh"

namespace askja {
namespace split {

template <int N>
struct Dims {
  static constexpr int NCOEF = N * N - 1;        // real coordinates of a momentum
  static constexpr int NLOW = (NCOEF + 1) / 2;   // residual words of a momentum
  static constexpr int NDIAG = N * (N - 1);      // index of the first diagonal coordinate
};

// ---- residuals -------------------------------------------------------------
__device__ __forceinline__ float lo_low(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float lo_high(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ uint32_t lo_pack(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);  // a -> low half, b -> high half
  uint32_t w;
  memcpy(&w, &v, sizeof w);
  return w;
}

// (hi, lo) <- (hi, lo) + d.  TwoSum gives s + e = hi + d exactly; the residual
// r = lo + e is folded back by Fast2Sum so that |lo| stays within half an ulp
// of hi (exact for |s| >= |r|; where an element crosses zero and |r| > |s| the
// split is off by an ulp of r, far below the bfloat16 resolution of lo).
// Intrinsics keep the compiler from contracting or reassociating the sums.
__device__ __forceinline__ void add_split(float& hi, float& lo, float d) {
  const float s = __fadd_rn(hi, d);
  const float bb = __fsub_rn(s, hi);
  const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(d, bb));
  const float r = __fadd_rn(lo, e);
  const float h2 = __fadd_rn(s, r);
  lo = __fsub_rn(r, __fsub_rn(h2, s));
  hi = h2;
}

// add_split on two values at once in packed FP32x2 (FADD2 of sm_100): the
// same operations lane by lane, half the instructions.  p - q is formed as
// fma(q, -1, p) (exact negation, one rounding), the packed instructions having
// no negated operand.
__device__ __forceinline__ float2 sub2_rn(float2 p, float2 q) { return __ffma2_rn(q, make_float2(-1.f, -1.f), p); }

__device__ __forceinline__ void add_split2(float& hi0, float& hi1, float& lo0, float& lo1, float d0, float d1) {
  const float2 hi = make_float2(hi0, hi1), lo = make_float2(lo0, lo1), d = make_float2(d0, d1);
  const float2 s = __fadd2_rn(hi, d);
  const float2 bb = sub2_rn(s, hi);
  const float2 e = __fadd2_rn(sub2_rn(hi, sub2_rn(s, bb)), sub2_rn(d, bb));
  const float2 r = __fadd2_rn(lo, e);
  const float2 h2 = __fadd2_rn(s, r);
  const float2 l2 = sub2_rn(r, sub2_rn(h2, s));
  hi0 = h2.x;
  hi1 = h2.y;
  lo0 = l2.x;
  lo1 = l2.y;
}

// FP64 value -> (hi, lo)
__device__ __forceinline__ void split_of(double v, float& hi, float& lo) {
  hi = __double2float_rn(v);
  lo = __double2float_rn(v - (double)hi);
}

// ---- indexing ----------------------------------------------------------------
template <int N>
__host__ __device__ __forceinline__ size_t cbase(const Lat& L, int d, int s) {
  return ((size_t)d * L.B + (s >> 5)) * (size_t)Dims<N>::NCOEF * 32 + (s & 31);
}
template <int N>
__host__ __device__ __forceinline__ size_t lbase(const Lat& L, int d, int s) {
  return ((size_t)d * L.B + (s >> 5)) * (size_t)Dims<N>::NLOW * 32 + (s & 31);
}

// hi floats / lo words of a momentum field (padding included)
template <int N>
__host__ __device__ __forceinline__ size_t coef_floats(const Lat& L) {
  return (size_t)L.D * L.B * 32 * Dims<N>::NCOEF;
}
template <int N>
__host__ __device__ __forceinline__ size_t coef_words(const Lat& L) {
  return (size_t)L.D * L.B * 32 * Dims<N>::NLOW;
}

// ---- momenta -------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void load_coefs(float (&h)[Dims<N>::NCOEF], float (&l)[Dims<N>::NCOEF],
                                           const float* __restrict__ P, const uint32_t* __restrict__ PL,
                                           const Lat& L, int d, int s) {
  const float* ph = P + cbase<N>(L, d, s);
  const uint32_t* pl = PL + lbase<N>(L, d, s);
#pragma unroll
  for (int k = 0; k < Dims<N>::NCOEF; k++) h[k] = ph[k * 32];
#pragma unroll
  for (int w = 0; w < Dims<N>::NLOW; w++) {
    const uint32_t x = pl[w * 32];
    l[2 * w] = lo_low(x);
    if (2 * w + 1 < Dims<N>::NCOEF) l[2 * w + 1] = lo_high(x);
  }
}

template <int N>
__device__ __forceinline__ void store_coefs(float* __restrict__ P, uint32_t* __restrict__ PL,
                                            const float (&h)[Dims<N>::NCOEF], const float (&l)[Dims<N>::NCOEF],
                                            const Lat& L, int d, int s) {
  float* ph = P + cbase<N>(L, d, s);
  uint32_t* pl = PL + lbase<N>(L, d, s);
#pragma unroll
  for (int k = 0; k < Dims<N>::NCOEF; k++) ph[k * 32] = h[k];
#pragma unroll
  for (int w = 0; w < Dims<N>::NLOW; w++)
    pl[w * 32] = lo_pack(l[2 * w], 2 * w + 1 < Dims<N>::NCOEF ? l[2 * w + 1] : 0.f);
}

// Hermitian traceless matrix of coordinates c (any real type)
template <int N, typename T, typename C>
__device__ __forceinline__ void coefs_to_mat(small::Mat<N, T>& P, const C (&c)[Dims<N>::NCOEF]) {
  int p = 0;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i + 1; j < N; j++, p++) {
      P.a[i][j] = mkc<T>((T)c[2 * p], (T)c[2 * p + 1]);
      P.a[j][i] = mkc<T>((T)c[2 * p], -(T)c[2 * p + 1]);
    }
  T last = T(0);
#pragma unroll
  for (int m = 0; m < N - 1; m++) {
    P.a[m][m] = mkc<T>((T)c[Dims<N>::NDIAG + m], T(0));
    last -= (T)c[Dims<N>::NDIAG + m];
  }
  P.a[N - 1][N - 1] = mkc<T>(last, T(0));
}

// tr(P^2) of coordinates c: sum of the squared diagonal + 2 |upper entries|^2
template <int N>
__device__ __forceinline__ double coef_tr2(const double (&c)[Dims<N>::NCOEF]) {
  double off = 0.0, diag = 0.0, last = 0.0;
#pragma unroll
  for (int k = 0; k < Dims<N>::NDIAG; k++) off = fma(c[k], c[k], off);
#pragma unroll
  for (int m = 0; m < N - 1; m++) {
    diag = fma(c[Dims<N>::NDIAG + m], c[Dims<N>::NDIAG + m], diag);
    last -= c[Dims<N>::NDIAG + m];
  }
  return fma(last, last, diag) + 2.0 * off;
}

// Coordinates of the force F = Adjoint(W) written as the Hermitian matrix the
// kick subtracts (P <- P - eps F, as small::kick_ta):
//   F_ij = ((Im W_ij + Im W_ji) - i (Re W_ij - Re W_ji)) / 2,  F_ii = Im W_ii - Im tr W / N.
template <int N>
__device__ __forceinline__ void force_coefs(float (&f)[Dims<N>::NCOEF], const small::Mat<N, float>& W) {
  int p = 0;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i + 1; j < N; j++, p++) {
      f[2 * p] = 0.5f * (W.a[i][j].im + W.a[j][i].im);
      f[2 * p + 1] = -0.5f * (W.a[i][j].re - W.a[j][i].re);
    }
  // The trace is taken out in FP64.  Only the first N-1 diagonal entries are
  // kept (the last is minus their sum), so the last one's force is implied
  // as -(F_00 + ... ); an FP32 trace times fl(1/N) would give every link the
  // same relative error in that implied entry, an error along the diagonal
  // generator that correlates with the momentum and drifts the energy.
  double tr = 0.0;
#pragma unroll
  for (int k = 0; k < N; k++) tr += (double)W.a[k][k].im;
  tr /= N;
#pragma unroll
  for (int m = 0; m < N - 1; m++) f[Dims<N>::NDIAG + m] = (float)((double)W.a[m][m].im - tr);
}

// ---- links -----------------------------------------------------------------
template <int N>
__device__ __forceinline__ void load_lo(small::Mat<N, float>& M, const uint32_t* __restrict__ UL, const Lat& L, int d,
                                        int s) {
  const uint32_t* p = UL + mbase(L, d, s);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      const uint32_t w = p[(i * N + j) * 32];
      M.a[i][j] = mkc<float>(lo_low(w), lo_high(w));
    }
}

template <int N>
__device__ __forceinline__ void store_lo(uint32_t* __restrict__ UL, const small::Mat<N, float>& M, const Lat& L,
                                         int d, int s) {
  uint32_t* p = UL + mbase(L, d, s);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) p[(i * N + j) * 32] = lo_pack(M.a[i][j].re, M.a[i][j].im);
}

// link (d, s) as hi + lo in FP64
template <int N>
__device__ __forceinline__ void load_exact(small::Mat<N, double>& M, const float2* __restrict__ U,
                                           const uint32_t* __restrict__ UL, const Lat& L, int d, int s) {
  const size_t b = mbase(L, d, s);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      const float2 h = U[b + (i * N + j) * 32];
      const uint32_t w = UL[b + (i * N + j) * 32];
      M.a[i][j] = mkc<double>((double)h.x + (double)lo_low(w), (double)h.y + (double)lo_high(w));
    }
}

// row i of link (d, s) as hi + lo in FP64
template <int N>
__device__ __forceinline__ void load_exact_row(cpx<double> (&r)[N], const float2* __restrict__ U,
                                               const uint32_t* __restrict__ UL, const Lat& L, int d, int s, int i) {
  const size_t b = mbase(L, d, s) + (size_t)i * N * 32;
#pragma unroll
  for (int j = 0; j < N; j++) {
    const float2 h = U[b + j * 32];
    const uint32_t w = UL[b + j * 32];
    r[j] = mkc<double>((double)h.x + (double)lo_low(w), (double)h.y + (double)lo_high(w));
  }
}

template <int N>
__device__ __forceinline__ void store_exact(float2* __restrict__ U, uint32_t* __restrict__ UL,
                                            const small::Mat<N, double>& M, const Lat& L, int d, int s) {
  const size_t b = mbase(L, d, s);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      float hr, lr, hi, li;
      split_of(M.a[i][j].re, hr, lr);
      split_of(M.a[i][j].im, hi, li);
      U[b + (i * N + j) * 32] = make_float2(hr, hi);
      UL[b + (i * N + j) * 32] = lo_pack(lr, li);
    }
}

// ---- E - 1 = exp(i eps P) - 1 to Taylor order `order` --------------------------
// N = 3: the Cayley-Hamilton series in Hermitian P of small::expi_times_herm3
// (E - 1 = A + B P + C P^2 with A, B, C from a real three-term recursion);
// N = 2: X^2 = tr X X - det X 1 (small::expi_times_ch without the X^0 term);
// N = 4: Horner, X (1 + X/2 (1 + X/3 (...))).  All in FP32 from hi.
template <int N>
__device__ __forceinline__ void exp_minus_one(small::Mat<N, float>& E, const small::Mat<N, float>& P, float eps,
                                              int order) {
  using small::Mat;
  if constexpr (N == 3) {
    const float p0 = P.a[0][0].re, p1 = P.a[1][1].re, p2 = P.a[2][2].re;
    const cpx<float>& P01 = P.a[0][1];
    const cpx<float>& P02 = P.a[0][2];
    const cpx<float>& P12 = P.a[1][2];
    const float n01 = cnorm2_add(P01, 0.f), n02 = cnorm2_add(P02, 0.f), n12 = cnorm2_add(P12, 0.f);
    const float q0 = fmaf(p0, p0, n01 + n02), q1 = fmaf(p1, p1, n01 + n12), q2 = fmaf(p2, p2, n02 + n12);
    const float s01 = p0 + p1, s02 = p0 + p2, s12 = p1 + p2;
    cpx<float> Q01 = mkc<float>(s01 * P01.re, s01 * P01.im);
    cmac_nc(Q01, P02, P12);
    cpx<float> Q02 = mkc<float>(s02 * P02.re, s02 * P02.im);
    cmac(Q02, P01, P12);
    cpx<float> Q12 = mkc<float>(s12 * P12.re, s12 * P12.im);
    cmac_cn(Q12, P01, P02);
    const float trp = p0 + p1 + p2;
    const float trq = q0 + q1 + q2;
    const cpx<float> t = small::cmul(P01, P12);
    const float re3 = fmaf(t.re, P02.re, t.im * P02.im);
    float det = p0 * fmaf(p1, p2, -n12);
    det = fmaf(-p1, n02, det);
    det = fmaf(-p2, n01, det);
    det = fmaf(2.f, re3, det);
    // The scalar series runs in FP64.  In FP32 the P^2 coefficient would carry
    // fl(eps^2) while the P coefficient carries eps: that rounding is the same
    // for every link, so E would miss unitarity by the fixed amount
    // (eps^2 - fl(eps^2)) P^2 at every update, and the link norms -- hence
    // the action -- would drift in one direction (about +0.04 in dH per
    // 50-step trajectory at SU(3) 32^4).  From FP64 coefficients each FP32
    // rounding is link-dependent and the remaining error averages out.
    const double e1 = (double)eps;
    const double tau = e1 * (double)trp;
    const double c1 = 0.5 * fma(e1 * e1, (double)trq, -tau * tau);
    const double dd = -(e1 * e1 * e1) * (double)det;
    double a = 1.0, b = 0.0, g = 0.0, f = 1.0;
    double Ar = 0.0, Ai = 0.0, Br = 0.0, Bi = 0.0, Cr = 0.0, Ci = 0.0;
#pragma unroll
    for (int k = 1; k <= 8; k++) {
      if (k > order) break;
      const double na = -dd * g;
      const double nb = fma(c1, g, a);
      const double ng = fma(tau, g, b);
      a = na;
      b = nb;
      g = ng;
      f = f * (1.0 / k);
      const double sf = (k & 2) ? -f : f;
      if (k & 1) {
        Ai = fma(sf, a, Ai);
        Bi = fma(sf, b, Bi);
        Ci = fma(sf, g, Ci);
      } else {
        Ar = fma(sf, a, Ar);
        Br = fma(sf, b, Br);
        Cr = fma(sf, g, Cr);
      }
    }
    const double e2 = e1 * e1;
    const cpx<float> A = mkc<float>((float)Ar, (float)Ai);
    const cpx<float> B = mkc<float>((float)(Br * e1), (float)(Bi * e1));
    const cpx<float> C = mkc<float>((float)(Cr * e2), (float)(Ci * e2));
    // Each entry is summed from its smallest term up and ends on its largest
    // (C q_i for the real diagonal, B P for everything else), so that it is
    // rounded once at its final size.  Rounded after the large term, a term
    // below half an ulp of the entry (C.im ~ eps^5 det P / 120, A.im) would be
    // dropped outright rather than rounded; those terms carry the part of
    // unitarity that goes as (det P)^2, so every link would lose norm
    // (~1.8e-12 in tr(E E^+) per update, +1e-3 in dH per 50-step trajectory
    // at SU(3) 32^4).
    const float pd[3] = {p0, p1, p2}, qd[3] = {q0, q1, q2};
#pragma unroll
    for (int i = 0; i < 3; i++) {
      E.a[i][i].re = fmaf(C.re, qd[i], fmaf(B.re, pd[i], A.re));
      E.a[i][i].im = fmaf(B.im, pd[i], fmaf(C.im, qd[i], A.im));
    }
    const cpx<float> Qu[3] = {Q01, Q02, Q12};
    const int iu[3] = {0, 0, 1}, ju[3] = {1, 2, 2};
#pragma unroll
    for (int u = 0; u < 3; u++) {
      const int i = iu[u], j = ju[u];
      const cpx<float> q = Qu[u], pu = P.a[i][j], pl = P.a[j][i];
      // upper: B P_ij + C Q_ij
      float r = fmaf(B.re, pu.re, -(C.im * q.im));
      r = fmaf(C.re, q.re, r);
      r = fmaf(-B.im, pu.im, r);
      float m = fmaf(B.re, pu.im, C.im * q.re);
      m = fmaf(C.re, q.im, m);
      m = fmaf(B.im, pu.re, m);
      E.a[i][j] = mkc<float>(r, m);
      // lower: B P_ji + C conj(Q_ij)
      r = fmaf(B.re, pl.re, C.im * q.im);
      r = fmaf(C.re, q.re, r);
      r = fmaf(-B.im, pl.im, r);
      m = fmaf(B.re, pl.im, C.im * q.re);
      m = fmaf(-C.re, q.im, m);
      m = fmaf(B.im, pl.re, m);
      E.a[j][i] = mkc<float>(r, m);
    }
  } else if constexpr (N == 2) {
    Mat<2, float> X;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) X.a[i][j] = mkc<float>(-eps * P.a[i][j].im, eps * P.a[i][j].re);
    // tr X and det X of the FP32 X, then the scalar series in FP64: summed in
    // FP32, its small high-order terms (d^2/120 ~ 1e-8 added to ~1) would be
    // rounded away in every link the same way, and E would lose norm on
    // average (~4e-12 per update at |X|^2 ~ 1e-3), an energy drift.
    const double trr = (double)X.a[0][0].re + (double)X.a[1][1].re;
    const double tri = (double)X.a[0][0].im + (double)X.a[1][1].im;
    const double dr = (double)X.a[0][0].re * X.a[1][1].re - (double)X.a[0][0].im * X.a[1][1].im -
                      ((double)X.a[0][1].re * X.a[1][0].re - (double)X.a[0][1].im * X.a[1][0].im);
    const double di = (double)X.a[0][0].re * X.a[1][1].im + (double)X.a[0][0].im * X.a[1][1].re -
                      ((double)X.a[0][1].re * X.a[1][0].im + (double)X.a[0][1].im * X.a[1][0].re);
    double alr = 1.0, ali = 0.0, ber = 0.0, bei = 0.0;
    double sar = 0.0, sai = 0.0, sbr = 0.0, sbi = 0.0;  // the X^0 term is left out: E - 1
    double f = 1.0;
#pragma unroll
    for (int k = 1; k <= 8; k++) {
      if (k > order) break;
      // X^k = -be_{k-1} det 1 + (al_{k-1} + be_{k-1} tr) X
      const double nalr = -(ber * dr - bei * di), nali = -(ber * di + bei * dr);
      const double nber = alr + (ber * trr - bei * tri), nbei = ali + (ber * tri + bei * trr);
      alr = nalr;
      ali = nali;
      ber = nber;
      bei = nbei;
      f = f * (1.0 / k);
      sar = fma(f, alr, sar);
      sai = fma(f, ali, sai);
      sbr = fma(f, ber, sbr);
      sbi = fma(f, bei, sbi);
    }
    const cpx<float> sa = mkc<float>((float)sar, (float)sai), sb = mkc<float>((float)sbr, (float)sbi);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        cpx<float> e = i == j ? sa : czero<float>();
        cmac(e, sb, X.a[i][j]);
        E.a[i][j] = e;
      }
  } else {
    Mat<N, float> X;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) X.a[i][j] = mkc<float>(-eps * P.a[i][j].im, eps * P.a[i][j].re);
    // Y_order = X / order;  Y_n = X/n (1 + Y_{n+1});  E - 1 = Y_1
    small::zero(E);
    for (int n = order; n >= 1; n--) {
      const float inv = 1.f / n;
      Mat<N, float> Y;
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          cpx<float> s = X.a[i][j];  // X * 1
#pragma unroll
          for (int k = 0; k < N; k++) cmac(s, X.a[i][k], E.a[k][j]);
          Y.a[i][j] = mkc<float>(s.re * inv, s.im * inv);
        }
      E = Y;
    }
  }
}

// ---- the fused kick + drift ------------------------------------------------------
// MODE 0: Pout = Pin - eps_k F(U)                      (updateE)
// MODE 1: P -= eps_k F(U);  U' = U + (E - 1) U_hi      (updateE + updateUandcopyDown)
// with U' written to (Uout, ULout); Pin may equal Pout.  Same site-tile
// mapping as small::k_force: 32 consecutive sites per CTA, one warp per
// direction.
template <int N, int MODE>
__device__ __forceinline__ void link_update(const Lat& L, const float2* __restrict__ U, const uint32_t* __restrict__ UL,
                                            const float* Pin, const uint32_t* PLin, float* Pout, uint32_t* PLout,
                                            float2* __restrict__ Uout, uint32_t* __restrict__ ULout, float eps_k,
                                            float eps_d, int order, int mu, int x) {
  using small::Mat;
  constexpr int NC = Dims<N>::NCOEF;
  Mat<N, float> acc, Ux, W;
  small::staple_sum<N, float, float2>(acc, U, L, mu, x);
  small::load(Ux, U, L, mu, x);
  small::mul_nn(W, Ux, acc);
  float f[NC], ph[NC], pl[NC];
  force_coefs<N>(f, W);
  load_coefs<N>(ph, pl, Pin, PLin, L, mu, x);
#pragma unroll
  for (int k = 0; k + 1 < NC; k += 2) {
    const float2 dk = __fmul2_rn(make_float2(-eps_k, -eps_k), make_float2(f[k], f[k + 1]));
    add_split2(ph[k], ph[k + 1], pl[k], pl[k + 1], dk.x, dk.y);
  }
  if constexpr (NC % 2 == 1) add_split(ph[NC - 1], pl[NC - 1], __fmul_rn(-eps_k, f[NC - 1]));
  store_coefs<N>(Pout, PLout, ph, pl, L, mu, x);
  if (MODE == 1) {
    Mat<N, float> P, E, Dm, Ul;
    coefs_to_mat<N, float>(P, ph);
    exp_minus_one<N>(E, P, eps_d, order);
    small::mul_nn(Dm, E, Ux);
    load_lo<N>(Ul, UL, L, mu, x);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        add_split2(Ux.a[i][j].re, Ux.a[i][j].im, Ul.a[i][j].re, Ul.a[i][j].im, Dm.a[i][j].re, Dm.a[i][j].im);
      }
    small::store(Uout, Ux, L, mu, x);
    store_lo<N>(ULout, Ul, L, mu, x);
  }
}

// Register budget: at most 128 registers (4 resident CTAs of 128 threads per
// SM) for OCC 0, bounded for 6 / 7 resident CTAs for OCC 1 / 2.
template <int N, int MODE, int OCC>
__global__ void __launch_bounds__(128, OCC == 0 ? 4 : 5 + OCC)
    k_force(Lat L, const float2* __restrict__ U, const uint32_t* __restrict__ UL, const float* Pin,
            const uint32_t* PLin, float* Pout, uint32_t* PLout, float2* __restrict__ Uout,
            uint32_t* __restrict__ ULout, float eps_k, float eps_d, int order) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  if (x >= L.V) return;
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5))
    link_update<N, MODE>(L, U, UL, Pin, PLin, Pout, PLout, Uout, ULout, eps_k, eps_d, order, mu, x);
}

// In-place link update without a kick: U <- U + (E - 1) U, E = exp(i eps P)
// (updateUandcopyDown on the momenta P).
template <int N>
__global__ void __launch_bounds__(128) k_drift(Lat L, float2* __restrict__ U, uint32_t* __restrict__ UL,
                                               const float* __restrict__ P, const uint32_t* __restrict__ PL, float eps,
                                               int order) {
  using small::Mat;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.V * L.D) return;
  const int mu = (int)(t / L.V);
  const int x = (int)(t - (long)mu * L.V);
  float ph[Dims<N>::NCOEF], pl[Dims<N>::NCOEF];
  load_coefs<N>(ph, pl, P, PL, L, mu, x);
  Mat<N, float> Pm, E, Dm, Ux, Ul;
  coefs_to_mat<N, float>(Pm, ph);
  small::load(Ux, U, L, mu, x);
  exp_minus_one<N>(E, Pm, eps, order);
  small::mul_nn(Dm, E, Ux);
  load_lo<N>(Ul, UL, L, mu, x);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      add_split(Ux.a[i][j].re, Ul.a[i][j].re, Dm.a[i][j].re);
      add_split(Ux.a[i][j].im, Ul.a[i][j].im, Dm.a[i][j].im);
    }
  small::store(U, Ux, L, mu, x);
  store_lo<N>(UL, Ul, L, mu, x);
}

// Projection onto SU(N) in FP64 from hi + lo (small::reunitarise: modified
// Gram-Schmidt of the first N-1 rows, last row completing det = 1) of link t
// (t = mu V + x), written back and, when Usave is given, also to (Usave, ULsave).
template <int N>
__device__ __forceinline__ void reunit_link(const Lat& L, float2* __restrict__ U, uint32_t* __restrict__ UL,
                                            float2* __restrict__ Usave, uint32_t* __restrict__ ULsave, long t) {
  if (t >= (long)L.V * L.D) return;
  const int mu = (int)(t / L.V);
  const int x = (int)(t - (long)mu * L.V);
  small::Mat<N, double> M;
  load_exact<N>(M, U, UL, L, mu, x);
  small::reunitarise(M);
  store_exact<N>(U, UL, M, L, mu, x);
  if (Usave) store_exact<N>(Usave, ULsave, M, L, mu, x);
}

template <int N>
__global__ void __launch_bounds__(128) k_reunit(Lat L, float2* __restrict__ U, uint32_t* __restrict__ UL,
                                                float2* __restrict__ Usave, uint32_t* __restrict__ ULsave) {
  reunit_link<N>(L, U, UL, Usave, ULsave, (long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Plaquette sums of site s (misc::plaq_site) on hi + lo in FP64, added to v.
template <int N>
__device__ __forceinline__ void plaq_site(const Lat& L, const float2* __restrict__ U, const uint32_t* __restrict__ UL,
                                          int s, double (&v)[2]) {
  if (s < L.V && counted(L, s)) {
    for (int mu = 0; mu < L.D; mu++) {
      const int xpmu = nb_plus(L, mu, s);
      for (int nu = mu + 1; nu < L.D; nu++) {
        const int xpnu = nb_plus(L, nu, s);
        // B and C whole, A = U_mu(s) and Dn = U_nu(s) a row at a time (the
        // products and sums in the same order as with all four matrices held)
        small::Mat<N, double> B, C;
        load_exact<N>(B, U, UL, L, nu, xpmu);
        load_exact<N>(C, U, UL, L, mu, xpnu);
        double tr = 0.0;
#pragma unroll
        for (int i = 0; i < N; i++) {
          cpx<double> a[N], dn[N];
          load_exact_row<N>(a, U, UL, L, mu, s, i);
          load_exact_row<N>(dn, U, UL, L, nu, s, i);
#pragma unroll
          for (int j = 0; j < N; j++) {
            cpx<double> ab = czero<double>(), dc = czero<double>();
#pragma unroll
            for (int k = 0; k < N; k++) {
              cmac(ab, a[k], B.a[k][j]);
              cmac(dc, dn[k], C.a[k][j]);
            }
            tr = fma(ab.re, dc.re, tr);
            tr = fma(ab.im, dc.im, tr);
          }
        }
        v[mu == 0 ? 0 : 1] += 1.0 - tr / N;
      }
    }
  }
}

// N <= 3: at most 128 registers (two 256-thread CTAs per SM; with all four
// matrices held, unbounded, it took 172 and left one).  N = 4 keeps its two whole
// FP64 matrices in registers (one CTA per SM; capped at 128 it spills 1.5 KB).
template <int N>
__global__ void __launch_bounds__(misc::RED_THREADS, N <= 3 ? 2 : 1) k_plaq(Lat L, const float2* __restrict__ U,
                                                            const uint32_t* __restrict__ UL,
                                                            double* __restrict__ partial) {
  double v[2] = {0.0, 0.0};
  plaq_site<N>(L, U, UL, blockIdx.x * blockDim.x + threadIdx.x, v);
  misc::block_sum<2>(v);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 2 + 0] = v[0];
    partial[blockIdx.x * 2 + 1] = v[1];
  }
}

// tr(P^2) of link t (t = d V + s) from coordinates hi + lo, 0 past the end
template <int N>
__device__ __forceinline__ double kinetic_link(const Lat& L, const float* __restrict__ P,
                                               const uint32_t* __restrict__ PL, long t) {
  if (t >= (long)L.V * L.D) return 0.0;
  const int d = (int)(t / L.V);
  const int s = (int)(t - (long)d * L.V);
  if (!counted(L, s)) return 0.0;
  float h[Dims<N>::NCOEF], l[Dims<N>::NCOEF];
  double c[Dims<N>::NCOEF];
  load_coefs<N>(h, l, P, PL, L, d, s);
#pragma unroll
  for (int k = 0; k < Dims<N>::NCOEF; k++) c[k] = (double)h[k] + (double)l[k];
  return coef_tr2<N>(c);
}

// Per-link sums in FP64 from hi + lo (misc::link_sums):
// [0] sum tr(Pa^2), [1] sum 1/4 tr((Pa+Pb)^2) (Pb != null), [2] sum ReTr((U U^dag - 1)^2) (U != null).
template <int N>
__global__ void __launch_bounds__(misc::RED_THREADS) k_linksums(Lat L, const float* __restrict__ Pa,
                                                                const uint32_t* __restrict__ PLa,
                                                                const float* __restrict__ Pb,
                                                                const uint32_t* __restrict__ PLb,
                                                                const float2* __restrict__ U,
                                                                const uint32_t* __restrict__ UL,
                                                                double* __restrict__ partial) {
  constexpr int NC = Dims<N>::NCOEF;
  double v[3] = {0.0, 0.0, 0.0};
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (long)L.V * L.D && counted(L, (int)(t % L.V))) {
    const int d = (int)(t / L.V);
    const int s = (int)(t - (long)d * L.V);
    if (Pa) {
      float h[NC], l[NC];
      double ca[NC];
      load_coefs<N>(h, l, Pa, PLa, L, d, s);
#pragma unroll
      for (int k = 0; k < NC; k++) ca[k] = (double)h[k] + (double)l[k];
      v[0] = coef_tr2<N>(ca);
      if (Pb) {
        load_coefs<N>(h, l, Pb, PLb, L, d, s);
#pragma unroll
        for (int k = 0; k < NC; k++) ca[k] += (double)h[k] + (double)l[k];
        v[1] = 0.25 * coef_tr2<N>(ca);
      }
    }
    if (U) {
      small::Mat<N, double> M;
      load_exact<N>(M, U, UL, L, d, s);
      double c = 0.0;
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          cpx<double> aij = czero<double>(), aji = czero<double>();
#pragma unroll
          for (int k = 0; k < N; k++) {
            cmac_nc(aij, M.a[i][k], M.a[j][k]);
            cmac_nc(aji, M.a[j][k], M.a[i][k]);
          }
          if (i == j) {
            aij.re -= 1.0;
            aji.re -= 1.0;
          }
          c = fma(aij.re, aji.re, c);
          c = fma(-aij.im, aji.im, c);
        }
      v[2] = c;
    }
  }
  misc::block_sum<3>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; k++) partial[blockIdx.x * 3 + k] = v[k];
}

// Momentum refresh into coordinates: the entries misc::refresh_link draws
// (same Philox stream, FP64), split into hi + lo.
template <int N>
__device__ __forceinline__ void refresh_link(const Lat& L, float* __restrict__ P, uint32_t* __restrict__ PL,
                                             uint64_t seed, uint32_t traj, double scale, long t) {
  constexpr int NC = Dims<N>::NCOEF;
  if (t >= (long)L.V * L.D) return;
  const int d = (int)(t / L.V);
  const int s = (int)(t - (long)d * L.V);
  double c[NC];
  misc::refresh_entries(L, seed, traj, scale, d, s, [&](int i, int j, const cpx<double>& v) {
    if (i < j) {
      const int p = i * N - i * (i + 1) / 2 + (j - i - 1);  // row-major index of the pair (i, j)
      c[2 * p] = v.re;
      c[2 * p + 1] = v.im;
    } else if (i == j && i < N - 1) {
      c[Dims<N>::NDIAG + i] = v.re;
    }
  });
  float h[NC], l[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) split_of(c[k], h[k], l[k]);
  store_coefs<N>(P, PL, h, l, L, d, s);
}

template <int N>
__global__ void k_refresh(Lat L, float* __restrict__ P, uint32_t* __restrict__ PL, uint64_t seed,
                          const unsigned long long* __restrict__ traj_dev, unsigned long long traj_host,
                          double scale) {
  const uint32_t traj = (uint32_t)(traj_dev ? *traj_dev : traj_host);
  refresh_link<N>(L, P, PL, seed, traj, scale, (long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---- conversions to and from the host U-conf layout ([site][dir][row][col][re,im] FP64) ----
template <int N>
__global__ void k_links_from_conf(Lat L, const double2* __restrict__ conf, float2* __restrict__ U,
                                  uint32_t* __restrict__ UL) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)field_elems(L)) return;
  constexpr int NN = N * N;
  const long rest = t >> 5;
  const int e = (int)(rest % NN);
  const long db = rest / NN;
  const int d = (int)(db / L.B);
  const int s = (int)((db - (long)d * L.B) * 32 + (t & 31));
  double2 v = make_double2(0.0, 0.0);
  if (s < L.V) v = conf[((size_t)s * L.D + d) * NN + e];
  float hr, lr, hi, li;
  split_of(v.x, hr, lr);
  split_of(v.y, hi, li);
  U[t] = make_float2(hr, hi);
  UL[t] = lo_pack(lr, li);
}

template <int N>
__global__ void k_links_to_conf(Lat L, const float2* __restrict__ U, const uint32_t* __restrict__ UL,
                                double2* __restrict__ conf) {
  constexpr int NN = N * N;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.V * L.D * NN) return;
  const long lk = t / NN;
  const int e = (int)(t - lk * NN);
  const int s = (int)(lk / L.D);
  const int d = (int)(lk - (long)s * L.D);
  const size_t o = eoff(L, d, e, s);
  const float2 h = U[o];
  const uint32_t w = UL[o];
  conf[t] = make_double2((double)h.x + (double)lo_low(w), (double)h.y + (double)lo_high(w));
}

// Momenta from U-conf matrices: the Hermitian traceless part of each matrix
// (exactly the matrix itself for momenta of the reference's form).
template <int N>
__global__ void k_momenta_from_conf(Lat L, const double2* __restrict__ conf, float* __restrict__ P,
                                    uint32_t* __restrict__ PL) {
  constexpr int NC = Dims<N>::NCOEF, NN = N * N;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.D * L.B * 32) return;
  const int d = (int)(t / ((long)L.B * 32));
  const int s = (int)(t - (long)d * L.B * 32);
  double c[NC];
  if (s < L.V) {
    const double2* m = conf + ((size_t)s * L.D + d) * NN;
    int p = 0;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = i + 1; j < N; j++, p++) {
        c[2 * p] = 0.5 * (m[i * N + j].x + m[j * N + i].x);
        c[2 * p + 1] = 0.5 * (m[i * N + j].y - m[j * N + i].y);
      }
    double tr = 0.0;
#pragma unroll
    for (int i = 0; i < N; i++) tr += m[i * N + i].x;
#pragma unroll
    for (int i = 0; i < N - 1; i++) c[Dims<N>::NDIAG + i] = m[i * N + i].x - tr / N;
  } else {
#pragma unroll
    for (int k = 0; k < NC; k++) c[k] = 0.0;
  }
  float h[NC], l[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) split_of(c[k], h[k], l[k]);
  store_coefs<N>(P, PL, h, l, L, d, s);
}

template <int N>
__global__ void k_momenta_to_conf(Lat L, const float* __restrict__ P, const uint32_t* __restrict__ PL,
                                  double2* __restrict__ conf) {
  constexpr int NC = Dims<N>::NCOEF;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.V * L.D) return;
  const int s = (int)(t / L.D);
  const int d = (int)(t - (long)s * L.D);
  float h[NC], l[NC];
  double c[NC];
  load_coefs<N>(h, l, P, PL, L, d, s);
#pragma unroll
  for (int k = 0; k < NC; k++) c[k] = (double)h[k] + (double)l[k];
  small::Mat<N, double> M;
  coefs_to_mat<N, double>(M, c);
  double2* m = conf + (size_t)t * N * N;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) m[i * N + j] = make_double2(M.a[i][j].re, M.a[i][j].im);
}

// Full FP32 momentum matrices (the float2 field layout) from coordinates, for
// the diagnostics that read matrices (Gauss law, Tab).
template <int N>
__global__ void k_momenta_to_matrix(Lat L, const float* __restrict__ P, const uint32_t* __restrict__ PL,
                                    float2* __restrict__ F) {
  constexpr int NC = Dims<N>::NCOEF;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.D * L.B * 32) return;
  const int d = (int)(t / ((long)L.B * 32));
  const int s = (int)(t - (long)d * L.B * 32);
  float h[NC], l[NC];
  double c[NC];
  load_coefs<N>(h, l, P, PL, L, d, s);
#pragma unroll
  for (int k = 0; k < NC; k++) c[k] = (double)h[k] + (double)l[k];
  small::Mat<N, double> M;
  coefs_to_mat<N, double>(M, c);
  small::Mat<N, float> Mf;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) Mf.a[i][j] = mkc<float>((float)M.a[i][j].re, (float)M.a[i][j].im);
  small::store(F, Mf, L, d, s);
}

// ---- slabs of sites in the U-conf layout ----------------------------------------
// Links of the sites [s0, s0 + ns) to / from buf in the U-conf order (FP64,
// element t = ((s - s0) D + d) NN + e), for any storage: S2 = double2 or float2,
// with the residual plane `lo` when non-null.  Used for the halo slabs of a
// domain-decomposed chain.
template <typename S2>
__global__ void k_slab_get(Lat L, const S2* __restrict__ f, const uint32_t* __restrict__ lo, int s0, int ns,
                           double2* __restrict__ buf) {
  const int NN = L.N * L.N;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)ns * L.D * NN) return;
  const long lk = t / NN;
  const int e = (int)(t - lk * NN);
  const int s = s0 + (int)(lk / L.D);
  const int d = (int)(lk - (lk / L.D) * L.D);
  const size_t o = eoff(L, d, e, s);
  cpx<double> v = ldc<double>(f + o);
  if (lo) {
    const uint32_t w = lo[o];
    v.re += (double)lo_low(w);
    v.im += (double)lo_high(w);
  }
  buf[t] = make_double2(v.re, v.im);
}

template <typename S2>
__global__ void k_slab_set(Lat L, S2* __restrict__ f, uint32_t* __restrict__ lo, int s0, int ns,
                           const double2* __restrict__ buf) {
  const int NN = L.N * L.N;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)ns * L.D * NN) return;
  const long lk = t / NN;
  const int e = (int)(t - lk * NN);
  const int s = s0 + (int)(lk / L.D);
  const int d = (int)(lk - (lk / L.D) * L.D);
  const size_t o = eoff(L, d, e, s);
  const double2 v = buf[t];
  if (lo) {
    float hr, lr, hi, li;
    split_of(v.x, hr, lr);
    split_of(v.y, hi, li);
    stc(f + o, mkc<float>(hr, hi));
    lo[o] = lo_pack(lr, li);
  } else {
    stc(f + o, mkc<double>(v.x, v.y));
  }
}

}  // namespace split
}  // namespace askja
