// Thread-per-link kernels for small colour number (NC <= 4): every matrix of
// the staple sum lives in registers, one thread owns one link (d, s), and the
// threads of a warp walk 32 consecutive sites of the same direction so every
// element load is one coalesced 256 B (FP32) / 512 B (FP64) transaction.
//
// Physics follows the reference (sun.cpp, sunmat.h):
//   force   F = Adjoint(U_mu(x) * sum_{nu != mu} [upper + lower staple])
//           (sun.cpp:702-716, Adjoint = sunmat.h:355-371)
//   kick    P <- P - eps * F
//   drift   U <- exp(i eps P) U, Taylor order `order` in Horner form
//           (sunmat.h:200-248, applied to U directly: U + X(U + X/2(U + ...)));
//           the FP32 path sums the same series through Cayley-Hamilton
//           (two matrix products instead of `order`, expi_times_ch)
// with the staple product factored as U_mu(x) * (sum of the remaining three
// links), which saves one matrix product per staple against the reference's
// left-to-right evaluation; results agree to rounding.
#pragma once

#include "common.cuh"

namespace askja {
namespace small {

template <int N, typename T>
struct Mat {
  cpx<T> a[N][N];
};

// one base address per matrix; the elements are 32 complex numbers apart
template <int N, typename T, typename S2>
__device__ __forceinline__ void load(Mat<N, T>& m, const S2* __restrict__ f, const Lat& L, int d, int s) {
  const S2* p = f + ((size_t)d * L.B + (s >> 5)) * (N * N * 32) + (s & 31);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) m.a[i][j] = ldc<T>(p + (i * N + j) * 32);
}

template <int N, typename T, typename S2>
__device__ __forceinline__ void store(S2* __restrict__ f, const Mat<N, T>& m, const Lat& L, int d, int s) {
  S2* p = f + ((size_t)d * L.B + (s >> 5)) * (N * N * 32) + (s & 31);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) stc(p + (i * N + j) * 32, m.a[i][j]);
}

template <int N, typename T>
__device__ __forceinline__ void zero(Mat<N, T>& m) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) m.a[i][j] = czero<T>();
}

// FP32 products in packed FP32x2 (FFMA2 of sm_100).  Every product is
// written as X Y^dag: for each element, (re, im) += (x.re, x.im) * (y.re, y.re)
// then += (x.im, -x.re) * (y.im, y.im), two FFMA2 per complex multiply-add
// instead of four FFMA; the left element is used as loaded plus one swapped,
// negated copy, the right one's parts are broadcast (negated where Y is a
// conjugate).  A B is A (B^dag)^dag, A^dag B^dag is (A^dag) B^dag.  Per
// element A B^dag adds its terms in the order of cmac_nc (bit-identical to
// the scalar form); A B and A^dag B^dag add the imaginary part's two terms in
// the other order than cmac / cmac_cc.  At SU(3) 32^4 this took the residual-plane fused kernel
// from 409 to 388 us and the FP32-only one from 385 to 349 us (A B with
// broadcast left parts and a swapped right copy instead: 402-405 us).
// c[j] += sum_k x(k) conj(y(j, k)) for the N columns j of one row
template <int N, typename FL, typename FR>
__device__ __forceinline__ void row_x2(float2 (&c)[N], FL&& x, FR&& y) {
  float2 an[N], ar[N];
#pragma unroll
  for (int k = 0; k < N; k++) {
    const cpx<float> a = x(k);
    an[k] = make_float2(a.re, a.im);
    ar[k] = make_float2(a.im, -a.re);
  }
#pragma unroll
  for (int j = 0; j < N; j++)
#pragma unroll
    for (int k = 0; k < N; k++) {
      const cpx<float> b = y(j, k);
      c[j] = __ffma2_rn(an[k], make_float2(b.re, b.re), c[j]);
      c[j] = __ffma2_rn(ar[k], make_float2(b.im, b.im), c[j]);
    }
}

// rows 0 .. ROWS-1 of C (+)= X Y^dag in FP32, X and Y given element-wise
template <int N, int ROWS, bool ACC, typename FL, typename FR>
__device__ __forceinline__ void prod_x2(Mat<N, float>& C, FL&& x, FR&& y) {
#pragma unroll
  for (int i = 0; i < ROWS; i++) {
    float2 c[N];
#pragma unroll
    for (int j = 0; j < N; j++) c[j] = ACC ? make_float2(C.a[i][j].re, C.a[i][j].im) : make_float2(0.f, 0.f);
    row_x2<N>(c, [&](int k) { return x(i, k); }, y);
#pragma unroll
    for (int j = 0; j < N; j++) C.a[i][j] = mkc<float>(c[j].x, c[j].y);
  }
}

// C = A * B^dag (rows 0 .. ROWS-1)
template <int N, typename T, int ROWS = N>
__device__ __forceinline__ void mul_nd(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  if constexpr (sizeof(T) == 4) {
    prod_x2<N, ROWS, false>(C, [&](int i, int k) { return A.a[i][k]; }, [&](int j, int k) { return B.a[j][k]; });
  } else {
#pragma unroll
    for (int i = 0; i < ROWS; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        cpx<T> s = czero<T>();
#pragma unroll
        for (int k = 0; k < N; k++) cmac_nc(s, A.a[i][k], B.a[j][k]);
        C.a[i][j] = s;
      }
  }
}
// C += A * B^dag
template <int N, typename T>
__device__ __forceinline__ void mac_nd(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  if constexpr (sizeof(T) == 4) {
    prod_x2<N, N, true>(C, [&](int i, int k) { return A.a[i][k]; }, [&](int j, int k) { return B.a[j][k]; });
  } else {
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++)
#pragma unroll
        for (int k = 0; k < N; k++) cmac_nc(C.a[i][j], A.a[i][k], B.a[j][k]);
  }
}
// C = A^dag * B^dag  (= (B A)^dag; rows 0 .. ROWS-1)
template <int N, typename T, int ROWS = N>
__device__ __forceinline__ void mul_dd(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  if constexpr (sizeof(T) == 4) {
    prod_x2<N, ROWS, false>(
        C, [&](int i, int k) { return mkc<float>(A.a[k][i].re, -A.a[k][i].im); },
        [&](int j, int k) { return B.a[j][k]; });
  } else {
#pragma unroll
    for (int i = 0; i < ROWS; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        cpx<T> s = czero<T>();
#pragma unroll
        for (int k = 0; k < N; k++) cmac_cc(s, A.a[k][i], B.a[j][k]);
        C.a[i][j] = s;
      }
  }
}
// C += A * B
template <int N, typename T>
__device__ __forceinline__ void mac_nn(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  if constexpr (sizeof(T) == 4) {
    prod_x2<N, N, true>(C, [&](int i, int k) { return A.a[i][k]; },
                        [&](int j, int k) { return mkc<float>(B.a[k][j].re, -B.a[k][j].im); });
  } else {
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++)
#pragma unroll
        for (int k = 0; k < N; k++) cmac(C.a[i][j], A.a[i][k], B.a[k][j]);
  }
}
// C = A * B
template <int N, typename T>
__device__ __forceinline__ void mul_nn(Mat<N, T>& C, const Mat<N, T>& A, const Mat<N, T>& B) {
  if constexpr (sizeof(T) == 4) {
    prod_x2<N, N, false>(C, [&](int i, int k) { return A.a[i][k]; },
                         [&](int j, int k) { return mkc<float>(B.a[k][j].re, -B.a[k][j].im); });
  } else {
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        cpx<T> s = czero<T>();
#pragma unroll
        for (int k = 0; k < N; k++) cmac(s, A.a[i][k], B.a[k][j]);
        C.a[i][j] = s;
      }
  }
}

// Third row of an SU(3) matrix from the first two: conj(r0 x r1).
template <typename T>
__device__ __forceinline__ void su3_third_row(Mat<3, T>& M) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
    cpx<T> c = czero<T>();
    cmac(c, M.a[0][k1], M.a[1][k2]);
    cmsub(c, M.a[0][k2], M.a[1][k1]);
    M.a[2][k] = mkc<T>(c.re, -c.im);
  }
}

// Sum of the 2(D-1) staples around link (mu, x), without the leading U_mu(x):
//   sum_{nu != mu} U_nu(x+mu) U_mu^dag(x+nu) U_nu^dag(x)
//               + U_nu^dag(x+mu-nu) U_mu^dag(x-nu) U_nu(x-nu)
// FP32 SU(3): the product of the first two links of a staple is itself in
// SU(3), so its third row is taken as conj(r0 x r1) (24 instead of 36 real
// multiply-adds; exact for links in SU(3), which the FP32 path keeps by
// reunitarising every update).
template <int N, typename T, typename S2>
__device__ __forceinline__ void staple_sum(Mat<N, T>& acc, const S2* __restrict__ U, const Lat& L, int mu, int x) {
  constexpr bool R2 = N == 3 && sizeof(T) == 4;
  zero(acc);
  const int xpmu = nb_plus(L, mu, x);
  for (int nu = 0; nu < L.D; nu++) {
    if (nu == mu) continue;
    const int xpnu = nb_plus(L, nu, x);
    const int xmnu = nb_minus(L, nu, x);
    const int xpmu_mnu = nb_minus(L, nu, xpmu);
    {
      Mat<N, T> A, B, T1;
      load(A, U, L, nu, xpmu);
      load(B, U, L, mu, xpnu);
      mul_nd<N, T, R2 ? 2 : N>(T1, A, B);
      if constexpr (R2) su3_third_row(T1);
      load(A, U, L, nu, x);
      mac_nd(acc, T1, A);
    }
    {
      Mat<N, T> A, B, T1;
      load(A, U, L, nu, xpmu_mnu);
      load(B, U, L, mu, xmnu);
      mul_dd<N, T, R2 ? 2 : N>(T1, A, B);
      if constexpr (R2) su3_third_row(T1);
      load(A, U, L, nu, xmnu);
      mac_nn(acc, T1, A);
    }
  }
}

// P <- P - eps * Adjoint(W), Adjoint(W) = -i/2 [(W - W^dag) - Tr(W - W^dag)/N]
template <int N, typename T>
__device__ __forceinline__ void kick_ta(Mat<N, T>& P, const Mat<N, T>& W, T eps) {
  T trim = T(0);
#pragma unroll
  for (int k = 0; k < N; k++) trim += W.a[k][k].im;
  if constexpr (sizeof(T) == 4)
    trim = trim * (T(1) / T(N));  // FP32: a constant multiply instead of a division
  else
    trim = trim / T(N);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      T fr, fi;
      if (i == j) {
        fr = W.a[i][i].im - trim;
        fi = T(0);
      } else {
        fr = T(0.5) * (W.a[i][j].im + W.a[j][i].im);
        fi = T(-0.5) * (W.a[i][j].re - W.a[j][i].re);
      }
      P.a[i][j].re = fma(-eps, fr, P.a[i][j].re);
      P.a[i][j].im = fma(-eps, fi, P.a[i][j].im);
    }
}

// Tm <- exp(i eps P) U to Taylor order `order` (Horner, applied to U)
template <int N, typename T>
__device__ __forceinline__ void expi_times(Mat<N, T>& Tm, const Mat<N, T>& P, const Mat<N, T>& Ux, T eps, int order) {
  Mat<N, T> X;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) X.a[i][j] = mkc<T>(-eps * P.a[i][j].im, eps * P.a[i][j].re);
  Tm = Ux;
  for (int n = order; n >= 1; n--) {
    const T inv = T(1) / T(n);
    Mat<N, T> Y;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        cpx<T> s = czero<T>();
#pragma unroll
        for (int k = 0; k < N; k++) cmac(s, X.a[i][k], Tm.a[k][j]);
        Y.a[i][j] = mkc<T>(fma(s.re, inv, Ux.a[i][j].re), fma(s.im, inv, Ux.a[i][j].im));
      }
    Tm = Y;
  }
}

template <typename T>
__device__ __forceinline__ cpx<T> cmul(const cpx<T>& a, const cpx<T>& b) {
  cpx<T> z = czero<T>();
  cmac(z, a, b);
  return z;
}

// The same truncated series sum_{k<=order} X^k / k!, X = i eps P, for N = 2
// and 3, evaluated through the Cayley-Hamilton theorem instead of Horner:
// X^N is a combination of 1 .. X^(N-1) (coefficients from tr X, tr X^2 and
// det X), so X^k = al_k 1 + be_k X (+ ga_k X^2) with a scalar recursion, and
// E = sum (al_k, be_k, ga_k) / k! needs one matrix product (X^2, N = 3) before
// the final E U -- two products instead of `order`.  Exact in real
// arithmetic for any X (no hermiticity assumed); rounding differs from
// Horner at the level of the storage precision.
template <int N, typename T>
__device__ __forceinline__ void expi_times_ch(Mat<N, T>& Tm, const Mat<N, T>& P, const Mat<N, T>& Ux, T eps,
                                              int order) {
  static_assert(N == 2 || N == 3, "Cayley-Hamilton form for N = 2, 3");
  Mat<N, T> X;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) X.a[i][j] = mkc<T>(-eps * P.a[i][j].im, eps * P.a[i][j].re);
  cpx<T> tr = czero<T>();
#pragma unroll
  for (int i = 0; i < N; i++) {
    tr.re += X.a[i][i].re;
    tr.im += X.a[i][i].im;
  }
  Mat<N, T> E;
  if constexpr (N == 2) {
    // X^2 = tr X X - det X 1
    cpx<T> d = cmul(X.a[0][0], X.a[1][1]);
    cmsub(d, X.a[0][1], X.a[1][0]);
    cpx<T> al = mkc<T>(T(1), T(0)), be = czero<T>();  // X^0
    cpx<T> sa = al, sb = be;
    T f = T(1);
#pragma unroll
    for (int k = 1; k <= 8; k++) {  // order <= 8; unrolled so that 1/k is a constant
      if (k > order) break;
      // X^k = -be_{k-1} det 1 + (al_{k-1} + be_{k-1} tr) X
      cpx<T> nal = czero<T>(), nbe = al;
      cmsub(nal, be, d);
      cmac(nbe, be, tr);
      al = nal;
      be = nbe;
      f = f * T(1.0 / k);
      sa.re = fma(f, al.re, sa.re);
      sa.im = fma(f, al.im, sa.im);
      sb.re = fma(f, be.re, sb.re);
      sb.im = fma(f, be.im, sb.im);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        cpx<T> e = i == j ? sa : czero<T>();
        cmac(e, sb, X.a[i][j]);
        E.a[i][j] = e;
      }
  } else {
    Mat<N, T> X2;
    mul_nn(X2, X, X);
    cpx<T> tr2 = czero<T>();
#pragma unroll
    for (int i = 0; i < 3; i++) {
      tr2.re += X2.a[i][i].re;
      tr2.im += X2.a[i][i].im;
    }
    // c1 = ((tr X)^2 - tr X^2) / 2, c0 = det X; X^3 = tr X X^2 - c1 X + c0 1
    cpx<T> c1 = cmul(tr, tr);
    c1.re = T(0.5) * (c1.re - tr2.re);
    c1.im = T(0.5) * (c1.im - tr2.im);
    cpx<T> m0 = cmul(X.a[1][1], X.a[2][2]), m1 = cmul(X.a[1][0], X.a[2][2]), m2 = cmul(X.a[1][0], X.a[2][1]);
    cmsub(m0, X.a[1][2], X.a[2][1]);
    cmsub(m1, X.a[1][2], X.a[2][0]);
    cmsub(m2, X.a[1][1], X.a[2][0]);
    cpx<T> c0 = cmul(X.a[0][0], m0);
    cmsub(c0, X.a[0][1], m1);
    cmac(c0, X.a[0][2], m2);
    cpx<T> al = mkc<T>(T(1), T(0)), be = czero<T>(), ga = czero<T>();  // X^0
    cpx<T> sa = al, sb = be, sc = ga;
    T f = T(1);
#pragma unroll
    for (int k = 1; k <= 8; k++) {  // order <= 8; unrolled so that 1/k is a constant
      if (k > order) break;
      // X^k = ga c0 1 + (al - ga c1) X + (be + ga tr) X^2  (coefficients of X^(k-1))
      const cpx<T> nal = cmul(ga, c0);
      cpx<T> nbe = al, nga = be;
      cmsub(nbe, ga, c1);
      cmac(nga, ga, tr);
      al = nal;
      be = nbe;
      ga = nga;
      f = f * T(1.0 / k);
      sa.re = fma(f, al.re, sa.re);
      sa.im = fma(f, al.im, sa.im);
      sb.re = fma(f, be.re, sb.re);
      sb.im = fma(f, be.im, sb.im);
      sc.re = fma(f, ga.re, sc.re);
      sc.im = fma(f, ga.im, sc.im);
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        cpx<T> e = i == j ? sa : czero<T>();
        cmac(e, sb, X.a[i][j]);
        cmac(e, sc, X2.a[i][j]);
        E.a[i][j] = e;
      }
  }
  mul_nn(Tm, E, Ux);
}

// The same series for N = 3 written in P, for Hermitian P (every momentum
// field of the reference and of this engine: the refresh draws P in the
// algebra and the kick adds the same real part to P_ij and P_ji and opposite
// imaginary parts, so P_ij = conj(P_ji) holds exactly; the diagonal is taken
// real).  With X = i eps P, tr X = i tau, det X = i d and the coefficient c1
// of the characteristic polynomial are imaginary, imaginary and real, so the
// coefficients of X^k = al_k 1 + be_k X + ga_k X^2 are al_k = i^k a_k,
// be_k = i^(k-1) b_k, ga_k = i^(k-2) g_k with a real recursion
//   a_k = -d g_(k-1),  b_k = a_(k-1) + c1 g_(k-1),  g_k = b_(k-1) + tau g_(k-1),
// and  E = A 1 + B P + C P^2  with  A = sum i^k a_k/k!, B = eps sum i^k b_k/k!,
// C = eps^2 sum i^k g_k/k!.  P^2 is Hermitian: its upper triangle and real
// diagonal are formed (no X, no full X^2 product).  E - 1 is formed and the
// result is U + (E - 1) U.
template <typename T>
__device__ __forceinline__ void expi_times_herm3(Mat<3, T>& Tm, const Mat<3, T>& P, const Mat<3, T>& Ux, T eps,
                                                 int order) {
  const T p0 = P.a[0][0].re, p1 = P.a[1][1].re, p2 = P.a[2][2].re;
  const cpx<T>& P01 = P.a[0][1];
  const cpx<T>& P02 = P.a[0][2];
  const cpx<T>& P12 = P.a[1][2];
  const T n01 = cnorm2_add(P01, T(0)), n02 = cnorm2_add(P02, T(0)), n12 = cnorm2_add(P12, T(0));
  // Q = P^2: diagonal and upper triangle
  const T q0 = fma(p0, p0, n01 + n02), q1 = fma(p1, p1, n01 + n12), q2 = fma(p2, p2, n02 + n12);
  const T s01 = p0 + p1, s02 = p0 + p2, s12 = p1 + p2;
  cpx<T> Q01 = mkc<T>(s01 * P01.re, s01 * P01.im);
  cmac_nc(Q01, P02, P12);  // + P02 P21
  cpx<T> Q02 = mkc<T>(s02 * P02.re, s02 * P02.im);
  cmac(Q02, P01, P12);  // + P01 P12
  cpx<T> Q12 = mkc<T>(s12 * P12.re, s12 * P12.im);
  cmac_cn(Q12, P01, P02);  // + P10 P02
  // invariants: tr P, tr P^2, det P (real)
  const T trp = p0 + p1 + p2;
  const T trq = q0 + q1 + q2;
  const cpx<T> t = cmul(P01, P12);
  const T re3 = fma(t.re, P02.re, t.im * P02.im);  // Re(P01 P12 P20)
  T det = p0 * fma(p1, p2, -n12);
  det = fma(-p1, n02, det);
  det = fma(-p2, n01, det);
  det = fma(T(2), re3, det);
  const T tau = eps * trp;
  const T c1 = T(0.5) * fma(eps * eps, trq, -tau * tau);
  const T d = -(eps * eps * eps) * det;
  T a = T(1), b = T(0), g = T(0);
  // A without its k = 0 term: E - 1 is formed, and Tm = U + (E - 1) U keeps the
  // small update apart from U's own bits
  cpx<T> A = czero<T>(), B = czero<T>(), C = czero<T>();
  T f = T(1);
#pragma unroll
  for (int k = 1; k <= 8; k++) {  // order <= 8; unrolled so that 1/k! and i^k are constants
    if (k > order) break;
    const T na = -d * g;
    const T nb = fma(c1, g, a);
    const T ng = fma(tau, g, b);
    a = na;
    b = nb;
    g = ng;
    f = f * T(1.0 / k);
    const T sf = (k & 2) ? -f : f;  // i^k = +1, +i, -1, -i
    if (k & 1) {
      A.im = fma(sf, a, A.im);
      B.im = fma(sf, b, B.im);
      C.im = fma(sf, g, C.im);
    } else {
      A.re = fma(sf, a, A.re);
      B.re = fma(sf, b, B.re);
      C.re = fma(sf, g, C.re);
    }
  }
  B.re *= eps;
  B.im *= eps;
  const T e2 = eps * eps;
  C.re *= e2;
  C.im *= e2;
  // Each entry is summed from its smallest term up and ends on its largest, so
  // that terms below half an ulp of the entry (C.im, A.im) are rounded with
  // it instead of being dropped: dropped, they take away a (det P)^2 part of
  // unitarity and every update shrinks the link a little.
  Mat<3, T> E;
  const T pd[3] = {p0, p1, p2}, qd[3] = {q0, q1, q2};
#pragma unroll
  for (int i = 0; i < 3; i++) {
    E.a[i][i].re = fma(C.re, qd[i], fma(B.re, pd[i], A.re));
    E.a[i][i].im = fma(B.im, pd[i], fma(C.im, qd[i], A.im));
  }
  const cpx<T> Qu[3] = {Q01, Q02, Q12};
  const int iu[3] = {0, 0, 1}, ju[3] = {1, 2, 2};
#pragma unroll
  for (int u = 0; u < 3; u++) {
    const int i = iu[u], j = ju[u];
    const cpx<T> q = Qu[u], pu = P.a[i][j], pl = P.a[j][i];
    // upper: B P_ij + C Q_ij
    T r = fma(B.re, pu.re, -(C.im * q.im));
    r = fma(C.re, q.re, r);
    r = fma(-B.im, pu.im, r);
    T m = fma(B.re, pu.im, C.im * q.re);
    m = fma(C.re, q.im, m);
    m = fma(B.im, pu.re, m);
    E.a[i][j] = mkc<T>(r, m);
    // lower: B P_ji + C conj(Q_ij)
    r = fma(B.re, pl.re, C.im * q.im);
    r = fma(C.re, q.re, r);
    r = fma(-B.im, pl.im, r);
    m = fma(B.re, pl.im, C.im * q.re);
    m = fma(-C.re, q.im, m);
    m = fma(B.im, pl.re, m);
    E.a[j][i] = mkc<T>(r, m);
  }
  Tm = Ux;
  mac_nn(Tm, E, Ux);
}

// Link update of the FP32 path: the Cayley-Hamilton form (for N = 3 in P,
// Hermitian P); the FP64 path keeps the reference's Horner evaluation.
template <int N, typename T>
__device__ __forceinline__ void expi_update(Mat<N, T>& Tm, const Mat<N, T>& P, const Mat<N, T>& Ux, T eps, int order) {
  if constexpr (sizeof(T) == 4 && N == 3)
    expi_times_herm3(Tm, P, Ux, eps, order);
  else if constexpr (sizeof(T) == 4 && N == 2)
    expi_times_ch(Tm, P, Ux, eps, order);
  else
    expi_times(Tm, P, Ux, eps, order);
}

// Project onto SU(N): modified Gram-Schmidt of rows 0..N-2 (in order), then
// the last row is the unique unit row that completes them to determinant 1
// (the conjugated generalised cross product of the other rows).
template <int N, typename T>
__device__ __forceinline__ void reunitarise(Mat<N, T>& M) {
#pragma unroll
  for (int r = 0; r < N - 1; r++) {
#pragma unroll
    for (int q = 0; q < r; q++) {
      cpx<T> pr = czero<T>();
#pragma unroll
      for (int k = 0; k < N; k++) cmac_cn(pr, M.a[q][k], M.a[r][k]);
#pragma unroll
      for (int k = 0; k < N; k++) cmsub(M.a[r][k], pr, M.a[q][k]);
    }
    T nrm = T(0);
#pragma unroll
    for (int k = 0; k < N; k++) nrm = cnorm2_add(M.a[r][k], nrm);
    T inv;
    if constexpr (sizeof(T) == 4)
      inv = rsqrtf(nrm);  // FP32 path: the approximate reciprocal square root (2 ulp) suffices
    else
      inv = T(1) / sqrt(nrm);
#pragma unroll
    for (int k = 0; k < N; k++) {
      M.a[r][k].re *= inv;
      M.a[r][k].im *= inv;
    }
  }
  if (N == 1) {
    M.a[0][0] = mkc<T>(T(1), T(0));
  } else if (N == 2) {
    // last row = (-conj(a01), conj(a00))
    M.a[1][0] = mkc<T>(-M.a[0][1].re, M.a[0][1].im);
    M.a[1][1] = mkc<T>(M.a[0][0].re, -M.a[0][0].im);
  } else if (N == 3) {
    // last row = conj(r0 x r1)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
      cpx<T> c = czero<T>();
      cmac(c, M.a[0][k1], M.a[1][k2]);
      cmsub(c, M.a[0][k2], M.a[1][k1]);
      M.a[2][k] = mkc<T>(c.re, -c.im);
    }
  } else if (N == 4) {
    // last row k = conj of cofactor C_{3k} of rows 0..2, so that det = sum_k a3k C3k = 1
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int c0 = (k == 0) ? 1 : 0;
      int c1 = (k <= 1) ? 2 : 1;
      int c2 = (k <= 2) ? 3 : 2;
      // 3x3 minor of rows 0..2, columns c0<c1<c2
      cpx<T> m = czero<T>();
      const int cols[3] = {c0, c1, c2};
#pragma unroll
      for (int p = 0; p < 3; p++) {
        const int q1 = (p + 1) % 3, q2 = (p + 2) % 3;
        cpx<T> t = czero<T>();
        cmac(t, M.a[1][cols[q1]], M.a[2][cols[q2]]);
        cmsub(t, M.a[1][cols[q2]], M.a[2][cols[q1]]);
        cmac(m, M.a[0][cols[p]], t);
      }
      const T sgn = ((3 + k) & 1) ? T(-1) : T(1);
      M.a[3][k] = mkc<T>(sgn * m.re, -sgn * m.im);
    }
  }
}

// MODE 0: out-of-place kick        Pout = Pin - eps_k F(U)                (updateE)
// MODE 1: fused kick + drift       P -= eps_k F(U); Uout = exp(i eps_d P) U
//
// Work mapping (site tiles): a CTA of 32*min(D,4) threads owns 32 consecutive
// sites; warp w handles directions w, w+4, ... of those sites.  All D
// directions of a site neighbourhood are therefore processed by one CTA at the
// same time, so the neighbour links each staple needs are fetched from DRAM
// once and then served from L1/L2 to the other warps, instead of being
// re-fetched in D separate direction sweeps.  Each warp still reads 32
// consecutive sites per element.
template <int N, typename T, typename S2, int MODE>
__device__ __forceinline__ void force_link(const Lat& L, const S2* __restrict__ U, const S2* Pin, S2* Pout,
                                           S2* __restrict__ Uout, T eps_k, T eps_d, int order, int reunit, int mu,
                                           int x) {
  Mat<N, T> acc, Ux, W;
  staple_sum<N, T, S2>(acc, U, L, mu, x);
  load(Ux, U, L, mu, x);
  mul_nn(W, Ux, acc);
  Mat<N, T> P;
  load(P, Pin, L, mu, x);
  kick_ta(P, W, eps_k);
  store(Pout, P, L, mu, x);
  if (MODE == 1) {
    Mat<N, T> Tm;
    expi_update(Tm, P, Ux, eps_d, order);
    if (reunit) reunitarise(Tm);
    store(Uout, Tm, L, mu, x);
  }
}

template <int N, typename T, typename S2, int MODE>
__global__ void __launch_bounds__(128) k_force(Lat L, const S2* __restrict__ U, const S2* Pin,
                                               S2* Pout, S2* __restrict__ Uout, T eps_k, T eps_d,
                                               int order, int reunit) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  if (x >= L.V) return;
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5)) force_link<N, T, S2, MODE>(
      L, U, Pin, Pout, Uout, eps_k, eps_d, order, reunit, mu, x);
}

// The same kernel with a tighter register budget for more resident CTAs
// (OCC = 1: 6 per SM in FP32, 3 in FP64; OCC = 2: 7 / 4); the autotuner picks
// the budget where it is faster.
template <int N, typename T, typename S2, int MODE, int OCC = 1>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 5 + OCC : 2 + OCC)
    k_force_occ(Lat L, const S2* __restrict__ U, const S2* Pin, S2* Pout, S2* __restrict__ Uout, T eps_k, T eps_d,
                int order, int reunit) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  if (x >= L.V) return;
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5))
    force_link<N, T, S2, MODE>(L, U, Pin, Pout, Uout, eps_k, eps_d, order, reunit, mu, x);
}

// In-place drift: U <- exp(i eps P) U (updateUandcopyDown; the copy pi = Pi is
// done by the caller).  Optionally reunitarises.
template <int N, typename T, typename S2>
__global__ void __launch_bounds__(128) k_drift(Lat L, S2* __restrict__ U, const S2* __restrict__ P, T eps, int order,
                                               int reunit) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.V * L.D) return;
  const int mu = (int)(t / L.V);
  const int x = (int)(t - (long)mu * L.V);
  Mat<N, T> Ux, Pm, Tm;
  load(Ux, U, L, mu, x);
  load(Pm, P, L, mu, x);
  expi_update(Tm, Pm, Ux, eps, order);
  if (reunit) reunitarise(Tm);
  store(U, Tm, L, mu, x);
}

// In-place reunitarisation of every link.
template <int N, typename T, typename S2>
__global__ void __launch_bounds__(128) k_reunit(Lat L, S2* __restrict__ U) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.V * L.D) return;
  const int mu = (int)(t / L.V);
  const int x = (int)(t - (long)mu * L.V);
  Mat<N, T> Ux;
  load(Ux, U, L, mu, x);
  reunitarise(Ux);
  store(U, Ux, L, mu, x);
}

}  // namespace small
}  // namespace askja
