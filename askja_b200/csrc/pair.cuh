// FP32 SU(3) fused kick+drift with two links per thread in packed f32x2
// arithmetic (FFMA2 / FMUL2 / FADD2 of sm_100).
//
// A thread owns the links (mu, s) and (mu, s+1), s even: two sites adjacent
// along the fastest lattice direction.  Every register pair holds one real
// number of both links (.x site s, .y site s+1), so each floating-point
// instruction does the work of two.  For the length of an MD loop the link
// and momentum fields are kept in the site-pair layout: the canonical blocked
// layout (common.cuh) with every 16-byte group of two adjacent sites' complex
// numbers (re_s, im_s, re_s+1, im_s+1) stored as (re_s, re_s+1, im_s, im_s+1);
// one 16-byte load then fills two register pairs with no moves.  k_pair_swap
// converts in place in either direction (the permutation is an involution).
//
// Neighbours across any direction but the fastest are again aligned pairs
// (every other stride is a multiple of the even extent n[D-1]); across the
// fastest direction they straddle two pairs and are loaded per site.
//
// A complex product needs one subtraction per real or imaginary part and the
// packed instructions have no free operand negation, so each output number is
// summed in two chains, P (added terms) and Q (subtracted terms), joined by
// fma(Q, -1, P): an exact negation and a single rounding.
//
// Physics as small::k_force (sun.cpp:672-790, sunmat.h:200-248, 355-371):
// staple force, P -= eps F, U' = exp(i eps P) U summed to Taylor order
// `order` through Cayley-Hamilton, optional reunitarisation.  Only the order of
// the FP32 sums differs from the scalar kernel.
#pragma once

#include "common.cuh"

namespace askja {
namespace pair {

struct c2 {
  float2 re, im;
};
struct M3 {
  c2 a[3][3];
};
// the two sites of a pair position: a in .x, b in .y
struct Pr {
  int a, b;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// p - q with one rounding
__device__ __forceinline__ float2 sub2(float2 p, float2 q) { return __ffma2_rn(q, f2(-1.f, -1.f), p); }

// sum_k op(a_k) op(b_k) (+ acc), op = complex conjugate where CA / CB
template <bool CA, bool CB, bool ACC>
__device__ __forceinline__ c2 dot3(const c2 (&a)[3], const c2 (&b)[3], const c2& acc) {
  c2 r;
  // real part: + ar br, and ai bi added when exactly one side is conjugated
  float2 p = ACC ? fma2(a[0].re, b[0].re, acc.re) : mul2(a[0].re, b[0].re);
  p = fma2(a[1].re, b[1].re, p);
  p = fma2(a[2].re, b[2].re, p);
  if constexpr (CA != CB) {
#pragma unroll
    for (int k = 0; k < 3; k++) p = fma2(a[k].im, b[k].im, p);
    r.re = p;
  } else {
    float2 q = mul2(a[0].im, b[0].im);
    q = fma2(a[1].im, b[1].im, q);
    q = fma2(a[2].im, b[2].im, q);
    r.re = sub2(p, q);
  }
  // imaginary part: ar bi (subtracted if CB), ai br (subtracted if CA)
  if constexpr (!CA && !CB) {
    float2 s = ACC ? fma2(a[0].re, b[0].im, acc.im) : mul2(a[0].re, b[0].im);
    s = fma2(a[1].re, b[1].im, s);
    s = fma2(a[2].re, b[2].im, s);
#pragma unroll
    for (int k = 0; k < 3; k++) s = fma2(a[k].im, b[k].re, s);
    r.im = s;
  } else if constexpr (CA && CB) {
    float2 q = mul2(a[0].re, b[0].im);
    q = fma2(a[1].re, b[1].im, q);
    q = fma2(a[2].re, b[2].im, q);
#pragma unroll
    for (int k = 0; k < 3; k++) q = fma2(a[k].im, b[k].re, q);
    r.im = ACC ? sub2(acc.im, q) : mul2(q, f2(-1.f, -1.f));
  } else {
    // CB: + ai br - ar bi;  CA: + ar bi - ai br
    float2 s, q;
    if constexpr (CB) {
      s = ACC ? fma2(a[0].im, b[0].re, acc.im) : mul2(a[0].im, b[0].re);
      s = fma2(a[1].im, b[1].re, s);
      s = fma2(a[2].im, b[2].re, s);
      q = mul2(a[0].re, b[0].im);
      q = fma2(a[1].re, b[1].im, q);
      q = fma2(a[2].re, b[2].im, q);
    } else {
      s = ACC ? fma2(a[0].re, b[0].im, acc.im) : mul2(a[0].re, b[0].im);
      s = fma2(a[1].re, b[1].im, s);
      s = fma2(a[2].re, b[2].im, s);
      q = mul2(a[0].im, b[0].re);
      q = fma2(a[1].im, b[1].re, q);
      q = fma2(a[2].im, b[2].re, q);
    }
    r.im = sub2(s, q);
  }
  return r;
}

// C = opA(A) opB(B) (+ C when ACC), opX = dagger where DX.  C must not alias
// A or B.
template <bool DA, bool DB, bool ACC>
__device__ __forceinline__ void mm(M3& C, const M3& A, const M3& B) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      c2 a[3], b[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        a[k] = DA ? A.a[k][i] : A.a[i][k];
        b[k] = DB ? B.a[j][k] : B.a[k][j];
      }
      C.a[i][j] = dot3<DA, DB, ACC>(a, b, C.a[i][j]);
    }
}

__device__ __forceinline__ void zero(M3& m) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      m.a[i][j].re = f2(0.f, 0.f);
      m.a[i][j].im = f2(0.f, 0.f);
    }
}

// whether (a, b) is an aligned pair: one 16-byte group of the layout
__device__ __forceinline__ bool aligned(const Pr& p) { return p.b == p.a + 1 && !(p.a & 1); }

// float index of the real part of element 0 of site s (element e: + 64 e;
// imaginary part: + 2)
__device__ __forceinline__ size_t sbase(const Lat& L, int d, int s) {
  return 2 * ((((size_t)d * L.B + (s >> 5)) * 9) * 32 + (s & 30)) + (s & 1);
}
// float4 index of element 0 of the aligned pair starting at s (element e: + 16 e)
__device__ __forceinline__ size_t pbase(const Lat& L, int d, int s) {
  return (((size_t)d * L.B + (s >> 5)) * 9) * 16 + ((s & 31) >> 1);
}

// links of a read-only field (non-coherent loads)
__device__ __forceinline__ void load_ro(M3& m, const float* __restrict__ f, const Lat& L, int d, const Pr& p) {
  if (aligned(p)) {
    const float4* q = reinterpret_cast<const float4*>(f) + pbase(L, d, p.a);
#pragma unroll
    for (int e = 0; e < 9; e++) {
      const float4 v = __ldg(q + 16 * e);
      m.a[e / 3][e % 3].re = f2(v.x, v.y);
      m.a[e / 3][e % 3].im = f2(v.z, v.w);
    }
  } else {
    const float* qa = f + sbase(L, d, p.a);
    const float* qb = f + sbase(L, d, p.b);
#pragma unroll
    for (int e = 0; e < 9; e++) {
      m.a[e / 3][e % 3].re = f2(__ldg(qa + 64 * e), __ldg(qb + 64 * e));
      m.a[e / 3][e % 3].im = f2(__ldg(qa + 64 * e + 2), __ldg(qb + 64 * e + 2));
    }
  }
}

// own (aligned) pair of a field this thread also writes
__device__ __forceinline__ void load_own(M3& m, const float* f, const Lat& L, int d, int s) {
  const float4* q = reinterpret_cast<const float4*>(f) + pbase(L, d, s);
#pragma unroll
  for (int e = 0; e < 9; e++) {
    const float4 v = q[16 * e];
    m.a[e / 3][e % 3].re = f2(v.x, v.y);
    m.a[e / 3][e % 3].im = f2(v.z, v.w);
  }
}

__device__ __forceinline__ void store_own(float* f, const M3& m, const Lat& L, int d, int s) {
  float4* q = reinterpret_cast<float4*>(f) + pbase(L, d, s);
#pragma unroll
  for (int e = 0; e < 9; e++) {
    const c2& z = m.a[e / 3][e % 3];
    q[16 * e] = make_float4(z.re.x, z.re.y, z.im.x, z.im.y);
  }
}

// neighbours of both sites one step along d; an aligned pair stays aligned
// across every direction but the fastest (n[D-1] even)
__device__ __forceinline__ Pr step(const Lat& L, const Pr& p, int d, bool plus) {
  Pr q;
  q.a = plus ? nb_plus(L, d, p.a) : nb_minus(L, d, p.a);
  if (d != L.D - 1 && aligned(p))
    q.b = q.a + 1;
  else
    q.b = plus ? nb_plus(L, d, p.b) : nb_minus(L, d, p.b);
  return q;
}

// staple sum without the leading U_mu(x) (as small::staple_sum); the lower
// staple's first two links are formed as U_mu(x-nu) U_nu(x+mu-nu) and used
// daggered
__device__ __forceinline__ void staple_sum(M3& acc, const float* __restrict__ U, const Lat& L, int mu, const Pr& x) {
  zero(acc);
  const Pr xpmu = step(L, x, mu, true);
#pragma unroll 1
  for (int nu = 0; nu < L.D; nu++) {
    if (nu == mu) continue;
    const Pr xpnu = step(L, x, nu, true);
    const Pr xmnu = step(L, x, nu, false);
    const Pr xpmu_mnu = step(L, xpmu, nu, false);
    {
      M3 A, B, T1;
      load_ro(A, U, L, nu, xpmu);
      load_ro(B, U, L, mu, xpnu);
      mm<false, true, false>(T1, A, B);  // U_nu(x+mu) U_mu(x+nu)^dag
      load_ro(A, U, L, nu, x);
      mm<false, true, true>(acc, T1, A);  // ... U_nu(x)^dag
    }
    {
      M3 A, B, T1;
      load_ro(A, U, L, nu, xpmu_mnu);
      load_ro(B, U, L, mu, xmnu);
      mm<false, false, false>(T1, B, A);  // U_mu(x-nu) U_nu(x+mu-nu)
      load_ro(A, U, L, nu, xmnu);
      mm<true, false, true>(acc, T1, A);  // acc += T1^dag U_nu(x-nu)
    }
  }
}

// P <- P - eps Adjoint(W), Adjoint(W) = -i/2 [(W - W^dag) - Tr(W - W^dag)/3]
__device__ __forceinline__ void kick_ta(M3& P, const M3& W, float eps) {
  const float2 third = f2(1.f / 3.f, 1.f / 3.f);
  const float2 trim = mul2(add2(add2(W.a[0][0].im, W.a[1][1].im), W.a[2][2].im), third);
  const float2 me = f2(-eps, -eps), mh = f2(-0.5f * eps, -0.5f * eps), ph = f2(0.5f * eps, 0.5f * eps);
#pragma unroll
  for (int i = 0; i < 3; i++) P.a[i][i].re = fma2(me, sub2(W.a[i][i].im, trim), P.a[i][i].re);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i + 1; j < 3; j++) {
      const float2 s = add2(W.a[i][j].im, W.a[j][i].im);
      const float2 d = sub2(W.a[i][j].re, W.a[j][i].re);
      P.a[i][j].re = fma2(mh, s, P.a[i][j].re);
      P.a[j][i].re = fma2(mh, s, P.a[j][i].re);
      P.a[i][j].im = fma2(ph, d, P.a[i][j].im);
      P.a[j][i].im = fma2(mh, d, P.a[j][i].im);
    }
}

__device__ __forceinline__ c2 cmul(const c2& a, const c2& b) {
  c2 r;
  r.re = sub2(mul2(a.re, b.re), mul2(a.im, b.im));
  r.im = fma2(a.im, b.re, mul2(a.re, b.im));
  return r;
}
// a b - c d
__device__ __forceinline__ c2 cmul_sub(const c2& a, const c2& b, const c2& c, const c2& d) {
  c2 r;
  r.re = sub2(fma2(c.im, d.im, mul2(a.re, b.re)), fma2(c.re, d.re, mul2(a.im, b.im)));
  r.im = sub2(fma2(a.im, b.re, mul2(a.re, b.im)), fma2(c.im, d.re, mul2(c.re, d.im)));
  return r;
}

// Tm <- sum_{k<=order} X^k/k! Ux, X = i eps P, through Cayley-Hamilton
// (small::expi_times_ch restated for pairs)
__device__ __forceinline__ void expi_times_ch(M3& Tm, const M3& P, const M3& Ux, float eps, int order) {
  const float2 pe = f2(eps, eps), me = f2(-eps, -eps);
  M3 X;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      X.a[i][j].re = mul2(me, P.a[i][j].im);
      X.a[i][j].im = mul2(pe, P.a[i][j].re);
    }
  c2 tr;
  tr.re = add2(add2(X.a[0][0].re, X.a[1][1].re), X.a[2][2].re);
  tr.im = add2(add2(X.a[0][0].im, X.a[1][1].im), X.a[2][2].im);
  M3 X2;
  mm<false, false, false>(X2, X, X);
  c2 tr2;
  tr2.re = add2(add2(X2.a[0][0].re, X2.a[1][1].re), X2.a[2][2].re);
  tr2.im = add2(add2(X2.a[0][0].im, X2.a[1][1].im), X2.a[2][2].im);
  // c1 = ((tr X)^2 - tr X^2) / 2, c0 = det X; X^3 = tr X X^2 - c1 X + c0 1
  const float2 half = f2(0.5f, 0.5f);
  c2 c1 = cmul(tr, tr);
  c1.re = mul2(half, sub2(c1.re, tr2.re));
  c1.im = mul2(half, sub2(c1.im, tr2.im));
  const c2 m0 = cmul_sub(X.a[1][1], X.a[2][2], X.a[1][2], X.a[2][1]);
  const c2 m1 = cmul_sub(X.a[1][0], X.a[2][2], X.a[1][2], X.a[2][0]);
  const c2 m2 = cmul_sub(X.a[1][0], X.a[2][1], X.a[1][1], X.a[2][0]);
  c2 c0 = cmul_sub(X.a[0][0], m0, X.a[0][1], m1);
  c0.re = sub2(fma2(X.a[0][2].re, m2.re, c0.re), mul2(X.a[0][2].im, m2.im));
  c0.im = fma2(X.a[0][2].im, m2.re, fma2(X.a[0][2].re, m2.im, c0.im));
  const float2 one = f2(1.f, 1.f), zz = f2(0.f, 0.f);
  c2 al = {one, zz}, be = {zz, zz}, ga = {zz, zz};  // X^0
  c2 sa = al, sb = be, sc = ga;
  float f = 1.f;
#pragma unroll
  for (int k = 1; k <= 8; k++) {  // order <= 8; unrolled so that 1/k! is a constant
    if (k > order) break;
    // X^k = ga c0 1 + (al - ga c1) X + (be + ga tr) X^2  (coefficients of X^(k-1))
    const c2 nal = cmul(ga, c0);
    c2 nbe, nga;
    nbe.re = sub2(fma2(ga.im, c1.im, al.re), mul2(ga.re, c1.re));
    nbe.im = sub2(al.im, fma2(ga.im, c1.re, mul2(ga.re, c1.im)));
    nga.re = sub2(fma2(ga.re, tr.re, be.re), mul2(ga.im, tr.im));
    nga.im = fma2(ga.im, tr.re, fma2(ga.re, tr.im, be.im));
    al = nal;
    be = nbe;
    ga = nga;
    f = f * (1.f / k);
    const float2 ff = f2(f, f);
    sa.re = fma2(ff, al.re, sa.re);
    sa.im = fma2(ff, al.im, sa.im);
    sb.re = fma2(ff, be.re, sb.re);
    sb.im = fma2(ff, be.im, sb.im);
    sc.re = fma2(ff, ga.re, sc.re);
    sc.im = fma2(ff, ga.im, sc.im);
  }
  M3 E;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const c2& x = X.a[i][j];
      const c2& y = X2.a[i][j];
      float2 p = i == j ? fma2(sb.re, x.re, sa.re) : mul2(sb.re, x.re);
      p = fma2(sc.re, y.re, p);
      const float2 q = fma2(sc.im, y.im, mul2(sb.im, x.im));
      float2 s = i == j ? fma2(sb.re, x.im, sa.im) : mul2(sb.re, x.im);
      s = fma2(sb.im, x.re, s);
      s = fma2(sc.re, y.im, s);
      s = fma2(sc.im, y.re, s);
      E.a[i][j].re = sub2(p, q);
      E.a[i][j].im = s;
    }
  mm<false, false, false>(Tm, E, Ux);
}

__device__ __forceinline__ float2 rsqrt2(float2 n) { return f2(rsqrtf(n.x), rsqrtf(n.y)); }

// Project onto SU(3): Gram-Schmidt of rows 0 and 1, row 2 = conj(r0 x r1)
// (small::reunitarise for N = 3)
__device__ __forceinline__ void reunitarise(M3& M) {
  c2* r0 = M.a[0];
  c2* r1 = M.a[1];
  float2 n = mul2(r0[0].re, r0[0].re);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (k) n = fma2(r0[k].re, r0[k].re, n);
    n = fma2(r0[k].im, r0[k].im, n);
  }
  float2 inv = rsqrt2(n);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    r0[k].re = mul2(r0[k].re, inv);
    r0[k].im = mul2(r0[k].im, inv);
  }
  const c2 a[3] = {r0[0], r0[1], r0[2]};
  const c2 b[3] = {r1[0], r1[1], r1[2]};
  const c2 pr = dot3<true, false, false>(a, b, a[0]);  // <r0, r1>
  const float2 m1 = f2(-1.f, -1.f);
  const float2 npr_re = mul2(pr.re, m1), npr_im = mul2(pr.im, m1);
#pragma unroll
  for (int k = 0; k < 3; k++) {  // r1 -= pr r0
    r1[k].re = fma2(pr.im, r0[k].im, fma2(npr_re, r0[k].re, r1[k].re));
    r1[k].im = fma2(npr_im, r0[k].re, fma2(npr_re, r0[k].im, r1[k].im));
  }
  n = mul2(r1[0].re, r1[0].re);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (k) n = fma2(r1[k].re, r1[k].re, n);
    n = fma2(r1[k].im, r1[k].im, n);
  }
  inv = rsqrt2(n);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    r1[k].re = mul2(r1[k].re, inv);
    r1[k].im = mul2(r1[k].im, inv);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    // c = r0[k1] r1[k2] - r0[k2] r1[k1]; row 2 = conj(c)
    const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
    const c2& a1 = r0[k1];
    const c2& b2 = r1[k2];
    const c2& a2 = r0[k2];
    const c2& b1 = r1[k1];
    M.a[2][k].re = sub2(fma2(a2.im, b1.im, mul2(a1.re, b2.re)), fma2(a2.re, b1.re, mul2(a1.im, b2.im)));
    M.a[2][k].im = sub2(fma2(a2.im, b1.re, mul2(a2.re, b1.im)), fma2(a1.im, b2.re, mul2(a1.re, b2.im)));
  }
}

// One MD step for the link pairs of a 64-site tile: P -= eps_k F(U);
// Uout = exp(i eps_d P) U.  CTA = 32 pairs x one warp per direction (warp w
// takes directions w, w+4, ...), so the neighbour links of the tile are
// fetched from DRAM once for all directions.  Fields in the site-pair layout.
// OCC 0: 3 resident CTAs per SM (168 registers, no spills); OCC 1: 4 (128
// registers, a few spilled to local memory).
template <int OCC>
__global__ void __launch_bounds__(128, 3 + OCC) k_force_pair(Lat L, const float2* __restrict__ U, float2* P,
                                                             float2* __restrict__ Uout, float eps_k, float eps_d,
                                                             int order, int reunit) {
  const int s = 2 * (blockIdx.x * 32 + (threadIdx.x & 31));
  if (s >= L.V) return;
  const Pr x = {s, s + 1};
  const float* u = reinterpret_cast<const float*>(U);
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5)) {
    M3 acc, Ux, W;
    staple_sum(acc, u, L, mu, x);
    load_ro(Ux, u, L, mu, x);
    mm<false, false, false>(W, Ux, acc);
    M3 Pm;
    load_own(Pm, reinterpret_cast<float*>(P), L, mu, s);
    kick_ta(Pm, W, eps_k);
    store_own(reinterpret_cast<float*>(P), Pm, L, mu, s);
    M3 Tm;
    expi_times_ch(Tm, Pm, Ux, eps_d, order);
    if (reunit) reunitarise(Tm);
    store_own(reinterpret_cast<float*>(Uout), Tm, L, mu, s);
  }
}

// canonical <-> site-pair layout, in place: swap the middle two floats of
// every 16-byte group
static __global__ void __launch_bounds__(256) k_pair_swap(float4* f, long n4) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long)gridDim.x * blockDim.x) {
    const float4 v = f[i];
    f[i] = make_float4(v.x, v.z, v.y, v.w);
  }
}

}  // namespace pair
}  // namespace askja
