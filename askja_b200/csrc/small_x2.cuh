// FP32 small-NC fused kick+drift with two links per thread in packed f32x2
// arithmetic (sm_100 FFMA2/FADD2/FMUL2).  Each register pair holds the same
// matrix element of two links -- sites x and x+32 of a 64-site tile, same
// direction -- so every floating-point instruction of the scalar kernel
// (small.cuh) becomes one packed instruction for both links, with no operand
// shuffling.  FFMA2 has the same FLOP rate as FFMA on B200 (measured 73 vs
// 70 TFLOP/s) but needs half the issue slots, and the scalar kernel is bound
// by instruction issue.
//
// Same physics and rounding behaviour per link as small::k_force (sun.cpp:
// 672-790, sunmat.h:200-248, 355-371); only the instruction packing differs.
#pragma once

#include "common.cuh"

namespace askja {
namespace x2 {

struct c2 {
  float2 re, im;  // .x: link of site x, .y: link of site x+32
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ c2 z2() {
  c2 z;
  z.re = f2(0.f, 0.f);
  z.im = f2(0.f, 0.f);
  return z;
}
// acc += a b
__device__ __forceinline__ void mac(c2& acc, const c2& a, const c2& b) {
  acc.re = __ffma2_rn(a.re, b.re, acc.re);
  acc.re = __ffma2_rn(neg(a.im), b.im, acc.re);
  acc.im = __ffma2_rn(a.re, b.im, acc.im);
  acc.im = __ffma2_rn(a.im, b.re, acc.im);
}
// acc += a conj(b)
__device__ __forceinline__ void mac_nc(c2& acc, const c2& a, const c2& b) {
  acc.re = __ffma2_rn(a.re, b.re, acc.re);
  acc.re = __ffma2_rn(a.im, b.im, acc.re);
  acc.im = __ffma2_rn(a.im, b.re, acc.im);
  acc.im = __ffma2_rn(neg(a.re), b.im, acc.im);
}
// acc += conj(a) conj(b)
__device__ __forceinline__ void mac_cc(c2& acc, const c2& a, const c2& b) {
  acc.re = __ffma2_rn(a.re, b.re, acc.re);
  acc.re = __ffma2_rn(neg(a.im), b.im, acc.re);
  acc.im = __ffma2_rn(neg(a.re), b.im, acc.im);
  acc.im = __ffma2_rn(neg(a.im), b.re, acc.im);
}
// acc += conj(a) b
__device__ __forceinline__ void mac_cn(c2& acc, const c2& a, const c2& b) {
  acc.re = __ffma2_rn(a.re, b.re, acc.re);
  acc.re = __ffma2_rn(a.im, b.im, acc.re);
  acc.im = __ffma2_rn(a.re, b.im, acc.im);
  acc.im = __ffma2_rn(neg(a.im), b.re, acc.im);
}

template <int N>
struct M {
  c2 a[N][N];
};

template <int N>
__device__ __forceinline__ void load(M<N>& m, const float2* __restrict__ f, const Lat& L, int d, int s0, int s1) {
  const float2* p0 = f + ((size_t)d * L.B + (s0 >> 5)) * (N * N * 32) + (s0 & 31);
  const float2* p1 = f + ((size_t)d * L.B + (s1 >> 5)) * (N * N * 32) + (s1 & 31);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      const float2 v0 = p0[(i * N + j) * 32], v1 = p1[(i * N + j) * 32];
      m.a[i][j].re = f2(v0.x, v1.x);
      m.a[i][j].im = f2(v0.y, v1.y);
    }
}

template <int N>
__device__ __forceinline__ void store(float2* __restrict__ f, const M<N>& m, const Lat& L, int d, int s0, int s1,
                                      bool ok1) {
  float2* p0 = f + ((size_t)d * L.B + (s0 >> 5)) * (N * N * 32) + (s0 & 31);
  float2* p1 = f + ((size_t)d * L.B + (s1 >> 5)) * (N * N * 32) + (s1 & 31);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      p0[(i * N + j) * 32] = f2(m.a[i][j].re.x, m.a[i][j].im.x);
      if (ok1) p1[(i * N + j) * 32] = f2(m.a[i][j].re.y, m.a[i][j].im.y);
    }
}

template <int N>
__device__ __forceinline__ void zero(M<N>& m) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) m.a[i][j] = z2();
}

// staple sum without the leading U_mu(x), for two sites at once
template <int N>
__device__ __forceinline__ void staple_sum(M<N>& acc, const float2* __restrict__ U, const Lat& L, int mu, int x0,
                                           int x1) {
  zero(acc);
  const int p0 = nb_plus(L, mu, x0), p1 = nb_plus(L, mu, x1);
  for (int nu = 0; nu < L.D; nu++) {
    if (nu == mu) continue;
    const int a0 = nb_plus(L, nu, x0), a1 = nb_plus(L, nu, x1);
    const int b0 = nb_minus(L, nu, x0), b1 = nb_minus(L, nu, x1);
    const int c0 = nb_minus(L, nu, p0), c1 = nb_minus(L, nu, p1);
    {
      M<N> A, B, T1;
      load(A, U, L, nu, p0, p1);
      load(B, U, L, mu, a0, a1);
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          c2 s = z2();
#pragma unroll
          for (int k = 0; k < N; k++) mac_nc(s, A.a[i][k], B.a[j][k]);
          T1.a[i][j] = s;
        }
      load(A, U, L, nu, x0, x1);
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++)
#pragma unroll
          for (int k = 0; k < N; k++) mac_nc(acc.a[i][j], T1.a[i][k], A.a[j][k]);
    }
    {
      M<N> A, B, T1;
      load(A, U, L, nu, c0, c1);
      load(B, U, L, mu, b0, b1);
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          c2 s = z2();
#pragma unroll
          for (int k = 0; k < N; k++) mac_cc(s, A.a[k][i], B.a[j][k]);
          T1.a[i][j] = s;
        }
      load(A, U, L, nu, b0, b1);
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++)
#pragma unroll
          for (int k = 0; k < N; k++) mac(acc.a[i][j], T1.a[i][k], A.a[k][j]);
    }
  }
}

// last row of an SU(N) matrix from the others (rows 0..N-2 orthonormal)
template <int N>
__device__ __forceinline__ void complete_last_row(M<N>& m);

template <>
__device__ __forceinline__ void complete_last_row<2>(M<2>& m) {
  m.a[1][0].re = neg(m.a[0][1].re);
  m.a[1][0].im = m.a[0][1].im;
  m.a[1][1].re = m.a[0][0].re;
  m.a[1][1].im = neg(m.a[0][0].im);
}

template <>
__device__ __forceinline__ void complete_last_row<3>(M<3>& m) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
    c2 c = z2();
    mac(c, m.a[0][k1], m.a[1][k2]);
    c2 nb;
    nb.re = neg(m.a[1][k1].re);
    nb.im = neg(m.a[1][k1].im);
    mac(c, m.a[0][k2], nb);
    m.a[2][k].re = c.re;
    m.a[2][k].im = neg(c.im);
  }
}

template <>
__device__ __forceinline__ void complete_last_row<4>(M<4>& m) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int cols[3] = {k == 0 ? 1 : 0, k <= 1 ? 2 : 1, k <= 2 ? 3 : 2};
    c2 det = z2();
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const int q1 = (p + 1) % 3, q2 = (p + 2) % 3;
      c2 t = z2();
      mac(t, m.a[1][cols[q1]], m.a[2][cols[q2]]);
      c2 nb;
      nb.re = neg(m.a[2][cols[q1]].re);
      nb.im = neg(m.a[2][cols[q1]].im);
      mac(t, m.a[1][cols[q2]], nb);
      mac(det, m.a[0][cols[p]], t);
    }
    const float sg = ((3 + k) & 1) ? -1.f : 1.f;
    m.a[3][k].re = __fmul2_rn(f2(sg, sg), det.re);
    m.a[3][k].im = __fmul2_rn(f2(-sg, -sg), det.im);
  }
}

template <int N>
__device__ __forceinline__ void reunitarise(M<N>& m) {
#pragma unroll
  for (int r = 0; r < N - 1; r++) {
#pragma unroll
    for (int q = 0; q < r; q++) {
      c2 pr = z2();
#pragma unroll
      for (int k = 0; k < N; k++) mac_cn(pr, m.a[q][k], m.a[r][k]);
      c2 npr;
      npr.re = neg(pr.re);
      npr.im = neg(pr.im);
#pragma unroll
      for (int k = 0; k < N; k++) mac(m.a[r][k], npr, m.a[q][k]);
    }
    float2 nrm = f2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < N; k++) {
      nrm = __ffma2_rn(m.a[r][k].re, m.a[r][k].re, nrm);
      nrm = __ffma2_rn(m.a[r][k].im, m.a[r][k].im, nrm);
    }
    const float2 inv = f2(rsqrtf(nrm.x), rsqrtf(nrm.y));
#pragma unroll
    for (int k = 0; k < N; k++) {
      m.a[r][k].re = __fmul2_rn(m.a[r][k].re, inv);
      m.a[r][k].im = __fmul2_rn(m.a[r][k].im, inv);
    }
  }
  complete_last_row<N>(m);
}

// MODE 0: out-of-place kick; MODE 1: fused kick + drift (see small::k_force).
// CTA of 128 threads = 64 sites x 4 direction warps (warps loop when D > 4).
template <int N, int MODE>
__device__ __forceinline__ void force_link(const Lat& L, const float2* __restrict__ U, const float2* Pin, float2* Pout,
                                           float2* __restrict__ Uout, float eps_k, float eps_d, int order, int reunit,
                                           int mu, int x0, int x1, bool ok1) {
  M<N> acc;
  staple_sum<N>(acc, U, L, mu, x0, x1);
  M<N> Ux, W;
  load(Ux, U, L, mu, x0, x1);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      c2 s = z2();
#pragma unroll
      for (int k = 0; k < N; k++) mac(s, Ux.a[i][k], acc.a[k][j]);
      W.a[i][j] = s;
    }
  M<N> P;
  load(P, Pin, L, mu, x0, x1);
  // P -= eps Adjoint(W)
  float2 trim = f2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < N; k++) trim = __fadd2_rn(trim, W.a[k][k].im);
  trim = __fmul2_rn(trim, f2(1.f / N, 1.f / N));
  const float2 mek = f2(-eps_k, -eps_k), hek = f2(-0.5f * eps_k, -0.5f * eps_k);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      if (i == j) {
        P.a[i][i].re = __ffma2_rn(mek, __fadd2_rn(W.a[i][i].im, neg(trim)), P.a[i][i].re);
      } else {
        P.a[i][j].re = __ffma2_rn(hek, __fadd2_rn(W.a[i][j].im, W.a[j][i].im), P.a[i][j].re);
        P.a[i][j].im = __ffma2_rn(neg(hek), __fadd2_rn(W.a[i][j].re, neg(W.a[j][i].re)), P.a[i][j].im);
      }
    }
  store(Pout, P, L, mu, x0, x1, ok1);
  if (MODE == 1) {
    // Tm <- U + (i eps/n) P Tm, n = order..1
    M<N> Tm = Ux;
    for (int n = order; n >= 1; n--) {
      const float c = eps_d / (float)n;
      const float2 cp = f2(c, c), cm = f2(-c, -c);
      M<N> Y;
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
          c2 s = z2();
#pragma unroll
          for (int k = 0; k < N; k++) mac(s, P.a[i][k], Tm.a[k][j]);
          // Y = U + i c s
          Y.a[i][j].re = __ffma2_rn(cm, s.im, Ux.a[i][j].re);
          Y.a[i][j].im = __ffma2_rn(cp, s.re, Ux.a[i][j].im);
        }
      Tm = Y;
    }
    if (reunit) reunitarise(Tm);
    store(Uout, Tm, L, mu, x0, x1, ok1);
  }
}

template <int N, int MODE>
__global__ void __launch_bounds__(128) k_force(Lat L, const float2* __restrict__ U, const float2* Pin, float2* Pout,
                                               float2* __restrict__ Uout, float eps_k, float eps_d, int order,
                                               int reunit) {
  const int x0 = blockIdx.x * 64 + (threadIdx.x & 31);
  if (x0 >= L.V) return;
  const bool ok1 = x0 + 32 < L.V;
  const int x1 = ok1 ? x0 + 32 : x0;
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5))
    force_link<N, MODE>(L, U, Pin, Pout, Uout, eps_k, eps_d, order, reunit, mu, x0, x1, ok1);
}

}  // namespace x2
}  // namespace askja
