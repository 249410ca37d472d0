// Shared device-side building blocks for the askja B200 engine: complex
// arithmetic on (re, im) pairs, the field layout, the periodic neighbour
// table, Philox4x32-10 and Box-Muller.
//
// Field layout in HBM (all link and momentum fields), blocked by 32 sites:
//   element e = r*NC + c of the matrix on link (site s, direction d) lives at
//   f[((d * B + s/32) * NC*NC + e) * 32 + s%32],   B = ceil(V/32) site blocks,
// as float2 (FP32 mode) or double2 (FP64 mode).  A warp that walks 32
// consecutive sites of one direction reads 32 consecutive complex numbers per
// element -- 256 B (FP32) / 512 B (FP64) per load instruction, coalesced --
// and the NC*NC elements of one link are a fixed 32-element stride apart, so a
// thread addresses a whole matrix from one base pointer with compile-time
// offsets.  Sites V..32B-1 are padding.  Site numbering is the reference's
// (structs.h:130-165): x0 slowest, x_{D-1} fastest.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define ASKJA_MAX_DIM 16

namespace askja {

template <typename T>
struct Storage;
template <>
struct Storage<float> {
  using type = float2;
};
template <>
struct Storage<double> {
  using type = double2;
};

template <typename T>
struct cpx {
  T re, im;
};

template <typename T>
__device__ __forceinline__ cpx<T> mkc(T r, T i) {
  cpx<T> z;
  z.re = r;
  z.im = i;
  return z;
}

template <typename T>
__device__ __forceinline__ cpx<T> czero() {
  return mkc<T>(T(0), T(0));
}

// acc += a * b
template <typename T>
__device__ __forceinline__ void cmac(cpx<T>& acc, const cpx<T>& a, const cpx<T>& b) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(-a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(a.im, b.re, acc.im);
}
// acc -= a * b
template <typename T>
__device__ __forceinline__ void cmsub(cpx<T>& acc, const cpx<T>& a, const cpx<T>& b) {
  acc.re = fma(-a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(-a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
}
// |a|^2 added to s
template <typename T>
__device__ __forceinline__ T cnorm2_add(const cpx<T>& a, T s) {
  return fma(a.im, a.im, fma(a.re, a.re, s));
}
// acc += a * conj(b)
template <typename T>
__device__ __forceinline__ void cmac_nc(cpx<T>& acc, const cpx<T>& a, const cpx<T>& b) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(a.im, b.re, acc.im);
  acc.im = fma(-a.re, b.im, acc.im);
}
// acc += conj(a) * b
template <typename T>
__device__ __forceinline__ void cmac_cn(cpx<T>& acc, const cpx<T>& a, const cpx<T>& b) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
}
// acc += conj(a) * conj(b)
template <typename T>
__device__ __forceinline__ void cmac_cc(cpx<T>& acc, const cpx<T>& a, const cpx<T>& b) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(-a.im, b.im, acc.re);
  acc.im = fma(-a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
}

template <typename T, typename S2>
__device__ __forceinline__ cpx<T> ldc(const S2* __restrict__ p) {
  S2 v = *p;
  return mkc<T>((T)v.x, (T)v.y);
}

template <typename S2, typename T>
__device__ __forceinline__ void stc(S2* __restrict__ p, const cpx<T>& z) {
  S2 v;
  v.x = (decltype(v.x))z.re;
  v.y = (decltype(v.y))z.im;
  *p = v;
}

// Geometry handed to every kernel by value.
struct Lat {
  int V;           // sites
  int B;           // 32-site blocks, ceil(V/32)
  int D;           // dimensions
  int N;           // colours
  const int* nbr;  // nbr[(2*d + 0)*V + s] = s + d^, nbr[(2*d + 1)*V + s] = s - d^
  int n[ASKJA_MAX_DIM];
  int stride[ASKJA_MAX_DIM];
  // sites [r0, r1) enter the plaquette and link sums (r1 = 0: up to V); a
  // domain-decomposed chain counts only the sites it owns, not its halo
  int r0, r1;
};

// whether site s enters the reductions
__host__ __device__ __forceinline__ bool counted(const Lat& L, int s) { return s >= L.r0 && (L.r1 == 0 || s < L.r1); }

__device__ __forceinline__ int nb_plus(const Lat& L, int d, int s) { return __ldg(L.nbr + (size_t)(2 * d) * L.V + s); }
__device__ __forceinline__ int nb_minus(const Lat& L, int d, int s) {
  return __ldg(L.nbr + (size_t)(2 * d + 1) * L.V + s);
}

// Offset of element 0 of the link (d, s); element e is at + 32*e.
__host__ __device__ __forceinline__ size_t mbase(const Lat& L, int d, int s) {
  return ((size_t)d * L.B + (s >> 5)) * (size_t)(L.N * L.N) * 32 + (s & 31);
}

// Offset of element e of the link (d, s).
__host__ __device__ __forceinline__ size_t eoff(const Lat& L, int d, int e, int s) {
  return mbase(L, d, s) + (size_t)e * 32;
}

// Complex elements in one field (padding included).
__host__ __device__ __forceinline__ size_t field_elems(const Lat& L) {
  return (size_t)L.D * L.B * 32 * L.N * L.N;
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ----
struct u32x4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    u32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ double u01(uint32_t w) { return ((double)w + 0.5) * (1.0 / 4294967296.0); }

// Four standard normals from one Philox block: Box-Muller on (u0,u1), (u2,u3).
__device__ __forceinline__ void normals4(u32x4 w, double g[4]) {
  double r0 = sqrt(-2.0 * log(u01(w.x)));
  double r1 = sqrt(-2.0 * log(u01(w.z)));
  double s0, c0, s1, c1;
  sincospi(2.0 * u01(w.y), &s0, &c0);
  sincospi(2.0 * u01(w.w), &s1, &c1);
  g[0] = r0 * c0;
  g[1] = r0 * s0;
  g[2] = r1 * c1;
  g[3] = r1 * s1;
}

// Effective Taylor order of the reference's mexpi (sunmat.h:215-246): orders
// 0..8 are taken as given, anything else falls to the 8th-order default case.
__host__ __device__ __forceinline__ int taylor_order(int level) { return (level >= 0 && level <= 8) ? level : 8; }

}  // namespace askja
