// Row-per-thread kernels for medium colour number (5 <= NC <= NMAX): a group
// of NC threads owns one link, thread r owns row r of every matrix of the
// staple sum in registers.  Products whose right operand is a stored link read
// it straight from global memory (all NC threads of a group read the same
// element in the same instruction, so L1 serves it as a broadcast); only
// products whose right operand is itself a computed matrix (U_mu * staple sum,
// the Horner recursion, Gram-Schmidt) stage it through a per-group tile of
// shared memory.  Groups of one CTA are lock-stepped by __syncthreads, so every
// thread, valid or not, runs the same barrier sequence.
//
// Same physics and conventions as small.cuh (sun.cpp:672-790, sunmat.h).
#pragma once

#include "common.cuh"

namespace askja {
namespace rows {

// shared memory per group: two NC x NC tiles
template <typename T>
__host__ __device__ inline size_t smem_per_group(int N) {
  return 2 * (size_t)N * N * sizeof(cpx<T>);
}

template <int NMAX, typename T, typename S2>
__device__ __forceinline__ void load_row(cpx<T> (&v)[NMAX], const S2* __restrict__ f, const Lat& L, int d, int s,
                                         int r) {
  const int N = L.N;
#pragma unroll
  for (int c = 0; c < NMAX; c++)
    if (c < N) v[c] = ldc<T>(f + eoff(L, d, r * N + c, s));
}

template <int NMAX, typename T, typename S2>
__device__ __forceinline__ void store_row(S2* __restrict__ f, const cpx<T> (&v)[NMAX], const Lat& L, int d, int s,
                                          int r) {
  const int N = L.N;
#pragma unroll
  for (int c = 0; c < NMAX; c++)
    if (c < N) stc(f + eoff(L, d, r * N + c, s), v[c]);
}

// Modified Gram-Schmidt of rows 0..N-2, then the last row is orthonormalised
// and multiplied by conj(det)/|det| so that det = 1.  Rows live in the
// group's tile S (row-major NxN); S2t is a second tile used for the LU
// determinant.  All threads of the block must call this (it contains barriers).
template <typename T>
__device__ void reunitarise_tile(cpx<T>* S, cpx<T>* S2t, int N, int r, bool act, int* piv_s, cpx<T>* det_s) {
  for (int q = 0; q < N; q++) {
    if (act && r == q) {
      T nrm = T(0);
      for (int k = 0; k < N; k++) nrm = cnorm2_add(S[q * N + k], nrm);
      const T inv = T(1) / sqrt(nrm);
      for (int k = 0; k < N; k++) {
        S[q * N + k].re *= inv;
        S[q * N + k].im *= inv;
      }
    }
    __syncthreads();
    if (act && r > q) {
      cpx<T> pr = czero<T>();
      for (int k = 0; k < N; k++) cmac_cn(pr, S[q * N + k], S[r * N + k]);
      for (int k = 0; k < N; k++) cmsub(S[r * N + k], pr, S[q * N + k]);
    }
    __syncthreads();
  }
  // determinant by LU with partial pivoting on a copy
  if (act)
    for (int k = 0; k < N; k++) S2t[r * N + k] = S[r * N + k];
  if (act && r == 0) {
    *det_s = mkc<T>(T(1), T(0));
  }
  __syncthreads();
  for (int c = 0; c < N; c++) {
    if (act && r == 0) {
      int piv = c;
      T best = T(-1);
      for (int i = c; i < N; i++) {
        const T v = cnorm2_add(S2t[i * N + c], T(0));
        if (v > best) {
          best = v;
          piv = i;
        }
      }
      if (piv != c) {
        for (int k = 0; k < N; k++) {
          const cpx<T> t0 = S2t[c * N + k];
          S2t[c * N + k] = S2t[piv * N + k];
          S2t[piv * N + k] = t0;
        }
        det_s->re = -det_s->re;
        det_s->im = -det_s->im;
      }
      cpx<T> dp = czero<T>();
      cmac(dp, *det_s, S2t[c * N + c]);
      *det_s = dp;
      *piv_s = piv;
    }
    __syncthreads();
    if (act && r > c) {
      const cpx<T> p = S2t[c * N + c];
      const T den = cnorm2_add(p, T(0));
      cpx<T> q = czero<T>();  // a conj(p)
      cmac_nc(q, S2t[r * N + c], p);
      const cpx<T> f = mkc<T>(q.re / den, q.im / den);
      for (int k = c; k < N; k++) cmsub(S2t[r * N + k], f, S2t[c * N + k]);
    }
    __syncthreads();
  }
  if (act && r == N - 1) {
    const cpx<T> d = *det_s;
    const T dn = sqrt(d.re * d.re + d.im * d.im);
    const cpx<T> cph = mkc<T>(d.re / dn, -d.im / dn);
    for (int k = 0; k < N; k++) {
      const cpx<T> x = S[r * N + k];
      S[r * N + k] = mkc<T>(x.re * cph.re - x.im * cph.im, x.re * cph.im + x.im * cph.re);
    }
  }
  __syncthreads();
}

// MODE 0: out-of-place kick  Pout = Pin - eps_k F(U)
// MODE 1: fused kick + drift P -= eps_k F(U); Uout = exp(i eps_d P) U
// The CTA's groups take links link_base, link_base+1, ... in site-major order
// (link = x*D + mu), so the groups of one CTA work on all directions of
// neighbouring sites and share their neighbour links through L1/L2.
template <int NMAX, typename T, typename S2, int MODE>
__device__ __forceinline__ void force_rows(const Lat& L, const S2* __restrict__ U, const S2* Pin, S2* Pout,
                                           S2* __restrict__ Uout, T eps_k, T eps_d, int order, int reunit,
                                           long link_base, unsigned char* smem_raw, int* piv_s, cpx<T>* det_s) {
  constexpr int KU = NMAX <= 16 ? NMAX : 1;
  const int N = L.N;
  const int G = blockDim.x / N;
  const int g = threadIdx.x / N;
  const int r = threadIdx.x - g * N;
  const bool in_group = g < G;
  const long link = link_base + g;
  const bool act = in_group && link < (long)L.V * L.D;
  const int x = act ? (int)(link / L.D) : 0;
  const int mu = act ? (int)(link - (long)x * L.D) : 0;
  cpx<T>* S0 = reinterpret_cast<cpx<T>*>(smem_raw) + (size_t)(in_group ? g : 0) * 2 * N * N;
  cpx<T>* S1 = S0 + N * N;

  cpx<T> acc[NMAX];
#pragma unroll
  for (int c = 0; c < NMAX; c++) acc[c] = czero<T>();

  if (act) {
    const int xpmu = nb_plus(L, mu, x);
    for (int nu = 0; nu < L.D; nu++) {
      if (nu == mu) continue;
      const int xpnu = nb_plus(L, nu, x);
      const int xmnu = nb_minus(L, nu, x);
      const int xpmu_mnu = nb_minus(L, nu, xpmu);
      cpx<T> t[NMAX];
      // upper: t = row r of U_nu(x+mu) U_mu^dag(x+nu)
#pragma unroll
      for (int c = 0; c < NMAX; c++) t[c] = czero<T>();
      for (int k = 0; k < N; k++) {
        const cpx<T> a = ldc<T>(U + eoff(L, nu, r * N + k, xpmu));
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) cmac_nc(t[c], a, ldc<T>(U + eoff(L, mu, c * N + k, xpnu)));
      }
      // acc += t U_nu^dag(x)
#pragma unroll KU
      for (int k = 0; k < NMAX; k++) {
        if (k >= N) break;
        const cpx<T> tk = t[k];
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) cmac_nc(acc[c], tk, ldc<T>(U + eoff(L, nu, c * N + k, x)));
      }
      // lower: t = row r of U_nu^dag(x+mu-nu) U_mu^dag(x-nu)
#pragma unroll
      for (int c = 0; c < NMAX; c++) t[c] = czero<T>();
      for (int k = 0; k < N; k++) {
        const cpx<T> a = ldc<T>(U + eoff(L, nu, k * N + r, xpmu_mnu));  // (A^dag)[r][k] = conj(A[k][r])
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) cmac_cc(t[c], a, ldc<T>(U + eoff(L, mu, c * N + k, xmnu)));
      }
      // acc += t U_nu(x-nu)
#pragma unroll KU
      for (int k = 0; k < NMAX; k++) {
        if (k >= N) break;
        const cpx<T> tk = t[k];
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) cmac(acc[c], tk, ldc<T>(U + eoff(L, nu, k * N + c, xmnu)));
      }
    }
  }
  // W = U_mu(x) * acc  (acc staged through S0)
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) S0[r * N + c] = acc[c];
  }
  __syncthreads();
  cpx<T> w[NMAX];
#pragma unroll
  for (int c = 0; c < NMAX; c++) w[c] = czero<T>();
  if (act) {
    for (int k = 0; k < N; k++) {
      const cpx<T> a = ldc<T>(U + eoff(L, mu, r * N + k, x));
#pragma unroll
      for (int c = 0; c < NMAX; c++)
        if (c < N) cmac(w[c], a, S0[k * N + c]);
    }
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) S1[r * N + c] = w[c];
  }
  __syncthreads();
  // kick with the traceless anti-hermitian part
  cpx<T> p[NMAX];
  if (act) {
    T trim = T(0);
    for (int k = 0; k < N; k++) trim += S1[k * N + k].im;
    trim = trim / T(N);
    load_row<NMAX, T, S2>(p, Pin, L, mu, x, r);
#pragma unroll
    for (int c = 0; c < NMAX; c++) {
      if (c < N) {
        const cpx<T> wrc = w[c];
        const cpx<T> wcr = S1[c * N + r];
        T fr, fi;
        if (c == r) {
          fr = wrc.im - trim;
          fi = T(0);
        } else {
          fr = T(0.5) * (wrc.im + wcr.im);
          fi = T(-0.5) * (wrc.re - wcr.re);
        }
        p[c].re = fma(-eps_k, fr, p[c].re);
        p[c].im = fma(-eps_k, fi, p[c].im);
      }
    }
    store_row<NMAX, T, S2>(Pout, p, L, mu, x, r);
  }
  if (MODE == 1) {
    // drift: T <- U + (X/n) T, X = i eps_d P, T staged through S0
    cpx<T> u[NMAX], tm[NMAX];
    if (act) {
      load_row<NMAX, T, S2>(u, U, L, mu, x, r);
#pragma unroll
      for (int c = 0; c < NMAX; c++) {
        tm[c] = u[c];
        p[c] = mkc<T>(-eps_d * p[c].im, eps_d * p[c].re);
      }
    }
    for (int n = order; n >= 1; n--) {
      __syncthreads();
      if (act) {
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) S0[r * N + c] = tm[c];
      }
      __syncthreads();
      if (act) {
        const T inv = T(1) / T(n);
        cpx<T> s[NMAX];
#pragma unroll
        for (int c = 0; c < NMAX; c++) s[c] = czero<T>();
#pragma unroll KU
        for (int k = 0; k < NMAX; k++) {
          if (k >= N) break;
          const cpx<T> xk = p[k];
#pragma unroll
          for (int c = 0; c < NMAX; c++)
            if (c < N) cmac(s[c], xk, S0[k * N + c]);
        }
#pragma unroll
        for (int c = 0; c < NMAX; c++) tm[c] = mkc<T>(fma(s[c].re, inv, u[c].re), fma(s[c].im, inv, u[c].im));
      }
    }
    if (reunit) {
      __syncthreads();
      if (act) {
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) S0[r * N + c] = tm[c];
      }
      __syncthreads();
      reunitarise_tile<T>(S0, S1, N, r, act, &piv_s[in_group ? g : 0], &det_s[in_group ? g : 0]);
      if (act) {
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) tm[c] = S0[r * N + c];
      }
    }
    if (act) store_row<NMAX, T, S2>(Uout, tm, L, mu, x, r);
  }
}

template <int NMAX, typename T, typename S2, int MODE>
__global__ void k_force(Lat L, const S2* __restrict__ U, const S2* Pin, S2* Pout, S2* __restrict__ Uout, T eps_k,
                        T eps_d, int order, int reunit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<T> det_s[64];
  force_rows<NMAX, T, S2, MODE>(L, U, Pin, Pout, Uout, eps_k, eps_d, order, reunit,
                                (long)blockIdx.x * (blockDim.x / L.N), smem_raw, piv_s, det_s);
}

// In-place drift U <- exp(i eps P) U, optional reunitarisation.
template <int NMAX, typename T, typename S2>
__global__ void k_drift(Lat L, S2* __restrict__ U, const S2* __restrict__ P, T eps, int order, int reunit) {
  constexpr int KU = NMAX <= 16 ? NMAX : 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<T> det_s[64];
  const int N = L.N;
  const int G = blockDim.x / N;
  const int g = threadIdx.x / N;
  const int r = threadIdx.x - g * N;
  const bool in_group = g < G;
  const long link = (long)blockIdx.x * G + g;
  const bool act = in_group && link < (long)L.V * L.D;
  const int mu = act ? (int)(link / L.V) : 0;
  const int x = act ? (int)(link - (long)mu * L.V) : 0;
  cpx<T>* S0 = reinterpret_cast<cpx<T>*>(smem_raw) + (size_t)(in_group ? g : 0) * 2 * N * N;
  cpx<T>* S1 = S0 + N * N;
  cpx<T> u[NMAX], tm[NMAX], p[NMAX];
  if (act) {
    load_row<NMAX, T, S2>(u, U, L, mu, x, r);
    load_row<NMAX, T, S2>(p, P, L, mu, x, r);
#pragma unroll
    for (int c = 0; c < NMAX; c++) {
      tm[c] = u[c];
      p[c] = mkc<T>(-eps * p[c].im, eps * p[c].re);
    }
  }
  for (int n = order; n >= 1; n--) {
    __syncthreads();
    if (act) {
#pragma unroll
      for (int c = 0; c < NMAX; c++)
        if (c < N) S0[r * N + c] = tm[c];
    }
    __syncthreads();
    if (act) {
      const T inv = T(1) / T(n);
      cpx<T> s[NMAX];
#pragma unroll
      for (int c = 0; c < NMAX; c++) s[c] = czero<T>();
#pragma unroll KU
      for (int k = 0; k < NMAX; k++) {
        if (k >= N) break;
        const cpx<T> xk = p[k];
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) cmac(s[c], xk, S0[k * N + c]);
      }
#pragma unroll
      for (int c = 0; c < NMAX; c++) tm[c] = mkc<T>(fma(s[c].re, inv, u[c].re), fma(s[c].im, inv, u[c].im));
    }
  }
  if (reunit) {
    __syncthreads();
    if (act) {
#pragma unroll
      for (int c = 0; c < NMAX; c++)
        if (c < N) S0[r * N + c] = tm[c];
    }
    __syncthreads();
    reunitarise_tile<T>(S0, S1, N, r, act, &piv_s[in_group ? g : 0], &det_s[in_group ? g : 0]);
    if (act) {
#pragma unroll
      for (int c = 0; c < NMAX; c++)
        if (c < N) tm[c] = S0[r * N + c];
    }
  }
  if (act) store_row<NMAX, T, S2>(U, tm, L, mu, x, r);
}

// In-place reunitarisation of every link (also used for the Haar hot start).
template <typename T, typename S2>
__global__ void k_reunit(Lat L, S2* __restrict__ U) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<T> det_s[64];
  const int N = L.N;
  const int G = blockDim.x / N;
  const int g = threadIdx.x / N;
  const int r = threadIdx.x - g * N;
  const bool in_group = g < G;
  const long link = (long)blockIdx.x * G + g;
  const bool act = in_group && link < (long)L.V * L.D;
  const int mu = act ? (int)(link / L.V) : 0;
  const int x = act ? (int)(link - (long)mu * L.V) : 0;
  cpx<T>* S0 = reinterpret_cast<cpx<T>*>(smem_raw) + (size_t)(in_group ? g : 0) * 2 * N * N;
  cpx<T>* S1 = S0 + N * N;
  if (act)
    for (int c = 0; c < N; c++) S0[r * N + c] = ldc<T>(U + eoff(L, mu, r * N + c, x));
  __syncthreads();
  reunitarise_tile<T>(S0, S1, N, r, act, &piv_s[in_group ? g : 0], &det_s[in_group ? g : 0]);
  if (act)
    for (int c = 0; c < N; c++) stc(U + eoff(L, mu, r * N + c, x), S0[r * N + c]);
}

}  // namespace rows
}  // namespace askja
