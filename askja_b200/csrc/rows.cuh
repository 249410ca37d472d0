// Row-per-thread kernels for medium colour number (5 <= NC <= NMAX): a group
// of NC threads owns one link, thread r owns row r of every matrix of the
// staple sum in registers.  Every operand of a product -- a stored neighbour
// link or a computed matrix (U_mu * staple sum, the Horner recursion,
// Gram-Schmidt) -- goes through a per-group shared-memory tile; stored links
// are copied in by the whole CTA with coalesced loads (see force_rows), and
// the products read the tiles two complex numbers per load.  Groups of one CTA
// are lock-stepped by __syncthreads, so every
// thread, valid or not, runs the same barrier sequence.  Loops over matrix
// indices are fully unrolled with predicated bodies (no early exits) so the
// row arrays stay in registers.
//
// Same physics and conventions as small.cuh (sun.cpp:672-790, sunmat.h).
#pragma once

#include "common.cuh"

namespace askja {
namespace rows {

// shared memory per group: three NC x NP staging tiles, NP = NC rounded up to
// even so that every row starts on a 16-byte boundary, plus 16 bytes of skew
// so that the groups of one warp start in different banks (without it the
// tiles are a multiple of 128 bytes apart and every load is a bank conflict)
template <typename T>
__host__ __device__ inline size_t group_elems(int N) {
  return 3 * (size_t)N * (N + (N & 1)) + 16 / sizeof(cpx<T>);
}
template <typename T>
__host__ __device__ inline size_t smem_per_group(int N) {
  return group_elems<T>(N) * sizeof(cpx<T>);
}
template <typename T>
__device__ __forceinline__ cpx<T>* group_tile(unsigned char* smem_raw, int g, int N) {
  return reinterpret_cast<cpx<T>*>(smem_raw) + (size_t)g * group_elems<T>(N);
}

// tile[r*NP + c] = element (r, c) of the link (d, s), for c < NC; elements are
// written in pairs (one 16-byte store in FP32; the odd padding column of an
// odd NC gets a zero)
template <int NMAX, typename T, typename S2>
__device__ __forceinline__ void stage_row(cpx<T>* tile, int NP, const S2* __restrict__ f, const Lat& L, int d,
                                          int s, int r) {
  const int N = L.N;
  const S2* p = f + mbase(L, d, s) + (size_t)r * N * 32;
#pragma unroll
  for (int c = 0; c < NMAX; c += 2) {
    if (c >= N) continue;
    const cpx<T> v0 = ldc<T>(p + c * 32);
    const cpx<T> v1 = c + 1 < N ? ldc<T>(p + (c + 1) * 32) : czero<T>();
    if constexpr (sizeof(T) == 4) {
      *reinterpret_cast<float4*>(tile + r * NP + c) = make_float4(v0.re, v0.im, v1.re, v1.im);
    } else {
      tile[r * NP + c] = v0;
      tile[r * NP + c + 1] = v1;
    }
  }
}

// two consecutive complex numbers from shared memory (16-byte load in FP32)
template <typename T>
__device__ __forceinline__ void ld2(const cpx<T>* p, cpx<T>& a, cpx<T>& b) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    a = mkc<T>(v.x, v.y);
    b = mkc<T>(v.z, v.w);
  } else {
    a = p[0];
    b = p[1];
  }
}

// t[c] = sum_k A_k conj(tile[c][k]),  A_k = conj(a[k]) when CONJ_A else a[k]
template <int NMAX, typename T, bool CONJ_A>
__device__ __forceinline__ void row_times_tile_dag(cpx<T> (&t)[NMAX], const cpx<T> (&a)[NMAX], const cpx<T>* tile,
                                                   int NP, int N) {
  constexpr int KU = NMAX <= 16 ? NMAX : 1;
#pragma unroll KU
  for (int c = 0; c < NMAX; c++) {
    if (c >= N) continue;
    cpx<T> s = czero<T>();
#pragma unroll KU
    for (int k = 0; k < NMAX; k += 2) {
      if (k >= N) continue;
      cpx<T> b0, b1;
      ld2(tile + c * NP + k, b0, b1);
      if (CONJ_A) {
        cmac_cc(s, a[k], b0);
        if (k + 1 < N) cmac_cc(s, a[k + 1], b1);
      } else {
        cmac_nc(s, a[k], b0);
        if (k + 1 < N) cmac_nc(s, a[k + 1], b1);
      }
    }
    t[c] = s;
  }
}

// acc[c] += sum_k t[k] conj(tile[c][k])
template <int NMAX, typename T>
__device__ __forceinline__ void row_times_tile_dag_acc(cpx<T> (&acc)[NMAX], const cpx<T> (&t)[NMAX],
                                                       const cpx<T>* tile, int NP, int N) {
  constexpr int KU = NMAX <= 16 ? NMAX : 1;
#pragma unroll KU
  for (int c = 0; c < NMAX; c++) {
    if (c >= N) continue;
#pragma unroll KU
    for (int k = 0; k < NMAX; k += 2) {
      if (k >= N) continue;
      cpx<T> b0, b1;
      ld2(tile + c * NP + k, b0, b1);
      cmac_nc(acc[c], t[k], b0);
      if (k + 1 < N) cmac_nc(acc[c], t[k + 1], b1);
    }
  }
}

// acc[c] += sum_k t[k] tile[k][c]
template <int NMAX, typename T>
__device__ __forceinline__ void row_times_tile_acc(cpx<T> (&acc)[NMAX], const cpx<T> (&t)[NMAX], const cpx<T>* tile,
                                                   int NP, int N) {
  constexpr int KU = NMAX <= 16 ? NMAX : 1;
#pragma unroll KU
  for (int k = 0; k < NMAX; k++) {
    if (k >= N) continue;
    const cpx<T> tk = t[k];
#pragma unroll KU
    for (int c = 0; c < NMAX; c += 2) {
      if (c >= N) continue;
      cpx<T> b0, b1;
      ld2(tile + k * NP + c, b0, b1);
      cmac(acc[c], tk, b0);
      if (c + 1 < N) cmac(acc[c + 1], tk, b1);
    }
  }
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
      cpx<T> y = czero<T>();
      cmac(y, S[r * N + k], cph);
      S[r * N + k] = y;
    }
  }
  __syncthreads();
}

// One Newton-Schulz step towards the nearest unitary matrix,
//   U <- U (3 - U^dag U) / 2,
// the per-update projection of the FP32 single-chain path: after the link
// update U is unitary to FP32 rounding and the step squares the defect, so it
// returns to the rounding level; two tile products and three barriers instead
// of reunitarise_tile's 4N.  It does not pin det U to 1: the engine runs the
// full reunitarisation (with the determinant phase) over all links every few
// trajectories.  tm: row r of U; the result rows go to T0 with stride N (the
// copy-out layout).  All threads of the block call this (it has barriers).
template <int NMAX, typename T>
__device__ void newton_schulz_tile(const cpx<T> (&tm)[NMAX], cpx<T>* T0, cpx<T>* T1, int N, int NP, int r,
                                   bool act) {
  __syncthreads();
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T0[r * NP + c] = tm[c];
  }
  __syncthreads();
  if (act) {
    cpx<T> a[NMAX], m[NMAX];
#pragma unroll
    for (int k = 0; k < NMAX; k++) {
      m[k] = czero<T>();
      if (k < N) {
        const cpx<T> z = T0[k * NP + r];
        a[k] = mkc<T>(z.re, -z.im);  // row r of U^dag
      }
    }
    row_times_tile_acc<NMAX, T>(m, a, T0, NP, N);  // m[c] = (U^dag U)_rc
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T1[r * NP + c] = mkc<T>((c == r ? T(1.5) : T(0)) - T(0.5) * m[c].re, T(-0.5) * m[c].im);
  }
  __syncthreads();
  if (act) {
    cpx<T> un[NMAX];
#pragma unroll
    for (int c = 0; c < NMAX; c++) un[c] = czero<T>();
    row_times_tile_acc<NMAX, T>(un, tm, T1, NP, N);
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T0[r * N + c] = un[c];
  }
  __syncthreads();
}

// Tm = sum_{k<=order} X^k/k! U by Paterson-Stockmeyer with block size 3:
// with X^3 staged once, E = (..(B_q X^3 + B_(q-1)) X^3 + ..) X^3 + B_0
// (formed without its identity term, Tm = U + (E - 1) U),
// B_j = sum_{i<3} X^i / (3j+i)!, needs X^2, X^3, q = order/3 block products
// and E U -- 5 tile products for order 8 instead of Horner's 8, and three
// barriers instead of two per product (the block steps multiply by the same
// staged X^3).  Exact in real arithmetic; p = row r of X, u = row r of U.
// All threads of the block call this (it has barriers).
template <int NMAX, typename T>
__device__ void drift_ps(cpx<T> (&tm)[NMAX], const cpx<T> (&p)[NMAX], const cpx<T> (&u)[NMAX], cpx<T>* T0,
                         cpx<T>* T1, cpx<T>* T2, int N, int NP, int r, bool act, int order) {
  __syncthreads();
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) {
        T0[r * NP + c] = p[c];
        T2[r * NP + c] = u[c];
      }
  }
  __syncthreads();
  cpx<T> x2[NMAX];
#pragma unroll
  for (int c = 0; c < NMAX; c++) x2[c] = czero<T>();
  if (act) {
    row_times_tile_acc<NMAX, T>(x2, p, T0, NP, N);
    cpx<T> x3[NMAX];
#pragma unroll
    for (int c = 0; c < NMAX; c++) x3[c] = czero<T>();
    row_times_tile_acc<NMAX, T>(x3, x2, T0, NP, N);
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T1[r * NP + c] = x3[c];
  }
  __syncthreads();
  if (act) {
    // 1/k! for k <= order, zero beyond
    auto invfact = [order](int k) {
      if (k > order) return T(0);
      T f = T(1);
      for (int i = 2; i <= k; i++) f = f / T(i);
      return f;
    };
    const int q = order / 3;
    cpx<T> acc[NMAX];
    for (int j = q; j >= 0; j--) {
      // the identity of B_0 is left out: Em = E - 1, and U' = U + Em U keeps
      // the small update apart from U's own bits
      const T a0 = j ? invfact(3 * j) : T(0), a1 = invfact(3 * j + 1), a2 = invfact(3 * j + 2);
      cpx<T> nb[NMAX];  // B_j (+ acc X^3)
#pragma unroll
      for (int c = 0; c < NMAX; c++)
        nb[c] = mkc<T>(fma(a2, x2[c].re, fma(a1, p[c].re, c == r ? a0 : T(0))), fma(a2, x2[c].im, a1 * p[c].im));
      if (j < q) row_times_tile_acc<NMAX, T>(nb, acc, T1, NP, N);
#pragma unroll
      for (int c = 0; c < NMAX; c++) acc[c] = nb[c];
    }
#pragma unroll
    for (int c = 0; c < NMAX; c++) tm[c] = u[c];
    row_times_tile_acc<NMAX, T>(tm, acc, T2, NP, N);
  }
}

// Rows of the updated link -> T0 (stride N), then the full reunitarisation
// when reunit (ends with a barrier either way).
template <int NMAX, typename T>
__device__ __forceinline__ void finish_update(const cpx<T> (&tm)[NMAX], cpx<T>* T0, int N, int r, bool act,
                                              int reunit, int* piv, cpx<T>* det) {
  __syncthreads();
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T0[r * N + c] = tm[c];
  }
  __syncthreads();
  if (reunit) reunitarise_tile<T>(T0, T0 + N * N, N, r, act, piv, det);
  if (!reunit) __syncthreads();
}

// MODE 0: out-of-place kick  Pout = Pin - eps_k F(U)
// MODE 1: fused kick + drift P -= eps_k F(U); Uout = exp(i eps_d P) U
//
// A CTA owns GS = blockDim/NC consecutive sites site0 .. site0+GS-1 of one
// direction mu; group g (NC threads) computes the link (site0+g, mu), thread r
// of the group owns row r.  Every matrix a group needs is copied into its
// shared-memory tile by the whole CTA in "copy role": thread t copies row
// t / GS of group t % GS, so consecutive threads read the same element of
// consecutive sites -- coalesced, in the 32-site blocked field layout -- and
// the compute role then reads rows and columns from the tiles.  Outputs (P and
// the new links) go back the same way.
template <int NMAX, typename T, typename S2, int MODE>
__device__ __forceinline__ void force_rows(const Lat& L, const S2* __restrict__ U, const S2* Pin, S2* Pout,
                                           S2* __restrict__ Uout, T eps_k, T eps_d, int order, int reunit, int mu,
                                           int site0, unsigned char* smem_raw, int* piv_s, cpx<T>* det_s) {
  const int N = L.N;
  const int NP = N + (N & 1);
  const int GS = blockDim.x / N;
  const int tid = threadIdx.x;
  // compute role
  const int g = tid / N;
  const int r = tid - g * N;
  const bool act = g < GS && site0 + g < L.V;
  cpx<T>* T0 = group_tile<T>(smem_raw, act ? g : 0, N);
  cpx<T>* T1 = T0 + N * NP;
  cpx<T>* T2 = T1 + N * NP;
  // copy role
  const int cg = tid % GS;
  const int cr = tid / GS;
  const int cx = site0 + cg;
  const bool cact = cr < N && cx < L.V;
  cpx<T>* C0 = group_tile<T>(smem_raw, cg, N);
  cpx<T>* C1 = C0 + N * NP;
  cpx<T>* C2 = C1 + N * NP;

  cpx<T> acc[NMAX], a[NMAX], t[NMAX];
#pragma unroll
  for (int c = 0; c < NMAX; c++) acc[c] = czero<T>();

  const int cxpmu = cact ? nb_plus(L, mu, cx) : 0;
  for (int j = 0; j < L.D - 1; j++) {
    const int nu = j < mu ? j : j + 1;
    // upper: t = row r of U_nu(x+mu) U_mu^dag(x+nu); acc += t U_nu^dag(x)
    __syncthreads();
    if (cact) {
      stage_row<NMAX, T, S2>(C0, NP, U, L, mu, nb_plus(L, nu, cx), cr);
      stage_row<NMAX, T, S2>(C1, NP, U, L, nu, cx, cr);
      stage_row<NMAX, T, S2>(C2, NP, U, L, nu, cxpmu, cr);
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int k = 0; k < NMAX; k++)
        if (k < N) a[k] = T2[r * NP + k];
      row_times_tile_dag<NMAX, T, false>(t, a, T0, NP, N);
      row_times_tile_dag_acc<NMAX, T>(acc, t, T1, NP, N);
    }
    // lower: t = row r of U_nu^dag(x+mu-nu) U_mu^dag(x-nu); acc += t U_nu(x-nu)
    __syncthreads();
    if (cact) {
      const int cxmnu = nb_minus(L, nu, cx);
      stage_row<NMAX, T, S2>(C0, NP, U, L, nu, nb_minus(L, nu, cxpmu), cr);
      stage_row<NMAX, T, S2>(C1, NP, U, L, mu, cxmnu, cr);
      stage_row<NMAX, T, S2>(C2, NP, U, L, nu, cxmnu, cr);
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int k = 0; k < NMAX; k++)
        if (k < N) a[k] = T0[k * NP + r];  // column r: row r of the adjoint, conjugated below
      row_times_tile_dag<NMAX, T, true>(t, a, T1, NP, N);
      row_times_tile_acc<NMAX, T>(acc, t, T2, NP, N);
    }
  }
  // U_mu(x) -> T2 (rows kept in u[]), P(x) -> T1 (rows kept in p[])
  cpx<T> u[NMAX], p[NMAX];
  __syncthreads();
  if (cact) {
    stage_row<NMAX, T, S2>(C2, NP, U, L, mu, cx, cr);
    stage_row<NMAX, T, S2>(C1, NP, Pin, L, mu, cx, cr);
  }
  __syncthreads();
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) {
        u[c] = T2[r * NP + c];
        p[c] = T1[r * NP + c];
      }
  }
  __syncthreads();
  // W = U_mu(x) acc: acc rows -> T0, w[c] = sum_k u[k] acc[k][c]; W rows -> T1
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T0[r * NP + c] = acc[c];
  }
  __syncthreads();
  cpx<T> w[NMAX];
#pragma unroll
  for (int c = 0; c < NMAX; c++) w[c] = czero<T>();
  if (act) {
    row_times_tile_acc<NMAX, T>(w, u, T0, NP, N);
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T1[r * NP + c] = w[c];
  }
  __syncthreads();
  // kick with the traceless anti-hermitian part; new P rows -> T2 for the copy out
  if (act) {
    T trim = T(0);
    for (int k = 0; k < N; k++) trim += T1[k * NP + k].im;
    trim = trim / T(N);
#pragma unroll
    for (int c = 0; c < NMAX; c++) {
      if (c < N) {
        const cpx<T> wrc = w[c];
        const cpx<T> wcr = T1[c * NP + r];
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
  }
  __syncthreads();
  if (act) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) T2[r * NP + c] = p[c];
  }
  __syncthreads();
  if (cact) {
#pragma unroll
    for (int c = 0; c < NMAX; c++)
      if (c < N) stc(Pout + eoff(L, mu, cr * N + c, cx), C2[cr * NP + c]);
  }
  if (MODE == 1) {
    // drift: Tm <- U + (X/n) Tm, X = i eps_d P, Tm staged through T0
    cpx<T> tm[NMAX];
#pragma unroll
    for (int c = 0; c < NMAX; c++) {
      tm[c] = u[c];
      p[c] = mkc<T>(-eps_d * p[c].im, eps_d * p[c].re);
    }
    // FP32, NC <= 8, order >= 5: the same series by Paterson-Stockmeyer (the
    // Horner loop below is then skipped; for larger NC its extra row arrays
    // cost more occupancy than it saves); FP64 keeps the reference's Horner order
    const bool ps = sizeof(T) == 4 && NMAX == 8 && order >= 5;
    if constexpr (sizeof(T) == 4 && NMAX == 8)
      if (ps) drift_ps<NMAX, T>(tm, p, u, T0, T1, T2, N, NP, r, act, order);
    for (int n = ps ? 0 : order; n >= 1; n--) {
      __syncthreads();
      if (act) {
#pragma unroll
        for (int c = 0; c < NMAX; c++)
          if (c < N) T0[r * NP + c] = tm[c];
      }
      __syncthreads();
      if (act) {
        const T inv = T(1) / T(n);
        cpx<T> s[NMAX];
#pragma unroll
        for (int c = 0; c < NMAX; c++) s[c] = czero<T>();
        row_times_tile_acc<NMAX, T>(s, p, T0, NP, N);
#pragma unroll
        for (int c = 0; c < NMAX; c++) tm[c] = mkc<T>(fma(s[c].re, inv, u[c].re), fma(s[c].im, inv, u[c].im));
      }
    }
    if constexpr (sizeof(T) == 4) {
      if (reunit == 2)  // Newton-Schulz projection (ends with a barrier)
        newton_schulz_tile<NMAX, T>(tm, T0, T1, N, NP, r, act);
      else
        finish_update<NMAX, T>(tm, T0, N, r, act, reunit, &piv_s[act ? g : 0], &det_s[act ? g : 0]);
    } else {
      finish_update<NMAX, T>(tm, T0, N, r, act, reunit, &piv_s[act ? g : 0], &det_s[act ? g : 0]);
    }
    if (cact) {
#pragma unroll
      for (int c = 0; c < NMAX; c++)
        if (c < N) stc(Uout + eoff(L, mu, cr * N + c, cx), C0[cr * N + c]);
    }
  }
}

template <int NMAX, typename T, typename S2, int MODE>
__global__ void k_force(Lat L, const S2* __restrict__ U, const S2* Pin, S2* Pout, S2* __restrict__ Uout, T eps_k,
                        T eps_d, int order, int reunit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<T> det_s[64];
  // CTAs run site-block-major: consecutive CTAs take the directions of the same sites
  const int GS = blockDim.x / L.N;
  const int mu = blockIdx.x % L.D;
  const int site0 = (blockIdx.x / L.D) * GS;
  force_rows<NMAX, T, S2, MODE>(L, U, Pin, Pout, Uout, eps_k, eps_d, order, reunit, mu, site0, smem_raw, piv_s,
                                det_s);
}

// The same for FP32 with NMAX = 8 (the Paterson-Stockmeyer drift): at most 128
// registers, so that four 128-thread CTAs stay resident per SM (OCC 0), or
// tighter budgets for six / eight (OCC 1 / 2).
template <typename S2, int MODE, int OCC = 0>
__global__ void __launch_bounds__(256, 2 + OCC) k_force8(Lat L, const S2* __restrict__ U, const S2* Pin, S2* Pout,
                                                   S2* __restrict__ Uout, float eps_k, float eps_d, int order,
                                                   int reunit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<float> det_s[64];
  const int GS = blockDim.x / L.N;
  const int mu = blockIdx.x % L.D;
  const int site0 = (blockIdx.x / L.D) * GS;
  force_rows<8, float, S2, MODE>(L, U, Pin, Pout, Uout, eps_k, eps_d, order, reunit, mu, site0, smem_raw, piv_s,
                                 det_s);
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
  cpx<T>* S0 = group_tile<T>(smem_raw, in_group ? g : 0, N);
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
        if (k >= N) continue;
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
// With a gate, the launch does nothing unless *gate % every == 0 (a counter
// in device memory, so that a captured trajectory graph can run it on every
// `every`-th replay).
template <typename T, typename S2>
__global__ void k_reunit(Lat L, S2* __restrict__ U, const unsigned long long* __restrict__ gate, int every) {
  if (gate && every > 1 && (*gate % (unsigned long long)every) != 0) return;
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
  cpx<T>* S0 = group_tile<T>(smem_raw, in_group ? g : 0, N);
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
