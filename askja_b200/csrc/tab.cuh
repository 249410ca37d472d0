// The reference's energy-momentum tensor at a site (sun.cpp:580-670, Tab) and
// the Fourier coefficients of the plaquette energy (sun.cpp:365-411,
// FourierTrafo).  Neither is called by the reference's drivers; both are
// diagnostics built on the clover field strength and the plaquette.
//
// k_tab: one CTA per site, FP64 throughout (links and momenta of either
// storage precision promoted on load).  For each plane a < b the clover sum
// C_ab (four leaves of four links, sun.cpp:603-616) is formed in shared
// memory, thread r owning row r of the running product, factors read from
// global memory (L1/L2-resident neighbours); the reference's
// F_ab = (C_ab - C_ba)/8 is (C_ab - C_ab^dag)/8, since every leaf of C_ba is
// the adjoint of a leaf of C_ab.  The per-site sums it needs are
//   e_j  = ReTr((pi_j + Pi_j)^2)                    (tr2, sunmat.h:331-338)
//   t_ab = ReTr(F_ab^2)                              (= ReTr(F_ba^2))
//   g_b  = ImTr((pi_b + Pi_b) F_b0) = -ImTr((pi_b + Pi_b) F_0b)
// and the site's contribution to mdata (sun.cpp:636-667) is
//   m[0]   = 1/4 sum_j e_j - sum_{a<b} t_ab
//   m[1]   = sum_b g_b
//   m[2+m] = -1/2 e_m + 1/4 sum_j e_j - 2 sum_j t_jm + sum_{a<b} t_ab.
#pragma once

#include "common.cuh"
#include "misc.cuh"

namespace askja {
namespace tab {

constexpr int TAB_MAX_D = 8;  // per-site sums kept in registers of thread 0

// shared memory of k_tab: three N x N FP64 complex matrices
inline size_t tab_smem(int N) { return (size_t)3 * N * N * sizeof(cpx<double>); }

template <typename S2>
__device__ __forceinline__ cpx<double> elem(const Lat& L, const S2* __restrict__ f, int d, int s, int r, int c,
                                            bool dag) {
  const int N = L.N;
  const cpx<double> z = ldc<double>(f + eoff(L, d, dag ? c * N + r : r * N + c, s));
  return dag ? mkc<double>(z.re, -z.im) : z;
}

// Rows of the product of four links (dir, site, dagger) into out (written or
// added); A, B are scratch.  Thread r < N owns row r.
template <typename S2>
__device__ void leaf(const Lat& L, const S2* __restrict__ U, const int (&dir)[4], const int (&site)[4],
                     const bool (&dag)[4], cpx<double>* A, cpx<double>* B, cpx<double>* out, bool accumulate) {
  const int N = L.N, r = threadIdx.x;
  if (r < N)
    for (int c = 0; c < N; c++) A[r * N + c] = elem(L, U, dir[0], site[0], r, c, dag[0]);
  __syncthreads();
  for (int f = 1; f < 4; f++) {
    cpx<double>* src = (f & 1) ? A : B;
    cpx<double>* dst = (f == 3) ? nullptr : ((f & 1) ? B : A);
    if (r < N)
      for (int c = 0; c < N; c++) {
        cpx<double> s = czero<double>();
        for (int k = 0; k < N; k++) cmac(s, src[r * N + k], elem(L, U, dir[f], site[f], k, c, dag[f]));
        if (dst) {
          dst[r * N + c] = s;
        } else if (accumulate) {
          out[r * N + c].re += s.re;
          out[r * N + c].im += s.im;
        } else {
          out[r * N + c] = s;
        }
      }
    __syncthreads();
  }
}

// out[(s - site0) * npt + m]: the site's contribution to Tab's mdata[m].
template <typename S2>
__global__ void k_tab(Lat L, const S2* __restrict__ U, const S2* __restrict__ Pa, const S2* __restrict__ Pb,
                      int site0, int npt, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char tsm[];
  const int N = L.N, D = L.D, r = threadIdx.x;
  cpx<double>* A = reinterpret_cast<cpx<double>*>(tsm);
  cpx<double>* B = A + N * N;
  cpx<double>* C = B + N * N;
  const int i = site0 + blockIdx.x;
  // e_j, g_j and tcol[m] = sum_j t_jm; only thread 0's copies hold the sums
  double e[TAB_MAX_D], g[TAB_MAX_D], tcol[TAB_MAX_D];
  double tsum = 0.0;
  for (int j = 0; j < D; j++) {
    double v[1] = {0.0};
    if (r < N)
      for (int c = 0; c < N; c++) {
        const cpx<double> x = ldc<double>(Pa + eoff(L, j, r * N + c, i)), y = ldc<double>(Pb + eoff(L, j, r * N + c, i));
        const cpx<double> u = ldc<double>(Pa + eoff(L, j, c * N + r, i)), w = ldc<double>(Pb + eoff(L, j, c * N + r, i));
        const cpx<double> p = mkc<double>(x.re + y.re, x.im + y.im), q = mkc<double>(u.re + w.re, u.im + w.im);
        v[0] += p.re * q.re - p.im * q.im;  // Re (pp)_rc (pp)_cr
      }
    misc::block_sum<1>(v);
    e[j] = v[0];
    g[j] = 0.0;
    tcol[j] = 0.0;
  }
  for (int a = 0; a < D; a++)
    for (int b = a + 1; b < D; b++) {
      const int right = nb_plus(L, a, i), up = nb_plus(L, b, i);
      const int left = nb_minus(L, a, i), down = nb_minus(L, b, i);
      const int downright = nb_plus(L, a, down), downleft = nb_minus(L, a, down), upleft = nb_minus(L, a, up);
      {  // U_a(i) U_b(i+a) U_a(i+b)^dag U_b(i)^dag
        const int d[4] = {a, b, a, b}, s[4] = {i, right, up, i};
        const bool dg[4] = {false, false, true, true};
        leaf(L, U, d, s, dg, A, B, C, false);
      }
      {  // U_b(i) U_a(i+b-a)^dag U_b(i-a)^dag U_a(i-a)
        const int d[4] = {b, a, b, a}, s[4] = {i, upleft, left, left};
        const bool dg[4] = {false, true, true, false};
        leaf(L, U, d, s, dg, A, B, C, true);
      }
      {  // U_a(i-a)^dag U_b(i-a-b)^dag U_a(i-a-b) U_b(i-b)
        const int d[4] = {a, b, a, b}, s[4] = {left, downleft, downleft, down};
        const bool dg[4] = {true, true, false, false};
        leaf(L, U, d, s, dg, A, B, C, true);
      }
      {  // U_b(i-b)^dag U_a(i-b) U_b(i-b+a) U_a(i)^dag
        const int d[4] = {b, a, b, a}, s[4] = {down, down, downright, i};
        const bool dg[4] = {true, false, false, true};
        leaf(L, U, d, s, dg, A, B, C, true);
      }
      // F = (C - C^dag) / 8; t = ReTr F^2; for a = 0 also ImTr(pp_b F_0b)
      double v[2] = {0.0, 0.0};
      if (r < N)
        for (int c = 0; c < N; c++) {
          const cpx<double> crc = C[r * N + c], ccr = C[c * N + r];
          const cpx<double> frc = mkc<double>(0.125 * (crc.re - ccr.re), 0.125 * (crc.im + ccr.im));
          const cpx<double> fcr = mkc<double>(0.125 * (ccr.re - crc.re), 0.125 * (ccr.im + crc.im));
          v[0] += frc.re * fcr.re - frc.im * fcr.im;
          if (a == 0) {  // Im (pp_b)_rc F_cr
            const cpx<double> x = ldc<double>(Pa + eoff(L, b, r * N + c, i));
            const cpx<double> y = ldc<double>(Pb + eoff(L, b, r * N + c, i));
            v[1] += (x.re + y.re) * fcr.im + (x.im + y.im) * fcr.re;
          }
        }
      misc::block_sum<2>(v);
      tsum += v[0];
      tcol[a] += v[0];
      tcol[b] += v[0];
      if (a == 0) g[b] = -v[1];
    }
  if (r == 0) {
    double esum = 0.0, gsum = 0.0;
    for (int j = 0; j < D; j++) {
      esum += e[j];
      gsum += g[j];
    }
    double* o = out + (size_t)blockIdx.x * npt;
    o[0] = 0.25 * esum - tsum;
    o[1] = gsum;
    for (int m = 0; m + 2 < npt; m++) o[m + 2] = -0.5 * e[m] + 0.25 * esum - 2.0 * tcol[m] + tsum;
  }
}

// coef[j] = |x_j|, x the inverse DFT (normalised by 1/n, as
// gsl_fft_complex_inverse) of the real sequence z_k = partial[2k] +
// partial[2k+1]: the plaquette energy sum_{a<b} (1 - ReTr P_ab / N) of site k,
// from misc::k_plaq_big.
static __global__ void k_dft_abs(const double* __restrict__ partial, int n, double* __restrict__ coef) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < n; k++) {
      const double z = partial[2 * k] + partial[2 * k + 1];
      double s, c;
      sincospi(2.0 * (double)(((long)j * k) % n) / (double)n, &s, &c);
      re = fma(z, c, re);
      im = fma(z, s, im);
    }
    coef[j] = hypot(re, im) / n;
  }
}

}  // namespace tab
}  // namespace askja
