// Eigenvalues of the closed Wilson / Polyakov line matrices, for the
// eigenphase distributions of measurements4d.cpp:185-309 (getevs), which the
// reference computes with Eigen's ComplexEigenSolver on the host.
//
// One CTA per line: the line product W is formed in FP64 as in k_lines (row
// per thread, running product in shared memory), then warp 0 computes the
// eigenvalues of W: Householder reduction to upper Hessenberg form, then the
// implicitly shifted complex QR iteration (single Wilkinson shift, an
// exceptional shift every 11th iteration without deflation) on the active
// window only, deflating from the bottom.  Rotations and reflections are
// applied with the 32 lanes spread over the rows or columns they touch.  The
// iteration count is bounded (60 N sweeps); a line that does not converge gets
// NaN eigenvalues and sets *fail.
#pragma once

#include "common.cuh"

namespace askja {
namespace eig {

__device__ __forceinline__ double cabs2(const cpx<double>& z) { return z.re * z.re + z.im * z.im; }
__device__ __forceinline__ double cabs(const cpx<double>& z) { return hypot(z.re, z.im); }
__device__ __forceinline__ cpx<double> cmulz(const cpx<double>& a, const cpx<double>& b) {
  return mkc<double>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ cpx<double> cconj(const cpx<double>& a) { return mkc<double>(a.re, -a.im); }
__device__ __forceinline__ cpx<double> csub(const cpx<double>& a, const cpx<double>& b) {
  return mkc<double>(a.re - b.re, a.im - b.im);
}
// principal square root
__device__ __forceinline__ cpx<double> csqrt(const cpx<double>& z) {
  const double r = hypot(z.re, z.im);
  if (r == 0.0) return czero<double>();
  const double t = sqrt(0.5 * (r + fabs(z.re)));
  if (z.re >= 0.0) return mkc<double>(t, z.im / (2.0 * t));
  return mkc<double>(fabs(z.im) / (2.0 * t), copysign(t, z.im));
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Eigenvalues of the N x N matrix H (row-major, shared memory; destroyed).
// Called by all 32 lanes of one warp; v is N elements of shared scratch.
static __device__ void hessenberg_qr(cpx<double>* H, int N, cpx<double>* v, cpx<double>* ev, int* fail) {
  const int lane = threadIdx.x & 31;
  // Householder: H <- P H P, P = 1 - 2 v v^H, zeroing column k below the subdiagonal
  for (int k = 0; k + 2 < N; k++) {
    double nrm2 = 0.0;
    for (int i = k + 1 + lane; i < N; i += 32) nrm2 += cabs2(H[i * N + k]);
    nrm2 = warp_sum(nrm2);
    const cpx<double> x0 = H[(k + 1) * N + k];
    const double ax0 = cabs(x0);
    if (nrm2 - ax0 * ax0 <= 0.0) continue;  // column already reduced
    const double xn = sqrt(nrm2);
    const cpx<double> ph = ax0 > 0.0 ? mkc<double>(x0.re / ax0, x0.im / ax0) : mkc<double>(1.0, 0.0);
    const cpx<double> alpha = mkc<double>(-ph.re * xn, -ph.im * xn);
    const double inv = 1.0 / sqrt(nrm2 - ax0 * ax0 + (ax0 + xn) * (ax0 + xn));
    for (int i = k + 1 + lane; i < N; i += 32) {
      const cpx<double> x = i == k + 1 ? csub(x0, alpha) : H[i * N + k];
      v[i] = mkc<double>(x.re * inv, x.im * inv);
    }
    __syncwarp();
    for (int j = k + lane; j < N; j += 32) {  // left: columns j >= k
      cpx<double> w = czero<double>();
      for (int i = k + 1; i < N; i++) cmac_cn(w, v[i], H[i * N + j]);
      for (int i = k + 1; i < N; i++) {
        const cpx<double> t = cmulz(v[i], w);
        H[i * N + j].re -= 2.0 * t.re;
        H[i * N + j].im -= 2.0 * t.im;
      }
    }
    __syncwarp();
    for (int i = lane; i < N; i += 32) {  // right: every row
      cpx<double> w = czero<double>();
      for (int j = k + 1; j < N; j++) cmac(w, H[i * N + j], v[j]);
      for (int j = k + 1; j < N; j++) {
        const cpx<double> t = cmulz(w, cconj(v[j]));
        H[i * N + j].re -= 2.0 * t.re;
        H[i * N + j].im -= 2.0 * t.im;
      }
    }
    __syncwarp();
    if (lane == 0) {
      H[(k + 1) * N + k] = alpha;
      for (int i = k + 2; i < N; i++) H[i * N + k] = czero<double>();
    }
    __syncwarp();
  }
  // shifted QR on the active window [l, hi], deflating at the bottom
  int hi = N - 1, iter = 0, total = 0;
  const double eps = 2.220446049250313e-16;
  while (hi >= 0) {
    __syncwarp();
    if (hi == 0) {
      if (lane == 0) ev[0] = H[0];
      break;
    }
    int l = hi;
    while (l > 0) {
      const double s = cabs(H[(l - 1) * N + l - 1]) + cabs(H[l * N + l]);
      if (cabs(H[l * N + l - 1]) <= eps * (s > 0.0 ? s : 1.0)) break;
      l--;
    }
    if (l == hi) {
      if (lane == 0) ev[hi] = H[hi * N + hi];
      hi--;
      iter = 0;
      continue;
    }
    if (++total > 60 * N) {
      if (lane == 0) {
        for (int i = 0; i <= hi; i++) ev[i] = mkc<double>(nan(""), nan(""));
        atomicOr(fail, 1);
      }
      break;
    }
    iter++;
    const cpx<double> a = H[(hi - 1) * N + hi - 1], b = H[(hi - 1) * N + hi];
    const cpx<double> c = H[hi * N + hi - 1], d = H[hi * N + hi];
    cpx<double> mu;
    if (iter % 11 == 0) {
      mu = mkc<double>(d.re + cabs(c), d.im);
    } else {  // the eigenvalue of the trailing 2 x 2 block closer to d
      const cpx<double> h = mkc<double>(0.5 * (a.re - d.re), 0.5 * (a.im - d.im));
      cpx<double> q = cmulz(h, h);
      const cpx<double> bc = cmulz(b, c);
      q.re += bc.re;
      q.im += bc.im;
      const cpx<double> r = csqrt(q);
      const cpx<double> m = mkc<double>(0.5 * (a.re + d.re), 0.5 * (a.im + d.im));
      const cpx<double> m1 = mkc<double>(m.re + r.re, m.im + r.im), m2 = mkc<double>(m.re - r.re, m.im - r.im);
      mu = cabs2(csub(m1, d)) <= cabs2(csub(m2, d)) ? m1 : m2;
    }
    cpx<double> x = csub(H[l * N + l], mu), y = H[(l + 1) * N + l];
    for (int k = l; k < hi; k++) {
      if (k > l) {
        x = H[k * N + k - 1];
        y = H[(k + 1) * N + k - 1];
      }
      const double ax = cabs(x), ay = cabs(y), r = hypot(ax, ay);
      double cg;
      cpx<double> sg;
      if (r == 0.0) {
        cg = 1.0;
        sg = czero<double>();
      } else if (ax == 0.0) {
        cg = 0.0;
        sg = mkc<double>(y.re / ay, -y.im / ay);
      } else {
        cg = ax / r;
        const cpx<double> t = cmulz(mkc<double>(x.re / ax, x.im / ax), cconj(y));
        sg = mkc<double>(t.re / r, t.im / r);
      }
      __syncwarp();
      for (int j = (k > l ? k - 1 : l) + lane; j <= hi; j += 32) {  // rows k, k+1
        const cpx<double> h1 = H[k * N + j], h2 = H[(k + 1) * N + j];
        const cpx<double> t1 = cmulz(sg, h2), t2 = cmulz(cconj(sg), h1);
        H[k * N + j] = mkc<double>(cg * h1.re + t1.re, cg * h1.im + t1.im);
        H[(k + 1) * N + j] = mkc<double>(cg * h2.re - t2.re, cg * h2.im - t2.im);
      }
      __syncwarp();
      const int ie = k + 2 < hi ? k + 2 : hi;
      for (int i = l + lane; i <= ie; i += 32) {  // columns k, k+1
        const cpx<double> h1 = H[i * N + k], h2 = H[i * N + k + 1];
        const cpx<double> t1 = cmulz(cconj(sg), h2), t2 = cmulz(sg, h1);
        H[i * N + k] = mkc<double>(cg * h1.re + t1.re, cg * h1.im + t1.im);
        H[i * N + k + 1] = mkc<double>(cg * h2.re - t2.re, cg * h2.im - t2.im);
      }
      __syncwarp();
    }
  }
  __syncwarp();
}

// Line q starts at q * start_stride and runs along `dir` through all
// n[dir] links (the lines of k_lines); ev[q*N + i] = eigenvalue i of W_q.
template <typename S2>
__global__ void k_line_eigs(Lat L, const S2* __restrict__ U, int dir, int start_stride, double2* __restrict__ ev,
                            int* __restrict__ fail) {
  extern __shared__ __align__(16) unsigned char esm[];
  const int N = L.N;
  cpx<double>* W = reinterpret_cast<cpx<double>*>(esm);
  cpx<double>* tmp = W + N * N;  // product scratch, later Householder vector and eigenvalues
  const int r = threadIdx.x;
  int pos = blockIdx.x * start_stride;
  if (r < N)
    for (int c = 0; c < N; c++) W[r * N + c] = ldc<double>(U + eoff(L, dir, r * N + c, pos));
  __syncthreads();
  for (int st = 0; st < L.n[dir] - 1; st++) {
    pos = nb_plus(L, dir, pos);
    if (r < N)
      for (int c = 0; c < N; c++) {
        cpx<double> s = czero<double>();
        for (int k = 0; k < N; k++) cmac(s, W[r * N + k], ldc<double>(U + eoff(L, dir, k * N + c, pos)));
        tmp[r * N + c] = s;
      }
    __syncthreads();
    if (r < N)
      for (int c = 0; c < N; c++) W[r * N + c] = tmp[r * N + c];
    __syncthreads();
  }
  if (r < 32) {
    cpx<double>* vsc = tmp;
    cpx<double>* e = tmp + N;
    hessenberg_qr(W, N, vsc, e, fail);
    for (int i = r; i < N; i += 32) ev[(size_t)blockIdx.x * N + i] = make_double2(e[i].re, e[i].im);
  }
}

}  // namespace eig
}  // namespace askja
