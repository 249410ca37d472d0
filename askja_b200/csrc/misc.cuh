// Reductions, measurements, momentum refresh, hot start and the Metropolis
// step.  Every reduction accumulates in FP64 whatever the storage precision
// of the links (FP32 links are promoted on load), writes one partial per
// block, and a single-block pass sums the partials in block order, so results
// are deterministic run to run.
//
// The kernels take the colour number as a template parameter NT for the small
// cases (fully unrolled) and NT = 0 for any NC (runtime loops).
#pragma once

#include "common.cuh"

namespace askja {
namespace misc {

constexpr int RED_THREADS = 256;

// Block-wide sum of K doubles; thread 0 gets the result.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
  __shared__ double sh[K][RED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double x = lane < (int)(blockDim.x >> 5) ? sh[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[k] = x;
    }
  }
  __syncthreads();
}

// Sum nblocks partials of width K (layout partial[b*K + k]) into out[k].
template <int K>
__global__ void k_finish(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
  double v[K];
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; k++) v[k] += partial[(size_t)b * K + k];
  block_sum<K>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = v[k];
}

// Plaquette sums per site (sun.cpp:507-537 EnergyMag; measurements4d.cpp:885-927
// PlaqExp).  partial[b*2 + 0] = temporal planes (0,k), [b*2+1] = spatial (j,k), j>=1.
// ReTr(A B C^dag D^dag) is evaluated as Re sum_ij (AB)_ij conj((DC)_ij).
template <int NT, typename S2>
__device__ __forceinline__ void plaq_site(const Lat& L, const S2* __restrict__ U, int s, double (&v)[2]) {
  const int N = NT > 0 ? NT : L.N;
  if (s < L.V && counted(L, s)) {
    for (int mu = 0; mu < L.D; mu++) {
      const int xpmu = nb_plus(L, mu, s);
      for (int nu = mu + 1; nu < L.D; nu++) {
        const int xpnu = nb_plus(L, nu, s);
        double tr = 0.0;
#pragma unroll(NT > 0 ? NT : 1)
        for (int i = 0; i < N; i++)
#pragma unroll(NT > 0 ? NT : 1)
          for (int j = 0; j < N; j++) {
            cpx<double> ab = czero<double>(), dc = czero<double>();
#pragma unroll(NT > 0 ? NT : 1)
            for (int k = 0; k < N; k++) {
              cmac(ab, ldc<double>(U + eoff(L, mu, i * N + k, s)), ldc<double>(U + eoff(L, nu, k * N + j, xpmu)));
              cmac(dc, ldc<double>(U + eoff(L, nu, i * N + k, s)), ldc<double>(U + eoff(L, mu, k * N + j, xpnu)));
            }
            // explicit fma: the same rounding in every kernel that inlines this
            tr = fma(ab.re, dc.re, tr);
            tr = fma(ab.im, dc.im, tr);
          }
        v[mu == 0 ? 0 : 1] += 1.0 - tr / N;
      }
    }
  }
}

template <int NT, typename S2>
__global__ void __launch_bounds__(RED_THREADS) k_plaq(Lat L, const S2* __restrict__ U, double* __restrict__ partial) {
  double v[2] = {0.0, 0.0};
  plaq_site<NT, S2>(L, U, blockIdx.x * blockDim.x + threadIdx.x, v);
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 2 + 0] = v[0];
    partial[blockIdx.x * 2 + 1] = v[1];
  }
}

// Per-link sums: [0] = sum ReTr(A A) for A = Pa (sun.cpp:540-548 simpleenergyEl),
// [1] = sum 1/4 ReTr((Pa+Pb)^2) (sun.cpp:560-567 EnergyEl, when Pb != null),
// [2] = sum ReTr((U U^dag - 1)^2) (sun.cpp:441-471 UViol, when U != null).
template <int NT, typename S2>
__device__ __forceinline__ void link_sums(const Lat& L, const S2* __restrict__ Pa, const S2* __restrict__ Pb,
                                          const S2* __restrict__ U, long t, double (&v)[3]) {
  const int N = NT > 0 ? NT : L.N;
  if (t < (long)L.V * L.D && counted(L, (int)(t % L.V))) {
    const int d = (int)(t / L.V);
    const int s = (int)(t - (long)d * L.V);
    if (Pa) {
      double a = 0.0, b = 0.0;
#pragma unroll(NT > 0 ? NT : 1)
      for (int i = 0; i < N; i++)
#pragma unroll(NT > 0 ? NT : 1)
        for (int j = 0; j < N; j++) {
          const cpx<double> x = ldc<double>(Pa + eoff(L, d, i * N + j, s));
          const cpx<double> y = ldc<double>(Pa + eoff(L, d, j * N + i, s));
          a = fma(x.re, y.re, a);
          a = fma(-x.im, y.im, a);
          if (Pb) {
            const cpx<double> x2 = ldc<double>(Pb + eoff(L, d, i * N + j, s));
            const cpx<double> y2 = ldc<double>(Pb + eoff(L, d, j * N + i, s));
            b = fma(x.re + x2.re, y.re + y2.re, b);
            b = fma(-(x.im + x2.im), y.im + y2.im, b);
          }
        }
      v[0] = a;
      v[1] = 0.25 * b;
    }
    if (U) {
      double c = 0.0;
#pragma unroll(NT > 0 ? NT : 1)
      for (int i = 0; i < N; i++)
#pragma unroll(NT > 0 ? NT : 1)
        for (int j = 0; j < N; j++) {
          cpx<double> aij = czero<double>(), aji = czero<double>();
#pragma unroll(NT > 0 ? NT : 1)
          for (int k = 0; k < N; k++) {
            cmac_nc(aij, ldc<double>(U + eoff(L, d, i * N + k, s)), ldc<double>(U + eoff(L, d, j * N + k, s)));
            cmac_nc(aji, ldc<double>(U + eoff(L, d, j * N + k, s)), ldc<double>(U + eoff(L, d, i * N + k, s)));
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
}

template <int NT, typename S2>
__global__ void __launch_bounds__(RED_THREADS) k_linksums(Lat L, const S2* __restrict__ Pa, const S2* __restrict__ Pb,
                                                          const S2* __restrict__ U, double* __restrict__ partial) {
  double v[3] = {0.0, 0.0, 0.0};
  link_sums<NT, S2>(L, Pa, Pb, U, (long)blockIdx.x * blockDim.x + threadIdx.x, v);
  block_sum<3>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; k++) partial[blockIdx.x * 3 + k] = v[k];
}

// Gauss law (sun.cpp:415-438): the lattice sum of Pi_j(x) - U_j^dag(x-j) Pi_j(x-j) U_j(x-j)
// over all sites and directions.  Re-indexing x -> x+j turns every term into a
// function of one link l: Pi_l - U_l^dag Pi_l U_l.  One block accumulates its
// links' matrices element by element; partial[b*2*N*N + 2e + {0,1}].
template <typename S2>
__global__ void __launch_bounds__(RED_THREADS) k_gauss(Lat L, const S2* __restrict__ U, const S2* __restrict__ Pi,
                                                       int links_per_block, double* __restrict__ partial) {
  const int N = L.N, NN = N * N;
  const long l0 = (long)blockIdx.x * links_per_block;
  const long l1 = min((long)L.V * L.D, l0 + links_per_block);
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int i = e / N, j = e - i * N;
    double sr = 0.0, si = 0.0;
    for (long l = l0; l < l1; l++) {
      const int d = (int)(l / L.V);
      const int s = (int)(l - (long)d * L.V);
      cpx<double> g = ldc<double>(Pi + eoff(L, d, e, s));
      // (U^dag Pi U)_ij = sum_ab conj(U_ai) Pi_ab U_bj
      cpx<double> t = czero<double>();
      for (int a = 0; a < N; a++) {
        cpx<double> pu = czero<double>();
        for (int b = 0; b < N; b++)
          cmac(pu, ldc<double>(Pi + eoff(L, d, a * N + b, s)), ldc<double>(U + eoff(L, d, b * N + j, s)));
        cmac_cn(t, ldc<double>(U + eoff(L, d, a * N + i, s)), pu);
      }
      sr += g.re - t.re;
      si += g.im - t.im;
    }
    partial[(size_t)blockIdx.x * 2 * NN + 2 * e] = sr;
    partial[(size_t)blockIdx.x * 2 * NN + 2 * e + 1] = si;
  }
}

// Sum the Gauss-law partials and return tr2 of the summed matrix.
static __global__ void k_gauss_finish(const double* __restrict__ partial, int nblocks, int N, double* __restrict__ out) {
  extern __shared__ double gsum[];
  const int NN = N * N;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int b = 0; b < nblocks; b++) {
      sr += partial[(size_t)b * 2 * NN + 2 * e];
      si += partial[(size_t)b * 2 * NN + 2 * e + 1];
    }
    gsum[2 * e] = sr;
    gsum[2 * e + 1] = si;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) {
        const double ar = gsum[2 * (i * N + j)], ai = gsum[2 * (i * N + j) + 1];
        const double br = gsum[2 * (j * N + i)], bi = gsum[2 * (j * N + i) + 1];
        r += ar * br - ai * bi;
      }
    *out = r;
  }
}

// Closed Wilson lines: line q starts at site q*start_stride and runs along
// direction `dir` through all n[dir] links; out[q] = |Tr W| / NC.
// One block (NC threads, thread r owns row r of W) per line; the running
// product is kept in shared memory.
// sun.cpp:307-362 (one line, dir 0 from site 0), measurements4d.cpp:410-466
// (Polyakov: dir 0 through (0,x1,0..)), measurements4d.cpp:311-355 (dir >= 1
// through (x0,0,..)).
template <typename S2>
__global__ void k_lines(Lat L, const S2* __restrict__ U, int dir, int start_stride, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char lsm[];
  cpx<double>* W = reinterpret_cast<cpx<double>*>(lsm);
  cpx<double>* tmp = W + L.N * L.N;
  const int N = L.N;
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
  if (r == 0) {
    double tr = 0.0, ti = 0.0;
    for (int k = 0; k < N; k++) {
      tr += W[k * N + k].re;
      ti += W[k * N + k].im;
    }
    out[blockIdx.x] = hypot(tr, ti) / N;
  }
}

// Slice averages for measurements4d.cpp:357-408 scalarLoopcorr:
// out[x0] = mean over the x0-slice of ReTr U_{D-1} / NC.  One block per slice.
template <typename S2>
__global__ void __launch_bounds__(RED_THREADS) k_slice_trace(Lat L, const S2* __restrict__ U, double* __restrict__ out) {
  const int N = L.N;
  const int slice = L.stride[0];
  double v[1] = {0.0};
  for (int s = blockIdx.x * slice + threadIdx.x; s < (blockIdx.x + 1) * slice; s += blockDim.x) {
    double t = 0.0;
    for (int k = 0; k < N; k++) t += ldc<double>(U + eoff(L, L.D - 1, k * N + k, s)).re;
    v[0] += t / N;
  }
  block_sum<1>(v);
  if (threadIdx.x == 0) out[blockIdx.x] = v[0] / slice;
}

// Momentum refresh (sun.cpp:209-252 initializeE with the reference's
// generator basis, sun.cpp:142-189): P = scale * sum_a xi_a T_a,
// scale = sqrt(2 NC / beta).  xi_a are Philox normals: link l = s*D + d
// (U-conf order), block j = a/4, counter (j, l_lo, l_hi, traj), key = seed.
// The explicit basis: for the p-th pair i<j (row-major), T_2p has 1/2 at
// (i,j),(j,i); T_2p+1 has -i/2 at (i,j), +i/2 at (j,i); the m-th diagonal
// generator is norm_m * diag(1,..,1 (m+1 times), -(m+1), 0, ..),
// norm_m = sqrt(1 / (2 (m+1)(m+2))).
// The entries of one link's momentum in generation order: emit(i, j, value)
// for the upper and lower entry of every off-diagonal pair, then the diagonal
// from the last row up.  Shared by the matrix refresh below and the refresh of
// the residual-plane FP32 mode (split.cuh), so both draw identical momenta.
template <typename Emit>
__device__ __forceinline__ void refresh_entries(const Lat& L, uint64_t seed, uint32_t traj, double scale, int d, int s,
                                                Emit&& emit) {
  const int N = L.N;
  const unsigned long long lk = (unsigned long long)s * L.D + d;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  int cur_blk = -1;
  double g[4];
  auto normal = [&](int a) -> double {
    const int blk = a >> 2;
    if (blk != cur_blk) {
      u32x4 c;
      c.x = (uint32_t)blk;
      c.y = (uint32_t)lk;
      c.z = (uint32_t)(lk >> 32);
      c.w = traj;
      normals4(philox4x32_10(c, k0, k1), g);
      cur_blk = blk;
    }
    return g[a & 3];
  };
  int p = 0;
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++, p++) {
      const double xs = normal(2 * p), xa = normal(2 * p + 1);
      emit(i, j, mkc<double>(0.5 * scale * xs, -0.5 * scale * xa));
      emit(j, i, mkc<double>(0.5 * scale * xs, 0.5 * scale * xa));
    }
  // diagonal: P_dd = scale * (S_d - d * norm_{d-1} xi_{d-1}),  S_d = sum_{m>=d} norm_m xi_m
  const int a0 = N * (N - 1);
  double suffix = 0.0;
  for (int dd = N - 1; dd >= 0; dd--) {
    double val = suffix;
    if (dd >= 1) {
      const int m = dd - 1;
      const double nm = sqrt(0.5 / ((double)(m + 1) * (m + 2)));
      const double xm = normal(a0 + m);
      val -= dd * nm * xm;
      suffix += nm * xm;
    }
    emit(dd, dd, mkc<double>(scale * val, 0.0));
  }
}

template <typename S2>
__device__ __forceinline__ void refresh_link(const Lat& L, S2* __restrict__ P, uint64_t seed, uint32_t traj,
                                             double scale, long t) {
  if (t >= (long)L.V * L.D) return;
  const int N = L.N;
  const int d = (int)(t / L.V);
  const int s = (int)(t - (long)d * L.V);
  refresh_entries(L, seed, traj, scale, d, s,
                  [&](int i, int j, const cpx<double>& v) { stc(P + eoff(L, d, i * N + j, s), v); });
}

template <typename S2>
__global__ void k_refresh(Lat L, S2* __restrict__ P, uint64_t seed, const unsigned long long* __restrict__ traj_dev,
                          unsigned long long traj_host, double scale) {
  const uint32_t traj = (uint32_t)(traj_dev ? *traj_dev : traj_host);
  refresh_link<S2>(L, P, seed, traj, scale, (long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Cold start (sun.cpp:194-207): every link the identity.
// (Padding sites get the identity too.)
template <typename S2>
__global__ void k_identity(Lat L, S2* __restrict__ U) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)field_elems(L)) return;
  const int N = L.N;
  const int e = (int)((t >> 5) % (N * N));
  const int i = e / N, j = e - i * N;
  stc(U + t, mkc<double>(i == j ? 1.0 : 0.0, 0.0));
}

// Complex Gaussian matrices (unit variance per component pair) for the Haar
// hot start; counter (0x48000000 | j, l_lo, l_hi, 0) keeps them apart from
// the momentum stream.  A reunitarisation pass (MGS rows + det phase) turns
// them into Haar-distributed SU(N) links.
template <typename S2>
__global__ void k_gauss_matrices(Lat L, S2* __restrict__ U, uint64_t seed) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)L.V * L.D) return;
  const int N = L.N;
  const int d = (int)(t / L.V);
  const int s = (int)(t - (long)d * L.V);
  const unsigned long long lk = (unsigned long long)s * L.D + d;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int e0 = 0; e0 < N * N; e0 += 2) {
    u32x4 c;
    c.x = 0x48000000u | (uint32_t)(e0 >> 1);
    c.y = (uint32_t)lk;
    c.z = (uint32_t)(lk >> 32);
    c.w = 0u;
    double g[4];
    normals4(philox4x32_10(c, k0, k1), g);
    stc(U + eoff(L, d, e0, s), mkc<double>(g[0], g[1]));
    if (e0 + 1 < N * N) stc(U + eoff(L, d, e0 + 1, s), mkc<double>(g[2], g[3]));
  }
}

// Device-side trajectory bookkeeping.  The Metropolis test of sun.cpp:1249-1318
// in FP64: H = beta * (EnergyMag + simpleenergyEl / (2 NC)); accept when
// H_new < H_old (case 1) or u < exp(H_old - H_new) (case 2), u a Philox uniform
// with counter (0xFFFFFFFF, 0, 0, traj).
struct TrajState {
  double h_old;
  double h_new;
  double dh;
  double u;
  int accepted;  // 0 reject, 1 case 1, 2 case 2
  int pad;
  unsigned long long traj;  // trajectory counter (momentum refresh / Metropolis stream)
  unsigned long long n_acc, n_acc1, n_rej, n_tot;
};

// sums: [0] = action (temporal), [1] = action (spatial), [2] = kinetic
static __global__ void k_energy(const double* __restrict__ sums, double beta, int N, double* __restrict__ h_out) {
  *h_out = beta * ((sums[0] + sums[1]) + sums[2] / (2.0 * N));
}

__device__ __forceinline__ void metropolis(TrajState* st, uint64_t seed, double* __restrict__ log_out, int log_cap) {
  const double hn = st->h_new, ho = st->h_old;
  u32x4 c;
  c.x = 0xFFFFFFFFu;
  c.y = 0u;
  c.z = 0u;
  c.w = (uint32_t)st->traj;
  const u32x4 w = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double u = u01(w.x);
  int acc = 0;
  if (hn < ho)
    acc = 1;
  else if (u < exp(-hn + ho))
    acc = 2;
  st->dh = hn - ho;
  st->u = u;
  st->accepted = acc;
  st->n_tot++;
  if (acc) st->n_acc++;
  if (acc == 1) st->n_acc1++;
  if (!acc) st->n_rej++;
  if (log_out && log_cap > 0) {
    const unsigned long long k = st->traj % (unsigned long long)log_cap;
    log_out[4 * k + 0] = ho;
    log_out[4 * k + 1] = hn;
    log_out[4 * k + 2] = hn - ho;
    log_out[4 * k + 3] = (double)acc;
  }
  st->traj++;
}

static __global__ void k_metropolis(TrajState* st, uint64_t seed, double* __restrict__ log_out, int log_cap) {
  metropolis(st, seed, log_out, log_cap);
}

// takeconfiguration / loadconfiguration (sun.cpp:725-742) after the test:
// accepted -> Uconf = U, rejected -> U = Uconf.  Vectorised 16-byte copy.
static __global__ void k_accept_copy(const TrajState* __restrict__ st, uint4* __restrict__ U, uint4* __restrict__ Uconf,
                              long n16) {
  const bool acc = st->accepted != 0;
  uint4* dst = acc ? Uconf : U;
  const uint4* src = acc ? U : Uconf;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// Conversion between the host U-conf layout (FP64, [site][dir][row][col][re,im])
// and the device layout in either precision.
template <typename S2>
__global__ void k_from_conf(Lat L, const double2* __restrict__ conf, S2* __restrict__ f) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)field_elems(L)) return;
  // t indexes the device field: t = ((d*B + b)*NN + e)*32 + lane, site = 32b + lane
  const int NN = L.N * L.N;
  const long rest = t >> 5;
  const int e = (int)(rest % NN);
  const long db = rest / NN;
  const int d = (int)(db / L.B);
  const int s = (int)((db - (long)d * L.B) * 32 + (t & 31));
  if (s >= L.V) {
    stc(f + t, mkc<double>(0.0, 0.0));
    return;
  }
  const double2 v = conf[((size_t)s * L.D + d) * NN + e];
  stc(f + t, mkc<double>(v.x, v.y));
}

template <typename S2>
__global__ void k_to_conf(Lat L, const S2* __restrict__ f, double2* __restrict__ conf) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int NN = L.N * L.N;
  const long tot = (long)L.V * L.D * NN;
  if (t >= tot) return;
  // t indexes the conf output: t = (s*D + d)*NN + e
  const long lk = t / NN;
  const int e = (int)(t - lk * NN);
  const int s = (int)(lk / L.D);
  const int d = (int)(lk - (long)s * L.D);
  const cpx<double> v = ldc<double>(f + eoff(L, d, e, s));
  conf[t] = make_double2(v.re, v.im);
}

// Non-finite scan of a host-uploaded U-conf buffer: counts NaN/Inf doubles.
static __global__ void k_count_nonfinite(const double* __restrict__ x, long n, unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    if (!isfinite(x[i])) c++;
  if (c) atomicAdd(count, c);
}

// ---- large colour number (NC >= BIG_NC): one CTA per site or per link ----
// The thread-per-site / thread-per-link kernels above carry O(NC^3) / O(NC^2)
// serial work per thread, which leaves a lattice of a few thousand sites with
// a few thousand threads; these spread one site or link over a CTA.

constexpr int BIG_NC = 16;

// Plaquette sums of one site (same sums as plaq_site): B = U_nu(x+mu) and
// C = U_mu(x+nu) staged in shared memory as FP64 ([N][N+1]), thread t owns row
// t / 4 and the columns j = 4q + t % 4 of AB and DC (A = U_mu(x), D = U_nu(x)
// read from global), tr = sum Re (AB)_ij conj((DC)_ij); partial[s*2 + {0,1}].
template <typename S2>
__global__ void __launch_bounds__(RED_THREADS) k_plaq_big(Lat L, const S2* __restrict__ U, double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = L.N, NP = N + 1;
  cpx<double>* Bs = reinterpret_cast<cpx<double>*>(smem_raw);
  cpx<double>* Cs = Bs + N * NP;
  const int s = blockIdx.x;
  const int tid = threadIdx.x;
  const int rows_per_pass = RED_THREADS / 4;
  double trt = 0.0, trs = 0.0;
  int nt = 0, ns = 0;
  for (int mu = 0; mu < L.D; mu++) {
    const int xpmu = nb_plus(L, mu, s);
    for (int nu = mu + 1; nu < L.D; nu++) {
      const int xpnu = nb_plus(L, nu, s);
      __syncthreads();
      for (int e = tid; e < N * N; e += RED_THREADS) {
        const int r = e / N, c = e - (e / N) * N;
        Bs[r * NP + c] = ldc<double>(U + eoff(L, nu, e, xpmu));
        Cs[r * NP + c] = ldc<double>(U + eoff(L, mu, e, xpnu));
      }
      __syncthreads();
      double tr = 0.0;
      for (int i0 = 0; i0 < N; i0 += rows_per_pass) {
        const int i = i0 + tid / 4;
        if (i >= N) continue;
        cpx<double> ab[16], dc[16];
#pragma unroll
        for (int q = 0; q < 16; q++) ab[q] = dc[q] = czero<double>();
        for (int k = 0; k < N; k++) {
          const cpx<double> a = ldc<double>(U + eoff(L, mu, i * N + k, s));
          const cpx<double> d = ldc<double>(U + eoff(L, nu, i * N + k, s));
#pragma unroll
          for (int q = 0; q < 16; q++) {
            const int j = 4 * q + (tid & 3);
            if (j < N) {
              cmac(ab[q], a, Bs[k * NP + j]);
              cmac(dc[q], d, Cs[k * NP + j]);
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 16; q++) {
          tr = fma(ab[q].re, dc[q].re, tr);
          tr = fma(ab[q].im, dc[q].im, tr);
        }
      }
      if (mu == 0) {
        trt += tr;
        nt++;
      } else {
        trs += tr;
        ns++;
      }
    }
  }
  double v[2] = {trt, trs};
  block_sum<2>(v);
  if (tid == 0) {
    const bool in = counted(L, s);
    partial[(size_t)s * 2 + 0] = in ? nt - v[0] / N : 0.0;
    partial[(size_t)s * 2 + 1] = in ? ns - v[1] / N : 0.0;
  }
}

// link_sums of one link per CTA; partial[t*3 + k]
template <typename S2>
__global__ void __launch_bounds__(RED_THREADS) k_linksums_big(Lat L, const S2* __restrict__ Pa,
                                                              const S2* __restrict__ Pb, const S2* __restrict__ U,
                                                              double* __restrict__ partial) {
  const int N = L.N;
  const long t = blockIdx.x;
  const int d = (int)(t / L.V);
  const int s = (int)(t - (long)d * L.V);
  double a = 0.0, b = 0.0, c = 0.0;
  for (int e = threadIdx.x; e < N * N; e += RED_THREADS) {
    const int i = e / N, j = e - (e / N) * N;
    if (Pa) {
      const cpx<double> x = ldc<double>(Pa + eoff(L, d, i * N + j, s));
      const cpx<double> y = ldc<double>(Pa + eoff(L, d, j * N + i, s));
      a = fma(x.re, y.re, a);
      a = fma(-x.im, y.im, a);
      if (Pb) {
        const cpx<double> x2 = ldc<double>(Pb + eoff(L, d, i * N + j, s));
        const cpx<double> y2 = ldc<double>(Pb + eoff(L, d, j * N + i, s));
        b = fma(x.re + x2.re, y.re + y2.re, b);
        b = fma(-(x.im + x2.im), y.im + y2.im, b);
      }
    }
    if (U) {
      cpx<double> aij = czero<double>(), aji = czero<double>();
      for (int k = 0; k < N; k++) {
        cmac_nc(aij, ldc<double>(U + eoff(L, d, i * N + k, s)), ldc<double>(U + eoff(L, d, j * N + k, s)));
        cmac_nc(aji, ldc<double>(U + eoff(L, d, j * N + k, s)), ldc<double>(U + eoff(L, d, i * N + k, s)));
      }
      if (i == j) {
        aij.re -= 1.0;
        aji.re -= 1.0;
      }
      c = fma(aij.re, aji.re, c);
      c = fma(-aij.im, aji.im, c);
    }
  }
  double v[3] = {a, 0.25 * b, c};
  block_sum<3>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; k++) partial[(size_t)t * 3 + k] = counted(L, s) ? v[k] : 0.0;
}

// refresh_link with one CTA per link: thread per off-diagonal pair (the pair's
// two normals come from one Philox block), the diagonal by thread 0 in the
// same order as refresh_link, so the momenta are identical.
template <typename S2>
__global__ void k_refresh_big(Lat L, S2* __restrict__ P, uint64_t seed, const unsigned long long* __restrict__ traj_dev,
                              unsigned long long traj_host, double scale) {
  const uint32_t traj = (uint32_t)(traj_dev ? *traj_dev : traj_host);
  const int N = L.N;
  const long t = blockIdx.x;
  const int d = (int)(t / L.V);
  const int s = (int)(t - (long)d * L.V);
  const unsigned long long lk = (unsigned long long)s * L.D + d;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  auto block = [&](int blk, double (&g)[4]) {
    u32x4 c;
    c.x = (uint32_t)blk;
    c.y = (uint32_t)lk;
    c.z = (uint32_t)(lk >> 32);
    c.w = traj;
    normals4(philox4x32_10(c, k0, k1), g);
  };
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int i = e / N, j = e - (e / N) * N;
    if (j <= i) continue;
    const int p = i * (2 * N - i - 1) / 2 + (j - i - 1);
    double g[4];
    block((2 * p) >> 2, g);
    const double xs = g[(2 * p) & 3], xa = g[(2 * p + 1) & 3];
    stc(P + eoff(L, d, i * N + j, s), mkc<double>(0.5 * scale * xs, -0.5 * scale * xa));
    stc(P + eoff(L, d, j * N + i, s), mkc<double>(0.5 * scale * xs, 0.5 * scale * xa));
  }
  if (threadIdx.x == 0) {
    const int a0 = N * (N - 1);
    int cur = -1;
    double g[4];
    double suffix = 0.0;
    for (int dd = N - 1; dd >= 0; dd--) {
      double val = suffix;
      if (dd >= 1) {
        const int m = dd - 1;
        const double nm = sqrt(0.5 / ((double)(m + 1) * (m + 2)));
        const int a = a0 + m;
        if ((a >> 2) != cur) {
          block(a >> 2, g);
          cur = a >> 2;
        }
        const double xm = g[a & 3];
        val -= dd * nm * xm;
        suffix += nm * xm;
      }
      stc(P + eoff(L, d, dd * N + dd, s), mkc<double>(scale * val, 0.0));
    }
  }
}

}  // namespace misc
}  // namespace askja
