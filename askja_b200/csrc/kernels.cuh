// Template body of a KernelSet for one storage precision.  Included once by
// kernels_fp64.cu (T = double) and once by kernels_fp32.cu (T = float).
#pragma once

#include <algorithm>

#include "launch.h"
#include "misc.cuh"
#include "rows.cuh"
#include "small.cuh"
#include "pair.cuh"
#include "tab.cuh"
#include "eig.cuh"
#include "tc.cuh"

namespace askja {

namespace detail {

constexpr int SMALL_THREADS = 128;
constexpr size_t ROWS_SMEM_BUDGET = 200 * 1024;

inline long nlinks(const Lat& L) { return (long)L.V * L.D; }
inline unsigned blocks_for(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <typename T>
struct Rows {
  // groups per block and dynamic shared memory for the row-per-thread kernels
  static void shape(int N, int* G, size_t* smem, int want = 0) {
    const size_t per = rows::smem_per_group<T>(N);
    int g = want > 0 ? want : std::max(1, 128 / N);
    // at most 256 threads: launchable at any register count up to 255
    g = std::min(g, std::max(1, 256 / N));
    g = std::min(g, 64);
    while (g > 1 && (size_t)g * per > ROWS_SMEM_BUDGET) g--;
    *G = g;
    *smem = (size_t)g * per;
  }
};

// Opt in to the dynamic shared memory a launch needs (the kernels also have
// static shared arrays, so the 48 KB default can be exceeded below 48 KB of
// dynamic memory).
template <typename Kern>
cudaError_t set_smem(Kern k, size_t smem) {
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int NMAX, typename T>
cudaError_t rows_force(const LaunchCtx& c, int mode, const void* U, const void* Pin, void* Pout, void* Uout,
                       double ek, double ed) {
  using S2 = typename Storage<T>::type;
  int G;
  size_t smem;
  Rows<T>::shape(c.lat.N, &G, &smem, c.rows_groups);
  // G consecutive sites of one direction per CTA, all directions of a site block adjacent
  const unsigned grid = blocks_for(c.lat.V, G) * c.lat.D;
  cudaError_t e;
  if (mode == 0) {
    auto k = rows::k_force<NMAX, T, S2, 0>;
    if ((e = set_smem(k, smem)) != cudaSuccess) return e;
    k<<<grid, G * c.lat.N, smem, c.stream>>>(c.lat, (const S2*)U, (const S2*)Pin, (S2*)Pout, (S2*)Uout, (T)ek, (T)ed,
                                             c.order, c.reunit);
  } else {
    auto k = rows::k_force<NMAX, T, S2, 1>;
    if constexpr (sizeof(T) == 4 && NMAX == 8)
      k = c.small_occ == 2 ? rows::k_force8<S2, 1, 2> : c.small_occ == 1 ? rows::k_force8<S2, 1, 1> : rows::k_force8<S2, 1, 0>;
    if ((e = set_smem(k, smem)) != cudaSuccess) return e;
    // reunit 2: Newton-Schulz projection (FP32 single chains, see LaunchCtx::rows_ns)
    const int ru = (sizeof(T) == 4 && c.reunit && c.rows_ns) ? 2 : c.reunit;
    k<<<grid, G * c.lat.N, smem, c.stream>>>(c.lat, (const S2*)U, (const S2*)Pin, (S2*)Pout, (S2*)Uout, (T)ek, (T)ed,
                                             c.order, ru);
  }
  return cudaGetLastError();
}

template <int NMAX, typename T>
cudaError_t rows_drift(const LaunchCtx& c, void* U, const void* P, double eps) {
  using S2 = typename Storage<T>::type;
  int G;
  size_t smem;
  Rows<T>::shape(c.lat.N, &G, &smem, c.rows_groups);
  auto k = rows::k_drift<NMAX, T, S2>;
  cudaError_t e;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  k<<<blocks_for(nlinks(c.lat), G), G * c.lat.N, smem, c.stream>>>(c.lat, (S2*)U, (const S2*)P, (T)eps, c.order,
                                                                     c.reunit);
  return cudaGetLastError();
}

template <int N, typename T>
cudaError_t small_force(const LaunchCtx& c, int mode, const void* U, const void* Pin, void* Pout, void* Uout,
                        double ek, double ed) {
  using S2 = typename Storage<T>::type;
  // site tiles: 32 sites per CTA, one warp per direction (warps loop when DIM > 4)
  const unsigned grid = blocks_for(c.lat.V, 32);
  const int threads = 32 * std::min(c.lat.D, 4);
  const S2* u = (const S2*)U;
  const S2* pi = (const S2*)Pin;
  if (c.small_occ == 2) {
    if (mode == 0)
      small::k_force_occ<N, T, S2, 0, 2><<<grid, threads, 0, c.stream>>>(c.lat, u, pi, (S2*)Pout, (S2*)Uout, (T)ek,
                                                                           (T)ed, c.order, c.reunit);
    else
      small::k_force_occ<N, T, S2, 1, 2><<<grid, threads, 0, c.stream>>>(c.lat, u, pi, (S2*)Pout, (S2*)Uout, (T)ek,
                                                                           (T)ed, c.order, c.reunit);
  } else if (c.small_occ) {
    if (mode == 0)
      small::k_force_occ<N, T, S2, 0><<<grid, threads, 0, c.stream>>>(c.lat, u, pi, (S2*)Pout, (S2*)Uout, (T)ek,
                                                                        (T)ed, c.order, c.reunit);
    else
      small::k_force_occ<N, T, S2, 1><<<grid, threads, 0, c.stream>>>(c.lat, u, pi, (S2*)Pout, (S2*)Uout, (T)ek,
                                                                        (T)ed, c.order, c.reunit);
  } else if (mode == 0) {
    small::k_force<N, T, S2, 0><<<grid, threads, 0, c.stream>>>(c.lat, u, pi, (S2*)Pout, (S2*)Uout, (T)ek, (T)ed,
                                                                c.order, c.reunit);
  } else {
    small::k_force<N, T, S2, 1><<<grid, threads, 0, c.stream>>>(c.lat, u, pi, (S2*)Pout, (S2*)Uout, (T)ek, (T)ed,
                                                                c.order, c.reunit);
  }
  return cudaGetLastError();
}

template <int N, typename T>
cudaError_t small_drift(const LaunchCtx& c, void* U, const void* P, double eps) {
  using S2 = typename Storage<T>::type;
  small::k_drift<N, T, S2><<<blocks_for(nlinks(c.lat), SMALL_THREADS), SMALL_THREADS, 0, c.stream>>>(
      c.lat, (S2*)U, (const S2*)P, (T)eps, c.order, c.reunit);
  return cudaGetLastError();
}

// Tensor-core link update (FP32 storage): per-link copy of U into the
// scratch buffer, then one persistent launch over all links.
// mode 0 kick, 1 kick + drift, 2 drift only (Uout may be U).
template <int NC>
cudaError_t tc_link(const LaunchCtx& c, int mode, const void* U, const void* Pin, void* Pout, void* Uout, double ek,
                    double ed) {
  const Lat& L = c.lat;
  if (!c.scratch || !c.status) return cudaErrorInvalidValue;
  float2* aos = static_cast<float2*>(c.scratch);
  int dev = 0, nsm = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int chunks = (NC * NC + 31) / 32;
  const int z = std::max(1, std::min(chunks, (4 * nsm + L.B * L.D - 1) / (L.B * L.D)));
  tc::k_to_aos<<<dim3(L.B, L.D, z), 256, 0, c.stream>>>(L, static_cast<const float2*>(U), aos);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  auto k = mode == 0 ? tc::k_link<NC, 0> : mode == 1 ? tc::k_link<NC, 1> : tc::k_link<NC, 2>;
  const size_t smem = tc::Shape<NC>::SMEM;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  // the whole unified L1/shared array as shared memory, so that as many CTAs
  // as registers and shared memory allow are resident (TMEM: 4 NC columns
  // each; shared memory admits at most 4 CTAs of NC = 32 and 1 of NC = 64,
  // so the allocations never exceed the 512 columns of an SM)
  if ((e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
    return e;
  // resident CTAs per SM from registers, shared memory, threads and tensor
  // memory (the occupancy query reports 1 for these kernels)
  cudaFuncAttributes fa{};
  if ((e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess) return e;
  int smem_sm = 0, smem_rsv = 0, regs_sm = 0;
  if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess) return e;
  const int regs = (std::max(fa.numRegs, 1) + 7) / 8 * 8;
  int per = std::min(regs_sm / (regs * tc::THREADS), smem_sm / (int)(smem + fa.sharedSizeBytes + smem_rsv));
  per = std::min(per, 2048 / tc::THREADS);
  per = std::max(1, std::min(per, 512 / tc::Shape<NC>::TMEM_COLS));
  const long grid = std::min(nlinks(L), (long)nsm * per);
  k<<<(unsigned)grid, tc::THREADS, smem, c.stream>>>(L, aos, static_cast<const float2*>(Pin),
                                                      static_cast<float2*>(Pout), static_cast<float2*>(Uout),
                                                      (float)ek, (float)ed, c.order, c.reunit, c.status);
  return cudaGetLastError();
}

template <typename T>
cudaError_t tc_dispatch(const LaunchCtx& c, int mode, const void* U, const void* Pin, void* Pout, void* Uout,
                        double ek, double ed) {
  if constexpr (sizeof(T) == 4) {
    if (c.lat.N == 16) return tc_link<16>(c, mode, U, Pin, Pout, Uout, ek, ed);
    if (c.lat.N == 32) return tc_link<32>(c, mode, U, Pin, Pout, Uout, ek, ed);
    if (c.lat.N == 64) return tc_link<64>(c, mode, U, Pin, Pout, Uout, ek, ed);
  }
  return cudaErrorInvalidValue;
}

// Fused kick+drift on site pairs (FP32 SU(3)); U, P and Uout in the site-pair
// layout, P updated in place.
template <typename T>
cudaError_t pair_force(const LaunchCtx& c, const void* U, const void* Pin, void* Pout, void* Uout, double ek,
                       double ed) {
  if constexpr (sizeof(T) == 4) {
    if (Pin != Pout || !pair_supported(c.lat.N, c.lat.D, false, c.lat.n[c.lat.D - 1])) return cudaErrorInvalidValue;
    const unsigned grid = blocks_for(c.lat.V, 64);
    const int threads = 32 * std::min(c.lat.D, 4);
    auto k = c.small_occ ? pair::k_force_pair<1> : pair::k_force_pair<0>;
    k<<<grid, threads, 0, c.stream>>>(c.lat, (const float2*)U, (float2*)Pout, (float2*)Uout, (float)ek, (float)ed,
                                      c.order, c.reunit);
    return cudaGetLastError();
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t pair_swap(const LaunchCtx& c, void* f) {
  if constexpr (sizeof(T) == 4) {
    const long n4 = (long)(field_elems(c.lat) / 2);
    pair::k_pair_swap<<<(unsigned)std::min<long>(blocks_for(n4, 256), 148L * 16), 256, 0, c.stream>>>((float4*)f, n4);
    return cudaGetLastError();
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t force(const LaunchCtx& c, int mode, const void* U, const void* Pin, void* Pout, void* Uout, double ek,
                  double ed) {
  const int N = c.lat.N;
  if (c.force_rows == 2 && tc_supported(N, c.lat.D, sizeof(T) == 8))
    return tc_dispatch<T>(c, mode, U, Pin, Pout, Uout, ek, ed);
  if (c.force_rows == 3 && mode == 1) return pair_force<T>(c, U, Pin, Pout, Uout, ek, ed);
  if (!c.force_rows || c.force_rows == 3) {
    if (N == 2) return small_force<2, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
    if (N == 3) return small_force<3, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
    if (N == 4) return small_force<4, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
  }
  if (N <= 8) return rows_force<8, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
  if (N <= 16) return rows_force<16, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
  if (N <= 32) return rows_force<32, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
  if (N <= 64) return rows_force<64, T>(c, mode, U, Pin, Pout, Uout, ek, ed);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t drift(const LaunchCtx& c, void* U, const void* P, double eps) {
  const int N = c.lat.N;
  if (c.force_rows == 2 && tc_supported(N, c.lat.D, sizeof(T) == 8))
    return tc_dispatch<T>(c, 2, U, P, nullptr, U, 0.0, eps);
  if (!c.force_rows || c.force_rows == 3) {
    if (N == 2) return small_drift<2, T>(c, U, P, eps);
    if (N == 3) return small_drift<3, T>(c, U, P, eps);
    if (N == 4) return small_drift<4, T>(c, U, P, eps);
  }
  if (N <= 8) return rows_drift<8, T>(c, U, P, eps);
  if (N <= 16) return rows_drift<16, T>(c, U, P, eps);
  if (N <= 32) return rows_drift<32, T>(c, U, P, eps);
  if (N <= 64) return rows_drift<64, T>(c, U, P, eps);
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t reunit(const LaunchCtx& c, void* U) {
  using S2 = typename Storage<T>::type;
  const int N = c.lat.N;
  const unsigned gsm = blocks_for(nlinks(c.lat), SMALL_THREADS);
  if (!c.force_rows || c.force_rows == 3) {
    if (N == 2) {
      small::k_reunit<2, T, S2><<<gsm, SMALL_THREADS, 0, c.stream>>>(c.lat, (S2*)U);
      return cudaGetLastError();
    }
    if (N == 3) {
      small::k_reunit<3, T, S2><<<gsm, SMALL_THREADS, 0, c.stream>>>(c.lat, (S2*)U);
      return cudaGetLastError();
    }
    if (N == 4) {
      small::k_reunit<4, T, S2><<<gsm, SMALL_THREADS, 0, c.stream>>>(c.lat, (S2*)U);
      return cudaGetLastError();
    }
  }
  int G;
  size_t smem;
  Rows<T>::shape(N, &G, &smem);
  auto k = rows::k_reunit<T, S2>;
  cudaError_t e;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  k<<<blocks_for(nlinks(c.lat), G), G * N, smem, c.stream>>>(c.lat, (S2*)U, c.gate, c.gate_every);
  return cudaGetLastError();
}

template <typename T>
cudaError_t plaq(const LaunchCtx& c, const void* U, double* partial, double* out) {
  using S2 = typename Storage<T>::type;
  const int N = c.lat.N;
  if (N >= misc::BIG_NC) {
    auto k = misc::k_plaq_big<S2>;
    const size_t smem = 2 * (size_t)N * (N + 1) * sizeof(cpx<double>);
    cudaError_t e;
    if ((e = set_smem(k, smem)) != cudaSuccess) return e;
    k<<<c.lat.V, misc::RED_THREADS, smem, c.stream>>>(c.lat, (const S2*)U, partial);
    misc::k_finish<2><<<1, misc::RED_THREADS, 0, c.stream>>>(partial, c.lat.V, out);
    return cudaGetLastError();
  }
  const unsigned nb = blocks_for(c.lat.V, misc::RED_THREADS);
  if (N == 2)
    misc::k_plaq<2, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)U, partial);
  else if (N == 3)
    misc::k_plaq<3, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)U, partial);
  else if (N == 4)
    misc::k_plaq<4, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)U, partial);
  else
    misc::k_plaq<0, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)U, partial);
  misc::k_finish<2><<<1, misc::RED_THREADS, 0, c.stream>>>(partial, (int)nb, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t linksums(const LaunchCtx& c, const void* Pa, const void* Pb, const void* U, double* partial, double* out) {
  using S2 = typename Storage<T>::type;
  const int N = c.lat.N;
  if (N >= misc::BIG_NC) {
    misc::k_linksums_big<S2><<<(unsigned)nlinks(c.lat), misc::RED_THREADS, 0, c.stream>>>(
        c.lat, (const S2*)Pa, (const S2*)Pb, (const S2*)U, partial);
    misc::k_finish<3><<<1, misc::RED_THREADS, 0, c.stream>>>(partial, (int)nlinks(c.lat), out);
    return cudaGetLastError();
  }
  const unsigned nb = blocks_for(nlinks(c.lat), misc::RED_THREADS);
  if (N == 2)
    misc::k_linksums<2, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)Pa, (const S2*)Pb,
                                                                    (const S2*)U, partial);
  else if (N == 3)
    misc::k_linksums<3, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)Pa, (const S2*)Pb,
                                                                    (const S2*)U, partial);
  else if (N == 4)
    misc::k_linksums<4, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)Pa, (const S2*)Pb,
                                                                    (const S2*)U, partial);
  else
    misc::k_linksums<0, S2><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)Pa, (const S2*)Pb,
                                                                    (const S2*)U, partial);
  misc::k_finish<3><<<1, misc::RED_THREADS, 0, c.stream>>>(partial, (int)nb, out);
  return cudaGetLastError();
}

constexpr int GAUSS_LINKS_PER_BLOCK = 256;

template <typename T>
cudaError_t gauss(const LaunchCtx& c, const void* U, const void* Pi, double* partial, double* out) {
  using S2 = typename Storage<T>::type;
  const unsigned nb = blocks_for(nlinks(c.lat), GAUSS_LINKS_PER_BLOCK);
  const int NN = c.lat.N * c.lat.N;
  const int thr = std::min(misc::RED_THREADS, ((NN + 31) / 32) * 32);
  misc::k_gauss<S2><<<nb, thr, 0, c.stream>>>(c.lat, (const S2*)U, (const S2*)Pi, GAUSS_LINKS_PER_BLOCK, partial);
  misc::k_gauss_finish<<<1, thr, 2 * NN * sizeof(double), c.stream>>>(partial, (int)nb, c.lat.N, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t lines(const LaunchCtx& c, const void* U, int dir, int nlines, int start_stride, double* out) {
  using S2 = typename Storage<T>::type;
  const int N = c.lat.N;
  const size_t smem = 2 * (size_t)N * N * sizeof(cpx<double>);
  auto k = misc::k_lines<S2>;
  cudaError_t e;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  k<<<nlines, ((N + 31) / 32) * 32, smem, c.stream>>>(c.lat, (const S2*)U, dir, start_stride, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t slice_trace(const LaunchCtx& c, const void* U, double* out) {
  using S2 = typename Storage<T>::type;
  misc::k_slice_trace<S2><<<c.lat.n[0], misc::RED_THREADS, 0, c.stream>>>(c.lat, (const S2*)U, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t line_eigs(const LaunchCtx& c, const void* U, int dir, int nlines, int start_stride, double2* ev,
                      int* fail) {
  using S2 = typename Storage<T>::type;
  const int N = c.lat.N;
  const size_t smem = 2 * (size_t)N * N * sizeof(cpx<double>);
  auto k = eig::k_line_eigs<S2>;
  cudaError_t e;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  k<<<nlines, std::max(32, (N + 31) / 32 * 32), smem, c.stream>>>(c.lat, (const S2*)U, dir, start_stride, ev, fail);
  return cudaGetLastError();
}

template <typename T>
cudaError_t refresh(const LaunchCtx& c, void* P, uint64_t seed, const unsigned long long* traj_dev,
                    unsigned long long traj_host, double scale) {
  using S2 = typename Storage<T>::type;
  if (c.lat.N >= misc::BIG_NC) {
    misc::k_refresh_big<S2><<<(unsigned)nlinks(c.lat), misc::RED_THREADS, 0, c.stream>>>(c.lat, (S2*)P, seed, traj_dev,
                                                                                         traj_host, scale);
    return cudaGetLastError();
  }
  misc::k_refresh<S2><<<blocks_for(nlinks(c.lat), 128), 128, 0, c.stream>>>(c.lat, (S2*)P, seed, traj_dev, traj_host,
                                                                              scale);
  return cudaGetLastError();
}

template <typename T>
cudaError_t identity(const LaunchCtx& c, void* U) {
  using S2 = typename Storage<T>::type;
  const long tot = (long)field_elems(c.lat);
  misc::k_identity<S2><<<blocks_for(tot, 256), 256, 0, c.stream>>>(c.lat, (S2*)U);
  return cudaGetLastError();
}

template <typename T>
cudaError_t gauss_matrices(const LaunchCtx& c, void* U, uint64_t seed) {
  using S2 = typename Storage<T>::type;
  misc::k_gauss_matrices<S2><<<blocks_for(nlinks(c.lat), 128), 128, 0, c.stream>>>(c.lat, (S2*)U, seed);
  return cudaGetLastError();
}

template <typename T>
cudaError_t from_conf(const LaunchCtx& c, const void* conf, void* f) {
  using S2 = typename Storage<T>::type;
  const long tot = (long)field_elems(c.lat);
  misc::k_from_conf<S2><<<blocks_for(tot, 256), 256, 0, c.stream>>>(c.lat, (const double2*)conf, (S2*)f);
  return cudaGetLastError();
}

template <typename T>
cudaError_t to_conf(const LaunchCtx& c, const void* f, void* conf) {
  using S2 = typename Storage<T>::type;
  const long tot = nlinks(c.lat) * c.lat.N * c.lat.N;
  misc::k_to_conf<S2><<<blocks_for(tot, 256), 256, 0, c.stream>>>(c.lat, (const S2*)f, (double2*)conf);
  return cudaGetLastError();
}

// FourierTrafo (sun.cpp:365-411): plaquette energy of sites 0..n-1 (one CTA
// per site), then |inverse DFT| of that sequence into coef[0..n-1].
template <typename T>
cudaError_t fourier(const LaunchCtx& c, const void* U, int n, double* partial, double* coef) {
  using S2 = typename Storage<T>::type;
  auto k = misc::k_plaq_big<S2>;
  const size_t smem = 2 * (size_t)c.lat.N * (c.lat.N + 1) * sizeof(cpx<double>);
  cudaError_t e;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  k<<<n, misc::RED_THREADS, smem, c.stream>>>(c.lat, (const S2*)U, partial);
  tab::k_dft_abs<<<blocks_for(n, 128), 128, 0, c.stream>>>(partial, n, coef);
  return cudaGetLastError();
}

// Tab (sun.cpp:580-670) for sites site0 .. site0+nsites-1: out[k*npt + m]
template <typename T>
cudaError_t tab_sites(const LaunchCtx& c, const void* U, const void* Pa, const void* Pb, int site0, int nsites,
                      int npt, double* out) {
  using S2 = typename Storage<T>::type;
  if (c.lat.D > tab::TAB_MAX_D || c.lat.N > 64 || npt < 2 || npt > c.lat.D + 2) return cudaErrorInvalidValue;
  auto k = tab::k_tab<S2>;
  const size_t smem = tab::tab_smem(c.lat.N);
  cudaError_t e;
  if ((e = set_smem(k, smem)) != cudaSuccess) return e;
  const int threads = 32 * ((c.lat.N + 31) / 32);
  k<<<nsites, threads, smem, c.stream>>>(c.lat, (const S2*)U, (const S2*)Pa, (const S2*)Pb, site0, npt, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t wait_probe(const LaunchCtx& c, long long cycles) {
  if constexpr (sizeof(T) == 4) {
    if (!c.status) return cudaErrorInvalidValue;
    if (c.lat.N == 32) {
      tc::k_wait_probe<32><<<1, tc::THREADS, 0, c.stream>>>(c.status, cycles);
      return cudaGetLastError();
    }
    if (c.lat.N == 64) {
      tc::k_wait_probe<64><<<1, tc::THREADS, 0, c.stream>>>(c.status, cycles);
      return cudaGetLastError();
    }
  }
  return cudaErrorInvalidValue;
}

template <typename T>
constexpr KernelSet make_set() {
  return KernelSet{&force<T>,   &drift<T>,   &reunit<T>,  &plaq<T>,           &linksums<T>,  &gauss<T>, &lines<T>,
                   &slice_trace<T>, &line_eigs<T>, &refresh<T>, &identity<T>, &gauss_matrices<T>, &from_conf<T>, &to_conf<T>, &pair_swap<T>, &fourier<T>, &tab_sites<T>,
                   &wait_probe<T>};
}

}  // namespace detail

}  // namespace askja
