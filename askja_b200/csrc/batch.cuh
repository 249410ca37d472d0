// Kernels that advance many independent Markov chains of uneven shape (NC,
// DIM, extents, BETA, DT) together.  Every launch covers all chains (of one
// colour number for the force) through a work list: work item i belongs to
// the chain c with item_start[c] <= i < item_start[c+1] (the force launches,
// which run every MD step, read (chain, item within the chain) from a per-item
// table instead); the CTA takes that chain's descriptor and runs the same
// per-link / per-site code as the single-chain kernels (small.cuh, rows.cuh,
// split.cuh, misc.cuh).  Chains of different sizes therefore share the GPU in
// proportion to their work.
#pragma once

#include <type_traits>

#include "misc.cuh"
#include "rows.cuh"
#include "small.cuh"
#include "split.cuh"

namespace askja {
namespace batch {

struct ChainDev {
  Lat lat;
  void* U[2];
  void* P;
  void* Uconf;
  double dt;
  double beta;
  double scale;  // sqrt(2 NC / beta)
  int order;
  int reunit;
  uint64_t seed;
  misc::TrajState* st;
  double* sums;     // 8 doubles: [0,1] plaquette t/s, [2..4] link sums
  double* partial;  // this chain's reduction partials
  int plaq_blocks;  // RED_THREADS-site blocks
  int link_blocks;  // RED_THREADS-link blocks
  long n16;         // field size in 16-byte units
  // residual-plane FP32 mode (FP32 chains with NC <= 4; null otherwise): link
  // residuals, momentum coordinates and their residuals (split.cuh)
  void* UL[2];
  void* ULconf;
  void* PC;
  void* PCL;
  long n16lo;       // residual field size in 16-byte units
};

// chain owning work item i (item_start has nchains+1 entries, ascending)
__device__ __forceinline__ int find_chain(const int* __restrict__ item_start, int nchains, int i) {
  int lo = 0, hi = nchains - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(item_start + mid) <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Copies the descriptor of the chain that owns this CTA's work item into
// shared memory; returns the item's index within its chain.  Every thread
// finds the chain (a few cached loads) and the copy is spread over the
// threads one word each, so the CTA's start costs one round of loads instead
// of one thread's serial copy of the whole descriptor.
__device__ __forceinline__ int load_chain(ChainDev& sd, const ChainDev* __restrict__ descs,
                                          const int* __restrict__ item_start, const int* __restrict__ chain_ids,
                                          int nchains) {
  static_assert(sizeof(ChainDev) % 4 == 0, "descriptor copied in 4-byte words");
  const int k = find_chain(item_start, nchains, blockIdx.x);
  const int c = chain_ids ? __ldg(chain_ids + k) : k;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(descs + c);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
  for (int w = threadIdx.x; w < (int)(sizeof(ChainDev) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
  __syncthreads();
  return blockIdx.x - __ldg(item_start + k);
}

// Copies the descriptor of the chain named by this CTA's entry (chain, item)
// of the per-item table into shared memory; returns the item's index within
// its chain (one load instead of load_chain's binary search).
__device__ __forceinline__ int load_chain_at(ChainDev& sd, const ChainDev* __restrict__ descs,
                                             const int2* __restrict__ item_chain) {
  static_assert(sizeof(ChainDev) % 4 == 0, "descriptor copied in 4-byte words");
  const int2 ct = __ldg(item_chain + blockIdx.x);
  const uint32_t* src = reinterpret_cast<const uint32_t*>(descs + ct.x);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
  for (int w = threadIdx.x; w < (int)(sizeof(ChainDev) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
  __syncthreads();
  return ct.y;
}

// Force (+ link update) for the small-NC chains of one colour number: item =
// 32-site tile, 32*min(D,4) threads (see small::k_force).
// BYVAL: the geometry by value, so that the fields the force uses (V, B, D,
// nbr) live in registers instead of being re-read from shared memory at every
// address (costs registers; used where the register budget is fixed anyway)
template <int N, typename T, int MODE, bool BYVAL>
__device__ __forceinline__ void force_small_item(const ChainDev* __restrict__ descs,
                                                 const int* __restrict__ item_start,
                                                 const int* __restrict__ chain_ids, int nchains, int cur,
                                                 double kick_scale) {
  using S2 = typename Storage<T>::type;
  __shared__ ChainDev sd;
  const int tile = load_chain(sd, descs, item_start, chain_ids, nchains);
  using LatRef = typename std::conditional<BYVAL, const Lat, const Lat&>::type;
  LatRef L = sd.lat;
  const int x = tile * 32 + (threadIdx.x & 31);
  if (x >= L.V) return;
  const S2* U = (const S2*)sd.U[cur];
  S2* P = (S2*)sd.P;
  S2* Uo = (S2*)sd.U[cur ^ 1];
  const T ek = (T)(kick_scale * sd.dt), ed = (T)sd.dt;
  const int order = sd.order, reunit = sd.reunit;
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5))
    small::force_link<N, T, S2, MODE>(L, U, P, P, Uo, ek, ed, order, reunit, mu, x);
}

// The residual-plane kernel on the same tiles (split::link_update).  The CTA
// finds its chain and tile in one load from the per-item table (chain, tile)
// and every thread reads the descriptor fields it uses straight from global
// memory (the same few cache lines for the whole CTA): two dependent loads
// before the first link load, where a binary search over the chain starts, a
// descriptor copy to shared memory and a barrier took several.
template <int N, int MODE>
__device__ __forceinline__ void force_split_item(const ChainDev* __restrict__ descs,
                                                 const int2* __restrict__ item_chain, int cur, double kick_scale) {
  const int2 ct = __ldg(item_chain + blockIdx.x);
  const ChainDev* __restrict__ d = descs + ct.x;
  const Lat L = d->lat;
  const int x = ct.y * 32 + (threadIdx.x & 31);
  if (x >= L.V) return;
  const float2* U = (const float2*)d->U[cur];
  const uint32_t* UL = (const uint32_t*)d->UL[cur];
  float* P = (float*)d->PC;
  uint32_t* PL = (uint32_t*)d->PCL;
  float2* Uo = (float2*)d->U[cur ^ 1];
  uint32_t* ULo = (uint32_t*)d->UL[cur ^ 1];
  const float ek = (float)(kick_scale * d->dt), ed = (float)d->dt;
  const int order = d->order;
  for (int mu = threadIdx.x >> 5; mu < L.D; mu += (blockDim.x >> 5))
    split::link_update<N, MODE>(L, U, UL, P, PL, P, PL, Uo, ULo, ek, ed, order, mu, x);
}

// SU(3): seven resident CTAs per SM, as the single-chain kernel's tuned budget
template <int N, int MODE>
__global__ void __launch_bounds__(128, N == 3 ? 7 : 4) kb_force_split(const ChainDev* __restrict__ descs,
                                                                       const int2* __restrict__ item_chain, int cur,
                                                                       double kick_scale) {
  force_split_item<N, MODE>(descs, item_chain, cur, kick_scale);
}

template <int N, typename T, int MODE>
__global__ void __launch_bounds__(128) kb_force_small(const ChainDev* __restrict__ descs,
                                                      const int* __restrict__ item_start,
                                                      const int* __restrict__ chain_ids, int nchains, int cur,
                                                      double kick_scale) {
  force_small_item<N, T, MODE, false>(descs, item_start, chain_ids, nchains, cur, kick_scale);
}

// FP32 SU(3): seven resident CTAs per SM, as the single-chain kernel's tuned budget
template <int MODE>
__global__ void __launch_bounds__(128, 7) kb_force_small3f(const ChainDev* __restrict__ descs,
                                                           const int* __restrict__ item_start,
                                                           const int* __restrict__ chain_ids, int nchains, int cur,
                                                           double kick_scale) {
  force_small_item<3, float, MODE, true>(descs, item_start, chain_ids, nchains, cur, kick_scale);
}

// Same for the row-per-thread path: item = G consecutive sites of one
// direction (G = blockDim / NC), directions of a site block adjacent.
template <int NMAX, typename T, int MODE>
__global__ void kb_force_rows(const ChainDev* __restrict__ descs, const int2* __restrict__ item_chain, int cur,
                              double kick_scale) {
  using S2 = typename Storage<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<T> det_s[64];
  __shared__ ChainDev sd;
  const int item = load_chain_at(sd, descs, item_chain);
  const int G = blockDim.x / sd.lat.N;
  rows::force_rows<NMAX, T, S2, MODE>(sd.lat, (const S2*)sd.U[cur], (const S2*)sd.P, (S2*)sd.P,
                                      (S2*)sd.U[cur ^ 1], (T)(kick_scale * sd.dt), (T)sd.dt, sd.order, sd.reunit,
                                      item % sd.lat.D, (item / sd.lat.D) * G, smem_raw, piv_s, det_s);
}

// FP32 with NMAX = 8, fused kick + drift: at most 128 registers (four
// 128-thread CTAs per SM), as the single-chain rows::k_force8.
static __global__ void __launch_bounds__(256, 2) kb_force_rows8f(const ChainDev* __restrict__ descs,
                                                          const int2* __restrict__ item_chain, int cur,
                                                          double kick_scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int piv_s[64];
  __shared__ cpx<float> det_s[64];
  __shared__ ChainDev sd;
  const int item = load_chain_at(sd, descs, item_chain);
  const int G = blockDim.x / sd.lat.N;
  rows::force_rows<8, float, float2, 1>(sd.lat, (const float2*)sd.U[cur], (const float2*)sd.P, (float2*)sd.P,
                                        (float2*)sd.U[cur ^ 1], (float)(kick_scale * sd.dt), (float)sd.dt, sd.order,
                                        sd.reunit, item % sd.lat.D, (item / sd.lat.D) * G, smem_raw, piv_s, det_s);
}

// Plaquette sums: item = RED_THREADS-site block; partial per chain block.
template <typename S2>
__global__ void __launch_bounds__(misc::RED_THREADS) kb_plaq(const ChainDev* __restrict__ descs,
                                                             const int* __restrict__ item_start, int nchains,
                                                             int cur) {
  __shared__ ChainDev sd;
  const int blk = load_chain(sd, descs, item_start, nullptr, nchains);
  const S2* U = (const S2*)sd.U[cur];
  const int s = blk * misc::RED_THREADS + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (sd.UL[0]) {
    const float2* Uh = (const float2*)sd.U[cur];
    const uint32_t* Ul = (const uint32_t*)sd.UL[cur];
    switch (sd.lat.N) {
      case 2: split::plaq_site<2>(sd.lat, Uh, Ul, s, v); break;
      case 3: split::plaq_site<3>(sd.lat, Uh, Ul, s, v); break;
      default: split::plaq_site<4>(sd.lat, Uh, Ul, s, v);
    }
  } else {
    switch (sd.lat.N) {
      case 2: misc::plaq_site<2, S2>(sd.lat, U, s, v); break;
      case 3: misc::plaq_site<3, S2>(sd.lat, U, s, v); break;
      case 4: misc::plaq_site<4, S2>(sd.lat, U, s, v); break;
      default: misc::plaq_site<0, S2>(sd.lat, U, s, v);
    }
  }
  misc::block_sum<2>(v);
  if (threadIdx.x == 0) {
    sd.partial[2 * blk + 0] = v[0];
    sd.partial[2 * blk + 1] = v[1];
  }
}

// Kinetic sums sum tr2(P): item = RED_THREADS-link block.
template <typename S2>
__global__ void __launch_bounds__(misc::RED_THREADS) kb_kinetic(const ChainDev* __restrict__ descs,
                                                                const int* __restrict__ item_start, int nchains) {
  __shared__ ChainDev sd;
  const int blk = load_chain(sd, descs, item_start, nullptr, nchains);
  const long t = (long)blk * misc::RED_THREADS + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (sd.PC) {
    const float* P = (const float*)sd.PC;
    const uint32_t* PL = (const uint32_t*)sd.PCL;
    switch (sd.lat.N) {
      case 2: v[0] = split::kinetic_link<2>(sd.lat, P, PL, t); break;
      case 3: v[0] = split::kinetic_link<3>(sd.lat, P, PL, t); break;
      default: v[0] = split::kinetic_link<4>(sd.lat, P, PL, t);
    }
  } else {
    switch (sd.lat.N) {
      case 2: misc::link_sums<2, S2>(sd.lat, (const S2*)sd.P, nullptr, nullptr, t, v); break;
      case 3: misc::link_sums<3, S2>(sd.lat, (const S2*)sd.P, nullptr, nullptr, t, v); break;
      case 4: misc::link_sums<4, S2>(sd.lat, (const S2*)sd.P, nullptr, nullptr, t, v); break;
      default: misc::link_sums<0, S2>(sd.lat, (const S2*)sd.P, nullptr, nullptr, t, v);
    }
  }
  misc::block_sum<3>(v);
  // kinetic partials live after the plaquette partials
  if (threadIdx.x == 0) sd.partial[2 * sd.plaq_blocks + blk] = v[0];
}

// One block per chain: sums its partials and, with `which` = 0 / 1, writes
// H = beta (S + K / (2 NC)) to st->h_old / st->h_new.
static __global__ void kb_energy(const ChainDev* __restrict__ descs, int which) {
  const ChainDev& d = descs[blockIdx.x];
  double v[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < d.plaq_blocks; b += blockDim.x) {
    v[0] += d.partial[2 * b];
    v[1] += d.partial[2 * b + 1];
  }
  for (int b = threadIdx.x; b < d.link_blocks; b += blockDim.x) v[2] += d.partial[2 * d.plaq_blocks + b];
  misc::block_sum<3>(v);
  if (threadIdx.x == 0) {
    d.sums[0] = v[0];
    d.sums[1] = v[1];
    d.sums[2] = v[2];
    const double h = d.beta * ((v[0] + v[1]) + v[2] / (2.0 * d.lat.N));
    if (which == 0)
      d.st->h_old = h;
    else if (which == 1)
      d.st->h_new = h;
  }
}

static __global__ void kb_metropolis(const ChainDev* __restrict__ descs, int nchains) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nchains) misc::metropolis(descs[c].st, descs[c].seed, nullptr, 0);
}

// Momentum refresh: item = 128-link block.
template <typename S2>
__global__ void __launch_bounds__(128) kb_refresh(const ChainDev* __restrict__ descs, const int* __restrict__ item_start,
                                                  int nchains) {
  __shared__ ChainDev sd;
  const int blk = load_chain(sd, descs, item_start, nullptr, nchains);
  const long t = (long)blk * 128 + threadIdx.x;
  const uint32_t traj = (uint32_t)sd.st->traj;
  if (sd.PC) {
    float* P = (float*)sd.PC;
    uint32_t* PL = (uint32_t*)sd.PCL;
    switch (sd.lat.N) {
      case 2: split::refresh_link<2>(sd.lat, P, PL, sd.seed, traj, sd.scale, t); break;
      case 3: split::refresh_link<3>(sd.lat, P, PL, sd.seed, traj, sd.scale, t); break;
      default: split::refresh_link<4>(sd.lat, P, PL, sd.seed, traj, sd.scale, t);
    }
  } else {
    misc::refresh_link<S2>(sd.lat, (S2*)sd.P, sd.seed, traj, sd.scale, t);
  }
}

// Residual-plane chains: projection onto SU(N) in FP64 before each
// trajectory, into the links and the saved copy (split::reunit_link); the
// other chains' items return at once.  Item = 128-link block (the refresh list).
static __global__ void __launch_bounds__(128) kb_reunit_split(const ChainDev* __restrict__ descs,
                                                              const int* __restrict__ item_start, int nchains,
                                                              int cur) {
  __shared__ ChainDev sd;
  const int blk = load_chain(sd, descs, item_start, nullptr, nchains);
  if (!sd.UL[0]) return;
  const long t = (long)blk * 128 + threadIdx.x;
  float2* U = (float2*)sd.U[cur];
  uint32_t* UL = (uint32_t*)sd.UL[cur];
  float2* C = (float2*)sd.Uconf;
  uint32_t* CL = (uint32_t*)sd.ULconf;
  switch (sd.lat.N) {
    case 2: split::reunit_link<2>(sd.lat, U, UL, C, CL, t); break;
    case 3: split::reunit_link<3>(sd.lat, U, UL, C, CL, t); break;
    default: split::reunit_link<4>(sd.lat, U, UL, C, CL, t);
  }
}

// Accept (uconf = u) or reject (u = uconf): item = 4096 x 16 bytes of the
// links, then (residual-plane chains) of their residuals.
static __global__ void __launch_bounds__(256) kb_accept_copy(const ChainDev* __restrict__ descs,
                                                             const int* __restrict__ item_start, int nchains,
                                                             int cur) {
  __shared__ ChainDev sd;
  const int blk = load_chain(sd, descs, item_start, nullptr, nchains);
  const bool acc = sd.st->accepted != 0;
  const long hi_items = (sd.n16 + 4095) / 4096;
  long i0 = (long)blk * 4096;
  uint4* U = (uint4*)sd.U[cur];
  uint4* C = (uint4*)sd.Uconf;
  long n = sd.n16;
  if (blk >= hi_items) {  // residual part
    i0 = (long)(blk - hi_items) * 4096;
    U = (uint4*)sd.UL[cur];
    C = (uint4*)sd.ULconf;
    n = sd.n16lo;
  }
  uint4* dst = acc ? C : U;
  const uint4* src = acc ? U : C;
  const long i1 = min(n, i0 + 4096);
  for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) dst[i] = src[i];
}

}  // namespace batch
}  // namespace askja
