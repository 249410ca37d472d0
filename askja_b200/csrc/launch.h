// Host-side launch interface between the engine (engine.cu) and the kernels,
// one table per storage precision (kernels_fp64.cu, kernels_fp32.cu).  Every
// entry enqueues work on `stream` and returns the launch status.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace askja {

// Makes `dev` current for the duration of one API call and gives the caller
// back its own current device on return (every entry point that switches
// devices uses it, so a caller working on another GPU keeps its device).
struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DevGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DevGuard(const DevGuard&) = delete;
  DevGuard& operator=(const DevGuard&) = delete;
};

struct LaunchCtx {
  Lat lat;
  cudaStream_t stream;
  int order;        // effective Taylor order
  int reunit;       // reunitarise after each link update
  int rows_ns;      // row kernels, FP32: project by one Newton-Schulz step per update (the engine
                    // re-orthonormalises with the determinant phase every few trajectories)
  int force_rows;   // kernel mapping: 0 thread-per-link (NC <= 4), 1 row-per-thread,
                    // 2 tensor cores (FP32, NC = 16, 32 or 64, DIM >= 2), 3 site pairs in
                    // packed FP32 (NC = 3, even n[DIM-1]; the fused kick+drift then
                    // expects the site-pair layout, see pair_swap)
  int rows_groups;  // row kernels: sites per CTA (0: default 128/NC)
  int small_occ;    // thread-per-link kernels: register budget for 0 default, 1 / 2 more resident CTAs
  void* scratch;    // tensor-core path: per-link contiguous copy of U (V*D*NC*NC float2)
  unsigned* status; // tensor-core path: nonzero after a bounded wait gave up
  // row-kernel reunitarisation: run only when *gate % gate_every == 0 (null: always)
  const unsigned long long* gate;
  int gate_every;
};

// Trajectories between two full reunitarisation passes (Gram-Schmidt with the
// determinant phase) over U, where the per-update projection leaves drift: the
// tensor-core path and the FP32 row kernels (Newton-Schulz per update).
constexpr int FULL_REUNIT_EVERY = 10;

// whether the tensor-core mapping exists for this shape and precision
inline bool tc_supported(int N, int D, bool fp64) { return !fp64 && (N == 16 || N == 32 || N == 64) && D >= 2; }

// whether the site-pair mapping exists (n_fast: extent of the fastest direction)
inline bool pair_supported(int N, int D, bool fp64, int n_fast) {
  return !fp64 && N == 3 && D >= 2 && n_fast % 2 == 0;
}

// Scalar reductions return their values in device memory:
//   plaq     -> out[0] temporal, out[1] spatial
//   linksums -> out[0] sum tr2(Pa), out[1] sum 1/4 tr2(Pa+Pb), out[2] UViol
//   gauss    -> out[0]
struct KernelSet {
  // mode 0: Pout = Pin - ek F(U); mode 1: also Uout = exp(i ed Pout) U
  cudaError_t (*force)(const LaunchCtx&, int mode, const void* U, const void* Pin, void* Pout, void* Uout, double ek,
                       double ed);
  cudaError_t (*drift)(const LaunchCtx&, void* U, const void* P, double eps);
  cudaError_t (*reunit)(const LaunchCtx&, void* U);
  cudaError_t (*plaq)(const LaunchCtx&, const void* U, double* partial, double* out);
  cudaError_t (*linksums)(const LaunchCtx&, const void* Pa, const void* Pb, const void* U, double* partial,
                          double* out);
  cudaError_t (*gauss)(const LaunchCtx&, const void* U, const void* Pi, double* partial, double* out);
  cudaError_t (*lines)(const LaunchCtx&, const void* U, int dir, int nlines, int start_stride, double* out);
  cudaError_t (*slice_trace)(const LaunchCtx&, const void* U, double* out);
  // eigenvalues of closed line matrices: ev[q*NC + i] (complex), *fail set on no convergence
  cudaError_t (*line_eigs)(const LaunchCtx&, const void* U, int dir, int nlines, int start_stride, double2* ev,
                           int* fail);
  cudaError_t (*refresh)(const LaunchCtx&, void* P, uint64_t seed, const unsigned long long* traj_dev,
                         unsigned long long traj_host, double scale);
  cudaError_t (*identity)(const LaunchCtx&, void* U);
  cudaError_t (*gauss_matrices)(const LaunchCtx&, void* U, uint64_t seed);
  cudaError_t (*from_conf)(const LaunchCtx&, const void* conf, void* f);
  cudaError_t (*to_conf)(const LaunchCtx&, const void* f, void* conf);
  // canonical <-> site-pair layout of a field, in place (FP32 only)
  cudaError_t (*pair_swap)(const LaunchCtx&, void* f);
  // FourierTrafo: coef[0..n-1] (partial: 2n doubles of scratch)
  cudaError_t (*fourier)(const LaunchCtx&, const void* U, int n, double* partial, double* coef);
  // Tab for nsites sites from site0 with momenta Pa + Pb: out[k*npt + m]
  cudaError_t (*tab)(const LaunchCtx&, const void* U, const void* Pa, const void* Pb, int site0, int nsites, int npt,
                     double* out);
  // tensor-core path: the give-up path of a bounded wait, on one CTA (tc::k_wait_probe)
  cudaError_t (*wait_probe)(const LaunchCtx&, long long cycles);
};

// size (in doubles) of the partial buffer the reductions need
size_t partial_doubles(const Lat& L);

// sites per CTA the row-per-thread kernels actually use for a requested value
// (0: default), after the thread-count and shared-memory limits
int rows_effective_groups(int N, bool fp64, int want);

extern const KernelSet kernels_fp64;
extern const KernelSet kernels_fp32;

}  // namespace askja
