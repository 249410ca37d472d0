// askja_plaqexp_static: plaquette sums without any device allocation.
//
// Who needs it: callers that hold the link field in device memory they manage
// themselves and cannot let a library call cudaMalloc -- code whose device
// memory is owned entirely by its own pool allocator (a framework's caching
// allocator, a fixed arena sized at start-up), or a long-running job on a
// strict memory budget, where an extra cudaMalloc either fails outright or
// synchronises the whole device in the middle of a step.  The regular entry
// points keep their partial sums in buffers allocated by askja_create; this one
// needs no context at all.
//
// How: the per-block partial sums live in a file-scope static __device__ array
// of fixed size (kMaxBlocks blocks, 2 doubles each: 128 KiB), present on every
// GPU that loads the library until the process exits.  Host code cannot use
// the array's name as a device address (on the host it names a host-side
// stand-in), so the address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and passed to the kernels.
// Neighbours are computed from the coordinates instead of the neighbour
// tables, which would also need allocating.
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>

#include "../../include/askja_gpu.h"
#include "common.cuh"
#include "launch.h"
#include "misc.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 8192;  // => at most kThreads * kMaxBlocks = 2,097,152 sites
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_plaq_scratch[2 * kMaxBlocks];

std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// periodic neighbour of site s one step along +d (sgn = 1) or -d (sgn = -1),
// from the reference's lexicographic order (structs.h:150-218)
__device__ __forceinline__ int step_site(const askja::Lat& L, int s, int d, int sgn) {
  const int c = (s / L.stride[d]) % L.n[d];
  int nc = c + sgn;
  if (nc == L.n[d]) nc = 0;
  if (nc < 0) nc = L.n[d] - 1;
  return s + (nc - c) * L.stride[d];
}

// Offset of element e of link (d, s) in the plain SoA layout this entry point
// takes: ((d*NC*NC + e)*V + s).
__device__ __forceinline__ size_t soa(const askja::Lat& L, int d, int e, int s) {
  return ((size_t)d * L.N * L.N + e) * (size_t)L.V + s;
}

// Same sums as askja::misc::k_plaq (temporal planes (0,k) / spatial planes
// (j,k), j >= 1; FP64 accumulation), neighbours by arithmetic.
template <typename S2>
__global__ void __launch_bounds__(kThreads) k_plaq_static(askja::Lat L, const S2* __restrict__ U,
                                                          double* __restrict__ partial) {
  using askja::cpx;
  const int N = L.N;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (s < L.V) {
    for (int mu = 0; mu < L.D; mu++) {
      const int xpmu = step_site(L, s, mu, 1);
      for (int nu = mu + 1; nu < L.D; nu++) {
        const int xpnu = step_site(L, s, nu, 1);
        double tr = 0.0;
        for (int i = 0; i < N; i++)
          for (int j = 0; j < N; j++) {
            cpx<double> ab = askja::czero<double>(), dc = askja::czero<double>();
            for (int k = 0; k < N; k++) {
              askja::cmac(ab, askja::ldc<double>(U + soa(L, mu, i * N + k, s)),
                          askja::ldc<double>(U + soa(L, nu, k * N + j, xpmu)));
              askja::cmac(dc, askja::ldc<double>(U + soa(L, nu, i * N + k, s)),
                          askja::ldc<double>(U + soa(L, mu, k * N + j, xpnu)));
            }
            tr = fma(ab.re, dc.re, tr);
            tr = fma(ab.im, dc.im, tr);
          }
        v[mu == 0 ? 0 : 1] += 1.0 - tr / N;
      }
    }
  }
  askja::misc::block_sum<2>(v);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 2 + 0] = v[0];
    partial[blockIdx.x * 2 + 1] = v[1];
  }
}

// Device address of the scratch array on `device` (looked up once per device).
int scratch_for(int device, double** out, char* msg, size_t cap) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_plaq_scratch);
    if (e != cudaSuccess) {
      snprintf(msg, cap, "cudaGetSymbolAddress(scratch) on device %d: %s", device, cudaGetErrorString(e));
      return ASKJA_ERR_CUDA;
    }
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[device];
  return ASKJA_OK;
}

}  // namespace

void askja_internal_set_error(const char* msg);

extern "C" int askja_plaqexp_static(const askja_params* p, const void* links, double* out, void* stream) {
  char msg[256];
  if (!p || !links || !out) {
    askja_internal_set_error("askja_plaqexp_static: null argument");
    return ASKJA_ERR_ARG;
  }
  if (p->nc < 2 || p->nc > ASKJA_MAX_NC || p->dim < 1 || p->dim > ASKJA_MAX_DIM ||
      (p->precision != ASKJA_FP64 && p->precision != ASKJA_FP32)) {
    askja_internal_set_error("askja_plaqexp_static: bad NC, DIM or precision");
    return ASKJA_ERR_ARG;
  }
  askja::Lat L{};
  long V = 1;
  for (int i = 0; i < p->dim; i++) {
    if (p->n[i] < 1) {
      askja_internal_set_error("askja_plaqexp_static: lattice extents must be >= 1");
      return ASKJA_ERR_ARG;
    }
    V *= p->n[i];
    if (V > (long)kThreads * kMaxBlocks) {
      snprintf(msg, sizeof msg,
               "askja_plaqexp_static: volume exceeds the static scratch limit of %d sites (%d blocks of %d)",
               kThreads * kMaxBlocks, kMaxBlocks, kThreads);
      askja_internal_set_error(msg);
      return ASKJA_ERR_ARG;
    }
  }
  L.V = (int)V;
  L.D = p->dim;
  L.N = p->nc;
  L.nbr = nullptr;
  for (int i = 0; i < p->dim; i++) {
    L.n[i] = p->n[i];
    long s = 1;
    for (int j = i + 1; j < p->dim; j++) s *= p->n[j];
    L.stride[i] = (int)s;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    askja_internal_set_error("askja_plaqexp_static: no CUDA device available");
    return ASKJA_ERR_NODEVICE;
  }
  if (p->device < 0 || p->device >= ndev || p->device >= kMaxDevices) {
    askja_internal_set_error("askja_plaqexp_static: device not present");
    return ASKJA_ERR_ARG;
  }
  // the caller's current device is restored on return
  askja::DevGuard guard(p->device);
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e == cudaSuccess && cur != p->device) e = cudaErrorInvalidDevice;
  double* scratch = nullptr;
  if (e == cudaSuccess) {
    if (int rc = scratch_for(p->device, &scratch, msg, sizeof msg)) {
      askja_internal_set_error(msg);
      return rc;
    }
  }
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = (int)((V + kThreads - 1) / kThreads);
  if (e == cudaSuccess) {
    if (p->precision == ASKJA_FP64)
      k_plaq_static<double2><<<nb, kThreads, 0, st>>>(L, static_cast<const double2*>(links), scratch);
    else
      k_plaq_static<float2><<<nb, kThreads, 0, st>>>(L, static_cast<const float2*>(links), scratch);
    askja::misc::k_finish<2><<<1, askja::misc::RED_THREADS, 0, st>>>(scratch, nb, out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    snprintf(msg, sizeof msg, "askja_plaqexp_static: %s", cudaGetErrorString(e));
    askja_internal_set_error(msg);
    return ASKJA_ERR_CUDA;
  }
  return ASKJA_OK;
}
