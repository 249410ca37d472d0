// Batched independent chains: askja_batch_* of include/askja_gpu.h.
//
// Many HMC chains of uneven shape (NC, DIM, extents, BETA, DT, LEVEL, seed)
// advance together: per MD step one force launch per colour number covers
// every chain of that colour number (work list of 32-site tiles or link
// groups), the launches of different colour numbers run on forked streams,
// and reductions, refresh, Metropolis and the accept/reject copy are one
// launch each for all chains.  A whole trajectory of all chains is captured
// once as a CUDA graph and replayed.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "../../include/askja_gpu.h"
#include "batch.cuh"
#include "kernels.cuh"
#include "launch.h"
#include "split.h"

using askja::Lat;
using askja::batch::ChainDev;
using askja::misc::TrajState;

struct askja_batch {
  int nchains = 0;
  int precision = ASKJA_FP32;
  int device = 0;
  std::vector<askja_chain_params> params;
  std::vector<ChainDev> desc;
  ChainDev* d_desc = nullptr;
  std::vector<void*> allocs;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev;
  struct Group {
    int N = 0;      // colour number (small path) or 0 for the row path
    int nmax = 0;   // row path register bucket
    int G = 1;      // row path groups per CTA
    size_t smem = 0;
    std::vector<int> chains;
    int* d_start = nullptr;
    int* d_ids = nullptr;
    int* d_item = nullptr;  // per item: chain index (into the descriptors) and item within the chain, interleaved
    int nitems = 0;
  };
  std::vector<Group> groups;
  int* d_plaq_start = nullptr;
  int* d_link_start = nullptr;
  int* d_refresh_start = nullptr;
  int* d_copy_start = nullptr;
  int n_plaq = 0, n_link = 0, n_refresh = 0, n_copy = 0;
  bool any_split = false;  // some chain runs the residual-plane mode
  void* staging = nullptr;
  int cur = 0;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int g_nsteps[2] = {-1, -1};
  std::string err;
};

namespace {

thread_local std::string g_batch_error;

int berr(askja_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  (b ? b->err : g_batch_error) = buf;
  return code;
}

#define BCK(call)                                                                                        \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return berr(b, ASKJA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));     \
  } while (0)

template <typename X>
int dalloc(askja_batch* b, X** p, size_t bytes) {
  void* q = nullptr;
  BCK(cudaMalloc(&q, std::max<size_t>(bytes, 16)));
  b->allocs.push_back(q);
  *p = static_cast<X*>(q);
  return ASKJA_OK;
}

int upload_ints(askja_batch* b, int** dst, const std::vector<int>& v) {
  if (int rc = dalloc(b, dst, v.size() * sizeof(int))) return rc;
  BCK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice));
  return ASKJA_OK;
}

askja::LaunchCtx chain_lc(const askja_batch* b, int c) {
  askja::LaunchCtx lc{};
  lc.lat = b->desc[c].lat;
  lc.stream = b->stream;
  lc.order = b->desc[c].order;
  lc.reunit = b->desc[c].reunit;
  lc.force_rows = 0;
  return lc;
}

const askja::KernelSet& kset(const askja_batch* b) {
  return b->precision == ASKJA_FP64 ? askja::kernels_fp64 : askja::kernels_fp32;
}

// ---- launches -------------------------------------------------------------

template <typename T>
cudaError_t launch_force(askja_batch* b, const askja_batch::Group& g, cudaStream_t st, int mode, double ks) {
  using namespace askja::batch;
  const dim3 grid(g.nitems);
  if (g.N == 2 || g.N == 3 || g.N == 4) {
    int maxd = 1;
    for (int c : g.chains) maxd = std::max(maxd, b->desc[c].lat.D);
    const dim3 blk(32 * std::min(maxd, 4));
    if constexpr (sizeof(T) == 4) {
      // residual-plane mode (every FP32 chain with NC <= 4)
#define SPLIT(NN)                                                                                                \
  if (g.N == NN) {                                                                                               \
    if (mode)                                                                                                    \
      kb_force_split<NN, 1><<<grid, blk, 0, st>>>(b->d_desc, (const int2*)g.d_item, b->cur, ks);                 \
    else                                                                                                         \
      kb_force_split<NN, 0><<<grid, blk, 0, st>>>(b->d_desc, (const int2*)g.d_item, b->cur, ks);                 \
    return cudaGetLastError();                                                                                   \
  }
      SPLIT(2) SPLIT(3) SPLIT(4)
#undef SPLIT
    }
    if constexpr (sizeof(T) == 4) {
      if (g.N == 3) {
        if (mode)
          kb_force_small3f<1><<<grid, blk, 0, st>>>(b->d_desc, g.d_start, g.d_ids, (int)g.chains.size(), b->cur, ks);
        else
          kb_force_small3f<0><<<grid, blk, 0, st>>>(b->d_desc, g.d_start, g.d_ids, (int)g.chains.size(), b->cur, ks);
        return cudaGetLastError();
      }
    }
#define SMALL(NN)                                                                                            \
  if (g.N == NN) {                                                                                           \
    if (mode)                                                                                                \
      kb_force_small<NN, T, 1><<<grid, blk, 0, st>>>(b->d_desc, g.d_start, g.d_ids, (int)g.chains.size(),   \
                                                      b->cur, ks);                                           \
    else                                                                                                     \
      kb_force_small<NN, T, 0><<<grid, blk, 0, st>>>(b->d_desc, g.d_start, g.d_ids, (int)g.chains.size(),   \
                                                      b->cur, ks);                                           \
  }
    SMALL(2) SMALL(3) SMALL(4)
#undef SMALL
    return cudaGetLastError();
  }
  const dim3 blk(g.G * b->params[g.chains[0]].nc);
#define ROWS(NM)                                                                                              \
  if (g.nmax == NM) {                                                                                         \
    auto k = mode ? kb_force_rows<NM, T, 1> : kb_force_rows<NM, T, 0>;                                        \
    if constexpr (sizeof(T) == 4 && NM == 8)                                                                  \
      if (mode) k = kb_force_rows8f;                                                                          \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem);                        \
    k<<<grid, blk, g.smem, st>>>(b->d_desc, (const int2*)g.d_item, b->cur, ks);                              \
  }
  ROWS(8) ROWS(16) ROWS(32) ROWS(64)
#undef ROWS
  return cudaGetLastError();
}

// all groups' force launches for one MD step, forked onto side streams
template <typename T>
int md_step(askja_batch* b, int mode, double ks) {
  const int ng = (int)b->groups.size();
  if (ng == 1) {
    if (cudaError_t e = launch_force<T>(b, b->groups[0], b->stream, mode, ks))
      return berr(b, ASKJA_ERR_CUDA, "force: %s", cudaGetErrorString(e));
    return ASKJA_OK;
  }
  BCK(cudaEventRecord(b->ev[0], b->stream));
  for (int i = 0; i < ng; i++) {
    BCK(cudaStreamWaitEvent(b->side[i], b->ev[0], 0));
    if (cudaError_t e = launch_force<T>(b, b->groups[i], b->side[i], mode, ks))
      return berr(b, ASKJA_ERR_CUDA, "force: %s", cudaGetErrorString(e));
    BCK(cudaEventRecord(b->ev[1 + i], b->side[i]));
    BCK(cudaStreamWaitEvent(b->stream, b->ev[1 + i], 0));
  }
  return ASKJA_OK;
}

template <typename T>
int energies(askja_batch* b, int which) {
  using S2 = typename askja::Storage<T>::type;
  using namespace askja::batch;
  kb_plaq<S2><<<b->n_plaq, askja::misc::RED_THREADS, 0, b->stream>>>(b->d_desc, b->d_plaq_start, b->nchains, b->cur);
  kb_kinetic<S2><<<b->n_link, askja::misc::RED_THREADS, 0, b->stream>>>(b->d_desc, b->d_link_start, b->nchains);
  kb_energy<<<b->nchains, askja::misc::RED_THREADS, 0, b->stream>>>(b->d_desc, which);
  BCK(cudaGetLastError());
  return ASKJA_OK;
}

template <typename T>
int enqueue_trajectory(askja_batch* b, int nsteps) {
  using S2 = typename askja::Storage<T>::type;
  using namespace askja::batch;
  for (int c = 0; c < b->nchains; c++) {  // gated full reunitarisation (d.reunit == 2)
    const auto& d = b->desc[c];
    if (d.reunit != 2) continue;
    askja::LaunchCtx lc = chain_lc(b, c);
    lc.gate = &d.st->traj;
    lc.gate_every = askja::FULL_REUNIT_EVERY;
    if (cudaError_t e = kset(b).reunit(lc, d.U[b->cur])) return berr(b, ASKJA_ERR_CUDA, "reunit: %s", cudaGetErrorString(e));
    BCK(cudaMemcpyAsync(d.Uconf, d.U[b->cur], askja::field_elems(d.lat) * sizeof(askja::cpx<T>), cudaMemcpyDeviceToDevice,
                        b->stream));
  }
  if (b->any_split)
    kb_reunit_split<<<b->n_refresh, 128, 0, b->stream>>>(b->d_desc, b->d_refresh_start, b->nchains, b->cur);
  kb_refresh<S2><<<b->n_refresh, 128, 0, b->stream>>>(b->d_desc, b->d_refresh_start, b->nchains);
  BCK(cudaGetLastError());
  if (int rc = energies<T>(b, 0)) return rc;
  for (int i = 0; i < nsteps; i++) {
    if (int rc = md_step<T>(b, 1, i == 0 ? 0.5 : 1.0)) return rc;
    b->cur ^= 1;
  }
  if (int rc = md_step<T>(b, 0, 0.5)) return rc;
  if (int rc = energies<T>(b, 1)) return rc;
  kb_metropolis<<<(b->nchains + 127) / 128, 128, 0, b->stream>>>(b->d_desc, b->nchains);
  kb_accept_copy<<<b->n_copy, 256, 0, b->stream>>>(b->d_desc, b->d_copy_start, b->nchains, b->cur);
  BCK(cudaGetLastError());
  return ASKJA_OK;
}

int enqueue(askja_batch* b, int nsteps) {
  return b->precision == ASKJA_FP64 ? enqueue_trajectory<double>(b, nsteps) : enqueue_trajectory<float>(b, nsteps);
}

void drop_graphs(askja_batch* b) {
  for (int i = 0; i < 2; i++) {
    if (b->gexec[i]) cudaGraphExecDestroy(b->gexec[i]);
    b->gexec[i] = nullptr;
    b->g_nsteps[i] = -1;
  }
}

int check_chain(askja_batch* b, int c) {
  if (!b) return berr(nullptr, ASKJA_ERR_ARG, "null batch");
  if (c < 0 || c >= b->nchains) return berr(b, ASKJA_ERR_ARG, "chain %d out of range", c);
  return ASKJA_OK;
}

}  // namespace

extern "C" {

const char* askja_batch_last_error(const askja_batch* b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

void* askja_batch_stream(askja_batch* b) { return b ? (void*)b->stream : nullptr; }

void askja_batch_destroy(askja_batch* b) {
  if (!b) return;
  askja::DevGuard g(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  for (void* p : b->allocs) cudaFree(p);
  for (cudaStream_t s : b->side) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int askja_batch_create(const askja_chain_params* chains, int nchains, int precision, int device, askja_batch** out) {
  askja_batch* b = nullptr;
  if (!chains || !out || nchains < 1) return berr(nullptr, ASKJA_ERR_ARG, "need at least one chain");
  *out = nullptr;
  if (precision != ASKJA_FP32 && precision != ASKJA_FP64) return berr(nullptr, ASKJA_ERR_ARG, "bad precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return berr(nullptr, ASKJA_ERR_NODEVICE, "no CUDA device available (no CPU fallback)");
  if (device < 0 || device >= ndev) return berr(nullptr, ASKJA_ERR_ARG, "device %d not present", device);
  for (int c = 0; c < nchains; c++) {
    const askja_chain_params& p = chains[c];
    if (p.nc < 2 || p.nc > ASKJA_MAX_NC || p.dim < 1 || p.dim > ASKJA_MAX_DIM || !(p.beta > 0))
      return berr(nullptr, ASKJA_ERR_ARG, "chain %d: bad NC, DIM or BETA", c);
    long V = 1;
    for (int i = 0; i < p.dim; i++) {
      if (p.n[i] < 1) return berr(nullptr, ASKJA_ERR_ARG, "chain %d: extent < 1", c);
      V *= p.n[i];
    }
    if (V > (1L << 30)) return berr(nullptr, ASKJA_ERR_ARG, "chain %d: volume too large", c);
  }
  askja::DevGuard g(device);
  b = new askja_batch();
  b->nchains = nchains;
  b->precision = precision;
  b->device = device;
  b->params.assign(chains, chains + nchains);
  auto fail = [&](int rc) {
    g_batch_error = b->err;
    askja_batch_destroy(b);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(berr(b, ASKJA_ERR_CUDA, "stream"));
  const size_t elem = precision == ASKJA_FP64 ? 16 : 8;
  b->desc.resize(nchains);
  size_t max_conf = 0;
  std::vector<int> plaq_start(1, 0), link_start(1, 0), refresh_start(1, 0), copy_start(1, 0);
  for (int c = 0; c < nchains; c++) {
    const askja_chain_params& p = chains[c];
    ChainDev& d = b->desc[c];
    memset(&d, 0, sizeof d);
    Lat& L = d.lat;
    long V = 1;
    for (int i = 0; i < p.dim; i++) V *= p.n[i];
    L.V = (int)V;
    L.B = (int)((V + 31) / 32);
    L.D = p.dim;
    L.N = p.nc;
    for (int i = 0; i < p.dim; i++) {
      L.n[i] = p.n[i];
      long s = 1;
      for (int j = i + 1; j < p.dim; j++) s *= p.n[j];
      L.stride[i] = (int)s;
    }
    std::vector<int> nbr((size_t)2 * p.dim * V);
    {
      long stride[ASKJA_MAX_DIM];
      for (int i = 0; i < p.dim; i++) stride[i] = L.stride[i];
      for (int dd = 0; dd < p.dim; dd++)
        for (long s = 0; s < V; s++) {
          const long co = (dd == 0) ? s / stride[0] : (s % stride[dd - 1]) / stride[dd];
          const long up = (co + 1) % p.n[dd];
          long dn = (co - 1) % p.n[dd];
          if (dn < 0) dn += p.n[dd];
          nbr[(size_t)(2 * dd) * V + s] = (int)(s + (up - co) * stride[dd]);
          nbr[(size_t)(2 * dd + 1) * V + s] = (int)(s + (dn - co) * stride[dd]);
        }
    }
    int* dn = nullptr;
    if (int rc = upload_ints(b, &dn, nbr)) return fail(rc);
    L.nbr = dn;
    const size_t fbytes = askja::field_elems(L) * elem;
    for (void** f : {&d.U[0], &d.U[1], &d.P, &d.Uconf})
      if (int rc = dalloc(b, f, fbytes)) return fail(rc);
    d.dt = p.dt;
    d.beta = p.beta;
    d.scale = std::sqrt(2.0 * p.nc / p.beta);
    d.order = askja::taylor_order(p.level);
    // FP32: reunitarise after each update; on the row kernels (NC > 4) by a
    // Newton-Schulz step, with a full pass every FULL_REUNIT_EVERY
    // trajectories, as a single chain does
    d.reunit = precision == ASKJA_FP32 ? (p.nc > 4 ? 2 : 1) : 0;
    if (precision == ASKJA_FP32 && askja::splitk::supported(p.nc)) d.reunit = 0;  // residual planes: per trajectory
    d.seed = p.seed;
    if (int rc = dalloc(b, &d.st, sizeof(TrajState))) return fail(rc);
    if (cudaMemset(d.st, 0, sizeof(TrajState)) != cudaSuccess) return fail(berr(b, ASKJA_ERR_CUDA, "memset"));
    if (int rc = dalloc(b, &d.sums, 8 * sizeof(double))) return fail(rc);
    d.plaq_blocks = (int)((V + askja::misc::RED_THREADS - 1) / askja::misc::RED_THREADS);
    d.link_blocks = (int)((V * p.dim + askja::misc::RED_THREADS - 1) / askja::misc::RED_THREADS);
    if (int rc = dalloc(b, &d.partial, (2 * (size_t)d.plaq_blocks + d.link_blocks) * sizeof(double))) return fail(rc);
    d.n16 = (long)(fbytes / 16);
    if (precision == ASKJA_FP32 && askja::splitk::supported(p.nc)) {
      // residual-plane mode, as a single FP32 chain of this colour number:
      // projected onto SU(N) in FP64 before every trajectory, not per update
      const size_t lo_bytes = askja::field_elems(L) * sizeof(uint32_t);
      for (void** f : {&d.UL[0], &d.UL[1], &d.ULconf})
        if (int rc = dalloc(b, f, lo_bytes)) return fail(rc);
      if (int rc = dalloc(b, &d.PC, askja::splitk::coef_floats(L) * sizeof(float))) return fail(rc);
      if (int rc = dalloc(b, &d.PCL, askja::splitk::coef_words(L) * sizeof(uint32_t))) return fail(rc);
      for (void* f : {d.UL[0], d.UL[1], d.ULconf})
        if (cudaMemset(f, 0, lo_bytes) != cudaSuccess) return fail(berr(b, ASKJA_ERR_CUDA, "memset"));
      d.n16lo = (long)(lo_bytes / 16);
      b->any_split = true;
    }
    plaq_start.push_back(plaq_start.back() + d.plaq_blocks);
    link_start.push_back(link_start.back() + d.link_blocks);
    refresh_start.push_back(refresh_start.back() + (int)((V * p.dim + 127) / 128));
    copy_start.push_back(copy_start.back() + (int)((d.n16 + 4095) / 4096) + (int)((d.n16lo + 4095) / 4096));
    max_conf = std::max(max_conf, (size_t)V * p.dim * p.nc * p.nc * 16);
    // cold start
    askja::LaunchCtx lc = chain_lc(b, c);
    if (kset(b).identity(lc, d.U[0]) != cudaSuccess) return fail(berr(b, ASKJA_ERR_CUDA, "identity"));
    if (cudaMemcpyAsync(d.Uconf, d.U[0], fbytes, cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess)
      return fail(berr(b, ASKJA_ERR_CUDA, "copy"));
  }
  if (int rc = upload_ints(b, &b->d_plaq_start, plaq_start)) return fail(rc);
  if (int rc = upload_ints(b, &b->d_link_start, link_start)) return fail(rc);
  if (int rc = upload_ints(b, &b->d_refresh_start, refresh_start)) return fail(rc);
  if (int rc = upload_ints(b, &b->d_copy_start, copy_start)) return fail(rc);
  b->n_plaq = plaq_start.back();
  b->n_link = link_start.back();
  b->n_refresh = refresh_start.back();
  b->n_copy = copy_start.back();
  if (int rc = dalloc(b, &b->staging, max_conf)) return fail(rc);
  // force groups: one per small colour number, one per row-path bucket and colour number
  std::map<int, std::vector<int>> by_nc;
  for (int c = 0; c < nchains; c++) by_nc[chains[c].nc].push_back(c);
  for (auto& kv : by_nc) {
    askja_batch::Group g;
    g.chains = kv.second;
    const int N = kv.first;
    std::vector<int> start(1, 0);
    std::vector<int> item;
    if (N <= 4) {
      g.N = N;
      for (int c : g.chains) {
        start.push_back(start.back() + b->desc[c].lat.B);
        for (int t = 0; t < b->desc[c].lat.B; t++) {
          item.push_back(c);
          item.push_back(t);
        }
      }
    } else {
      g.N = 0;
      g.nmax = N <= 8 ? 8 : N <= 16 ? 16 : N <= 32 ? 32 : 64;
      if (precision == ASKJA_FP64)
        askja::detail::Rows<double>::shape(N, &g.G, &g.smem);
      else
        askja::detail::Rows<float>::shape(N, &g.G, &g.smem);
      for (int c : g.chains) {
        const Lat& L = b->desc[c].lat;
        const int n = (int)((L.V + g.G - 1) / g.G) * L.D;
        start.push_back(start.back() + n);
        for (int t = 0; t < n; t++) {
          item.push_back(c);
          item.push_back(t);
        }
      }
    }
    g.nitems = start.back();
    if (int rc = upload_ints(b, &g.d_start, start)) return fail(rc);
    if (int rc = upload_ints(b, &g.d_ids, g.chains)) return fail(rc);
    if (!item.empty())
      if (int rc = upload_ints(b, &g.d_item, item)) return fail(rc);
    b->groups.push_back(g);
  }
  b->side.resize(b->groups.size());
  for (auto& s : b->side)
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
      return fail(berr(b, ASKJA_ERR_CUDA, "side stream"));
  b->ev.resize(b->groups.size() + 1);
  for (auto& e : b->ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      return fail(berr(b, ASKJA_ERR_CUDA, "event"));
  if (int rc = dalloc(b, &b->d_desc, sizeof(ChainDev) * nchains)) return fail(rc);
  if (cudaMemcpy(b->d_desc, b->desc.data(), sizeof(ChainDev) * nchains, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(berr(b, ASKJA_ERR_CUDA, "descriptor upload"));
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail(berr(b, ASKJA_ERR_CUDA, "init"));
  *out = b;
  return ASKJA_OK;
}

int askja_batch_hot_start(askja_batch* b, uint64_t seed) {
  if (int rc = check_chain(b, 0)) return rc;
  askja::DevGuard g(b->device);
  for (int c = 0; c < b->nchains; c++) {
    askja::LaunchCtx lc = chain_lc(b, c);
    ChainDev& d = b->desc[c];
    if (kset(b).gauss_matrices(lc, d.U[b->cur], seed + 1000003ull * c) != cudaSuccess)
      return berr(b, ASKJA_ERR_CUDA, "hot start launch");
    if (d.UL[0]) {
      BCK(cudaMemsetAsync(d.UL[b->cur], 0, d.n16lo * 16, b->stream));
      if (askja::splitk::reunit(lc, d.U[b->cur], d.UL[b->cur], d.Uconf, d.ULconf) != cudaSuccess)
        return berr(b, ASKJA_ERR_CUDA, "hot start launch");
      continue;
    }
    if (kset(b).reunit(lc, d.U[b->cur]) != cudaSuccess) return berr(b, ASKJA_ERR_CUDA, "hot start launch");
    BCK(cudaMemcpyAsync(d.Uconf, d.U[b->cur], d.n16 * 16, cudaMemcpyDeviceToDevice, b->stream));
  }
  BCK(cudaStreamSynchronize(b->stream));
  return ASKJA_OK;
}

int askja_batch_set_links(askja_batch* b, int c, const double* conf) {
  if (int rc = check_chain(b, c)) return rc;
  if (!conf) return berr(b, ASKJA_ERR_ARG, "null buffer");
  askja::DevGuard g(b->device);
  ChainDev& d = b->desc[c];
  const size_t bytes = (size_t)d.lat.V * d.lat.D * d.lat.N * d.lat.N * 16;
  for (size_t i = 0; i < bytes / 8; i++)
    if (!std::isfinite(conf[i])) return berr(b, ASKJA_ERR_NONFINITE, "non-finite value in chain %d links", c);
  BCK(cudaMemcpyAsync(b->staging, conf, bytes, cudaMemcpyHostToDevice, b->stream));
  askja::LaunchCtx lc = chain_lc(b, c);
  const cudaError_t ec = d.UL[0] ? askja::splitk::links_from_conf(lc, b->staging, d.U[b->cur], d.UL[b->cur])
                                 : kset(b).from_conf(lc, b->staging, d.U[b->cur]);
  if (ec != cudaSuccess) return berr(b, ASKJA_ERR_CUDA, "from_conf");
  BCK(cudaMemcpyAsync(d.Uconf, d.U[b->cur], d.n16 * 16, cudaMemcpyDeviceToDevice, b->stream));
  if (d.UL[0]) BCK(cudaMemcpyAsync(d.ULconf, d.UL[b->cur], d.n16lo * 16, cudaMemcpyDeviceToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return ASKJA_OK;
}

int askja_batch_get_links(askja_batch* b, int c, double* conf) {
  if (int rc = check_chain(b, c)) return rc;
  if (!conf) return berr(b, ASKJA_ERR_ARG, "null buffer");
  askja::DevGuard g(b->device);
  ChainDev& d = b->desc[c];
  const size_t bytes = (size_t)d.lat.V * d.lat.D * d.lat.N * d.lat.N * 16;
  askja::LaunchCtx lc = chain_lc(b, c);
  const cudaError_t ec = d.UL[0] ? askja::splitk::links_to_conf(lc, d.U[b->cur], d.UL[b->cur], b->staging)
                                 : kset(b).to_conf(lc, d.U[b->cur], b->staging);
  if (ec != cudaSuccess) return berr(b, ASKJA_ERR_CUDA, "to_conf");
  BCK(cudaMemcpyAsync(conf, b->staging, bytes, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return ASKJA_OK;
}

int askja_batch_run(askja_batch* b, int ntraj, int nsteps, int use_graph, askja_traj_result* results) {
  if (int rc = check_chain(b, 0)) return rc;
  if (ntraj < 0 || nsteps < 1) return berr(b, ASKJA_ERR_ARG, "bad trajectory counts");
  askja::DevGuard g(b->device);
  for (int t = 0; t < ntraj; t++) {
    if (!use_graph) {
      if (int rc = enqueue(b, nsteps)) return rc;
      continue;
    }
    const int start = b->cur;
    if (!b->gexec[start] || b->g_nsteps[start] != nsteps) {
      if (b->gexec[start]) cudaGraphExecDestroy(b->gexec[start]);
      b->gexec[start] = nullptr;
      cudaGraph_t graph;
      BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue(b, nsteps);
      cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
      b->cur = start;
      if (rc) return rc;
      if (ce != cudaSuccess) return berr(b, ASKJA_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&b->gexec[start], graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return berr(b, ASKJA_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      b->g_nsteps[start] = nsteps;
    }
    BCK(cudaGraphLaunch(b->gexec[start], b->stream));
    b->cur = start ^ (nsteps & 1);
  }
  BCK(cudaStreamSynchronize(b->stream));
  if (results)
    for (int c = 0; c < b->nchains; c++)
      BCK(cudaMemcpy(&results[c], b->desc[c].st, sizeof(TrajState), cudaMemcpyDeviceToHost));
  return ASKJA_OK;
}

int askja_batch_plaquette(askja_batch* b, double* out) {
  if (int rc = check_chain(b, 0)) return rc;
  if (!out) return berr(b, ASKJA_ERR_ARG, "null output");
  askja::DevGuard g(b->device);
  int rc = b->precision == ASKJA_FP64 ? energies<double>(b, 2) : energies<float>(b, 2);
  if (rc) return rc;
  BCK(cudaStreamSynchronize(b->stream));
  for (int c = 0; c < b->nchains; c++) {
    double s[2];
    BCK(cudaMemcpy(s, b->desc[c].sums, sizeof s, cudaMemcpyDeviceToHost));
    const Lat& L = b->desc[c].lat;
    const double np = (double)L.V * L.D * (L.D - 1) / 2;
    out[c] = np > 0 ? 1.0 - (s[0] + s[1]) / np : 1.0;
  }
  return ASKJA_OK;
}

}  // extern "C"
