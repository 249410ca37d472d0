// askja B200 engine: context, device fields, and the C ABI of include/askja_gpu.h.
//
// Device state per context (all in HBM, SoA layout of common.cuh):
//   U[0], U[1]  link field and its ping-pong partner (fused kick+drift writes
//               the updated links to the other buffer, because neighbouring
//               links are still being read)   -> the reference's u (and U)
//   P           current momenta                -> pi
//   P2          updated momenta                -> Pi
//   Uconf       last accepted configuration    -> uconf
//   nbr         periodic neighbour tables, 2*D planes of V int32
//   partial/sums/st/log  reduction scratch and trajectory bookkeeping
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/askja_gpu.h"
#include "launch.h"
#include "misc.cuh"
#include "split.h"

using askja::DevGuard;

// NVTX range over one host call or enqueue phase (visible to Nsight tools;
// free when no tool is attached)
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};
using askja::KernelSet;
using askja::Lat;
using askja::LaunchCtx;
using askja::misc::TrajState;

static_assert(sizeof(askja_traj_result) == sizeof(TrajState), "traj result layout");

static thread_local std::string g_last_error;

// autotuning results of this process, per (NC, DIM, precision)
static std::mutex g_tune_mutex;
static std::map<std::tuple<int, int, int>, askja_tuning> g_tune_cache;

struct askja_ctx {
  askja_params p{};
  Lat lat{};
  const KernelSet* ks = nullptr;
  LaunchCtx lc{};
  long V = 0, nl = 0;
  int N = 0, D = 0;
  size_t field_bytes = 0;
  void* U[2] = {nullptr, nullptr};
  int cur = 0;
  void* P = nullptr;
  void* P2 = nullptr;
  void* Uconf = nullptr;
  int* nbr = nullptr;
  double* partial = nullptr;
  double* sums = nullptr;   // [0..1] plaq t/s, [2..4] link sums, [5] gauss, [6..] line results
  double* lines = nullptr;  // per-line results
  double2* eigs = nullptr;  // eigenvalues of the N0 + N1 lines of askja_eigenphases
  int* eigfail = nullptr;
  TrajState* st = nullptr;
  double* logbuf = nullptr;
  int logcap = 0;
  void* staging = nullptr;  // U-conf layout staging buffer (V*D*NC*NC double2)
  unsigned long long* nonfinite = nullptr;
  unsigned* tc_status = nullptr;  // tensor-core kernels: set when a bounded wait gave up
  cudaStream_t stream = nullptr;
  // askja_set_links_async: copy stream and two device staging buffers, used in
  // turn; up_copied[b] marks the copy into up[b] done, up_free[b] the
  // conversion out of it; up_bad counts non-finite input values until the
  // next synchronisation
  cudaStream_t copy_stream = nullptr;
  void* up[2] = {nullptr, nullptr};
  cudaEvent_t up_copied[2] = {nullptr, nullptr};
  cudaEvent_t up_free[2] = {nullptr, nullptr};
  int up_next = 0;
  unsigned long long* up_bad = nullptr;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int g_nsteps[2] = {-1, -1};
  // residual-plane FP32 mode (ASKJA_FP32, NC <= 4, thread per link; split.h):
  // bfloat16 residuals of the links (UL, ULconf; lo_bytes each) and the
  // momenta pi / Pi as FP32 coordinates (PC, P2C; coef_bytes) plus residuals
  // (PCL, P2CL; coefl_bytes).  P and P2 then hold full FP32 matrices made from
  // the coordinates on demand, for the matrix diagnostics (Gauss law, Tab).
  bool split = false;
  void* UL[2] = {nullptr, nullptr};
  void* ULconf = nullptr;
  void* PC = nullptr;
  void* PCL = nullptr;
  void* P2C = nullptr;
  void* P2CL = nullptr;
  size_t lo_bytes = 0, coef_bytes = 0, coefl_bytes = 0;
  std::string err;
};

namespace {

int set_err(askja_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c)
    c->err = buf;
  else
    g_last_error = buf;
  return code;
}

#define CK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return set_err(c, ASKJA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)


// neighbour tables from the reference's coordinate scheme (structs.h:169-218)
void build_neighbours(const askja_params& p, long V, std::vector<int>& nbr) {
  long stride[ASKJA_MAX_DIM];
  for (int i = 0; i < p.dim; i++) {
    stride[i] = 1;
    for (int j = i + 1; j < p.dim; j++) stride[i] *= p.n[j];
  }
  nbr.assign((size_t)2 * p.dim * V, 0);
  for (int d = 0; d < p.dim; d++)
    for (long s = 0; s < V; s++) {
      const long c = (d == 0) ? s / stride[0] : (s % stride[d - 1]) / stride[d];
      const long up = (c + 1) % p.n[d];
      long dn = (c - 1) % p.n[d];
      if (dn < 0) dn += p.n[d];
      nbr[(size_t)(2 * d) * V + s] = (int)(s + (up - c) * stride[d]);
      nbr[(size_t)(2 * d + 1) * V + s] = (int)(s + (dn - c) * stride[d]);
    }
}

int scal(askja_ctx* c, const double* dev, double* host, int n) {
  CK(cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int check_ctx(askja_ctx* c) {
  if (!c) return set_err(nullptr, ASKJA_ERR_ARG, "null context");
  return ASKJA_OK;
}

void* cur_u(askja_ctx* c) { return c->U[c->cur]; }
void* cur_ul(askja_ctx* c) { return c->UL[c->cur]; }

// Uconf <- U (save) or U <- Uconf (restore), residual planes included
cudaError_t copy_saved(askja_ctx* c, bool save) {
  void* d = save ? c->Uconf : cur_u(c);
  const void* src = save ? cur_u(c) : c->Uconf;
  cudaError_t e = cudaMemcpyAsync(d, src, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess && c->split)
    e = cudaMemcpyAsync(save ? c->ULconf : cur_ul(c), save ? cur_ul(c) : c->ULconf, c->lo_bytes,
                        cudaMemcpyDeviceToDevice, c->stream);
  return e;
}

// pi <- Pi (the copy in updateUandcopyDown)
cudaError_t copy_down(askja_ctx* c) {
  if (!c->split) return cudaMemcpyAsync(c->P, c->P2, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream);
  cudaError_t e = cudaMemcpyAsync(c->PC, c->P2C, c->coef_bytes, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->PCL, c->P2CL, c->coefl_bytes, cudaMemcpyDeviceToDevice, c->stream);
  return e;
}

// the kick (mode 0) or fused kick + drift (mode 1) on pi (which 0) or Pi (1)
// into pi / Pi, links into the partner buffer (mode 1)
cudaError_t force_launch(askja_ctx* c, int mode, int in, int out, double ek, double ed) {
  if (c->split) {
    void* Uo = mode == 1 ? c->U[1 - c->cur] : nullptr;
    void* ULo = mode == 1 ? c->UL[1 - c->cur] : nullptr;
    return askja::splitk::force(c->lc, mode, cur_u(c), cur_ul(c), in ? c->P2C : c->PC, in ? c->P2CL : c->PCL,
                                out ? c->P2C : c->PC, out ? c->P2CL : c->PCL, Uo, ULo, ek, ed);
  }
  return c->ks->force(c->lc, mode, cur_u(c), in ? c->P2 : c->P, out ? c->P2 : c->P,
                      mode == 1 ? c->U[1 - c->cur] : nullptr, ek, ed);
}

// U <- exp(i eps Pi) U in place (updateUandcopyDown before its copy)
cudaError_t drift_launch(askja_ctx* c, double eps) {
  if (c->split) return askja::splitk::drift(c->lc, cur_u(c), cur_ul(c), c->P2C, c->P2CL, eps);
  return c->ks->drift(c->lc, cur_u(c), c->P2, eps);
}

cudaError_t plaq_launch(askja_ctx* c) {
  if (c->split) return askja::splitk::plaq(c->lc, cur_u(c), cur_ul(c), c->partial, c->sums);
  return c->ks->plaq(c->lc, cur_u(c), c->partial, c->sums);
}

// link sums into sums[2..4]: Pa / Pb = 0 pi, 1 Pi, -1 none
cudaError_t linksums_launch(askja_ctx* c, int pa, int pb, bool with_u) {
  if (c->split) {
    auto hi = [&](int w) -> const void* { return w < 0 ? nullptr : w ? c->P2C : c->PC; };
    auto lo = [&](int w) -> const void* { return w < 0 ? nullptr : w ? c->P2CL : c->PCL; };
    return askja::splitk::linksums(c->lc, hi(pa), lo(pa), hi(pb), lo(pb), with_u ? cur_u(c) : nullptr,
                                   with_u ? cur_ul(c) : nullptr, c->partial, c->sums + 2);
  }
  auto m = [&](int w) -> const void* { return w < 0 ? nullptr : w ? c->P2 : c->P; };
  return c->ks->linksums(c->lc, m(pa), m(pb), with_u ? cur_u(c) : nullptr, c->partial, c->sums + 2);
}

cudaError_t refresh_launch(askja_ctx* c, uint64_t seed, const unsigned long long* traj_dev,
                           unsigned long long traj_host) {
  const double scale = std::sqrt(2.0 * c->N / c->p.beta);
  if (c->split) return askja::splitk::refresh(c->lc, c->PC, c->PCL, seed, traj_dev, traj_host, scale);
  return c->ks->refresh(c->lc, c->P, seed, traj_dev, traj_host, scale);
}

// full FP32 matrices of pi and Pi in P / P2 (residual-plane mode) for the
// kernels that read momentum matrices
cudaError_t momenta_views(askja_ctx* c) {
  if (!c->split) return cudaSuccess;
  cudaError_t e = askja::splitk::momenta_to_matrix(c->lc, c->PC, c->PCL, c->P);
  if (e == cudaSuccess) e = askja::splitk::momenta_to_matrix(c->lc, c->P2C, c->P2CL, c->P2);
  return e;
}

int launch_ok(askja_ctx* c, cudaError_t e, const char* what) {
  if (e != cudaSuccess) return set_err(c, ASKJA_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return ASKJA_OK;
}

#define KL(expr, what)                            \
  do {                                            \
    int rc_ = launch_ok(c, (expr), what);         \
    if (rc_) return rc_;                          \
  } while (0)

// whether the fused kick+drift runs on the row-per-thread kernels
bool uses_rows(const askja_ctx* c) {
  return c->lc.force_rows == 1 || (c->lc.force_rows == 0 && c->N > 4);
}

bool paired(const askja_ctx* c) { return c->lc.force_rows == 3; }

// Site-pair mapping: the fused kick+drift launches run on the site-pair
// layout of the current links and of P; this converts both, in place, before
// (and again after) a run of such launches.  A no-op for the other mappings.
int pair_layout(askja_ctx* c, void* P) {
  if (!paired(c)) return ASKJA_OK;
  KL(c->ks->pair_swap(c->lc, cur_u(c)), "site-pair layout");
  KL(c->ks->pair_swap(c->lc, P), "site-pair layout");
  return ASKJA_OK;
}

// n fused kick+drift launches: the first kicks by first_kick, the others by dt
int fused_steps(askja_ctx* c, int n, double first_kick, double dt) {
  if (n <= 0) return ASKJA_OK;
  if (int rc = pair_layout(c, c->P)) return rc;
  for (int i = 0; i < n; i++) {
    KL(force_launch(c, 1, 0, 0, i == 0 ? first_kick : dt, dt), "kick+drift");
    c->cur ^= 1;
  }
  return pair_layout(c, c->P);
}

// Enqueue one whole trajectory (no host synchronisation; graph-capturable).
int enqueue_trajectory(askja_ctx* c, int nsteps) {
  Range r("askja: enqueue trajectory");
  const double dt = c->p.dt;
  if (c->split && c->lc.reunit) {
    // residual-plane mode: the link updates are not projected; every
    // trajectory starts from links projected onto SU(N) in FP64 (the saved
    // copy follows, so a rejected trajectory restores projected links)
    KL(askja::splitk::reunit(c->lc, cur_u(c), cur_ul(c), c->Uconf, c->ULconf), "reunitarise");
  } else if (c->lc.reunit && (c->lc.force_rows == 2 || (c->lc.rows_ns && uses_rows(c)))) {
    // the tensor-core link update keeps U' exactly as unitary as U (it
    // projects exp(i eps P), not U'); the rounding defect U accumulates (an
    // unbiased random walk, ~6e-8 sqrt(MD steps)) is removed here, before
    // every askja::FULL_REUNIT_EVERY-th trajectory, and the saved copy follows.  The
    // FP32 row kernels project each update by a Newton-Schulz step, which
    // leaves the determinant phase free; this pass pins it back to 1.
    askja::LaunchCtx lc = c->lc;
    lc.gate = &c->st->traj;
    lc.gate_every = askja::FULL_REUNIT_EVERY;
    KL(c->ks->reunit(lc, cur_u(c)), "reunitarise");
    KL(cudaMemcpyAsync(c->Uconf, cur_u(c), c->field_bytes, cudaMemcpyDeviceToDevice, c->stream), "save links");
  }
  {
    Range rh("askja: refresh + H_old");
    KL(refresh_launch(c, c->p.seed, &c->st->traj, 0), "refresh");
    KL(plaq_launch(c), "plaq");
    KL(linksums_launch(c, 0, -1, false), "kinetic");
    askja::misc::k_energy<<<1, 1, 0, c->stream>>>(c->sums, c->p.beta, c->N, &c->st->h_old);
    KL(cudaGetLastError(), "energy");
  }
  {
    Range rl("askja: leapfrog");
    if (int rc = fused_steps(c, nsteps, 0.5 * dt, dt)) return rc;
  }
  Range rm("askja: H_new + Metropolis");
  KL(force_launch(c, 0, 0, 0, 0.5 * dt, 0.0), "kick");
  KL(plaq_launch(c), "plaq");
  KL(linksums_launch(c, 0, -1, false), "kinetic");
  askja::misc::k_energy<<<1, 1, 0, c->stream>>>(c->sums, c->p.beta, c->N, &c->st->h_new);
  askja::misc::k_metropolis<<<1, 1, 0, c->stream>>>(c->st, c->p.seed, c->logbuf, c->logcap);
  askja::misc::k_accept_copy<<<4 * 148, 256, 0, c->stream>>>(c->st, (uint4*)cur_u(c), (uint4*)c->Uconf,
                                                             (long)(c->field_bytes / 16));
  if (c->split)
    askja::misc::k_accept_copy<<<4 * 148, 256, 0, c->stream>>>(c->st, (uint4*)cur_ul(c), (uint4*)c->ULconf,
                                                               (long)(c->lo_bytes / 16));
  KL(cudaGetLastError(), "metropolis");
  return ASKJA_OK;
}

void drop_graphs(askja_ctx* c) {
  for (int i = 0; i < 2; i++) {
    if (c->gexec[i]) cudaGraphExecDestroy(c->gexec[i]);
    c->gexec[i] = nullptr;
    c->g_nsteps[i] = -1;
  }
}

// synchronise the stream and report a tensor-core kernel that stopped after a
// bounded wait (its outputs are incomplete)
int sync_checked(askja_ctx* c) {
  CK(cudaStreamSynchronize(c->stream));
  if (c->up_bad) {
    unsigned long long bad = 0;
    CK(cudaMemcpy(&bad, c->up_bad, sizeof bad, cudaMemcpyDeviceToHost));
    if (bad) {
      CK(cudaMemset(c->up_bad, 0, sizeof bad));
      return set_err(c, ASKJA_ERR_NONFINITE, "an asynchronous upload held %llu non-finite values", bad);
    }
  }
  if (c->lc.force_rows == 2) {
    unsigned st = 0;
    CK(cudaMemcpy(&st, c->tc_status, sizeof st, cudaMemcpyDeviceToHost));
    if (st) {
      CK(cudaMemset(c->tc_status, 0, sizeof st));
      return set_err(c, ASKJA_ERR_CUDA, "tensor-core link update gave up waiting for its MMA");
    }
  }
  return ASKJA_OK;
}

// kind of a device field for the conversions: the links (current or saved) or a momentum buffer
enum class FieldKind { links, saved_links, pi, Pi };

// U-conf layout (FP64) -> device field; in the residual-plane mode `dst` is
// ignored and the kind picks the hi/lo (links) or coordinate (momenta) buffers
cudaError_t from_conf_launch(askja_ctx* c, const void* conf, void* dst, FieldKind kind) {
  if (!c->split) return c->ks->from_conf(c->lc, conf, dst);
  switch (kind) {
    case FieldKind::links:
      return askja::splitk::links_from_conf(c->lc, conf, cur_u(c), cur_ul(c));
    case FieldKind::saved_links:
      return askja::splitk::links_from_conf(c->lc, conf, c->Uconf, c->ULconf);
    case FieldKind::pi:
      return askja::splitk::momenta_from_conf(c->lc, conf, c->PC, c->PCL);
    case FieldKind::Pi:
      return askja::splitk::momenta_from_conf(c->lc, conf, c->P2C, c->P2CL);
  }
  return cudaErrorInvalidValue;
}

cudaError_t to_conf_launch(askja_ctx* c, const void* src, void* conf, FieldKind kind) {
  if (!c->split) return c->ks->to_conf(c->lc, src, conf);
  switch (kind) {
    case FieldKind::links:
      return askja::splitk::links_to_conf(c->lc, cur_u(c), cur_ul(c), conf);
    case FieldKind::saved_links:
      return askja::splitk::links_to_conf(c->lc, c->Uconf, c->ULconf, conf);
    case FieldKind::pi:
      return askja::splitk::momenta_to_conf(c->lc, c->PC, c->PCL, conf);
    case FieldKind::Pi:
      return askja::splitk::momenta_to_conf(c->lc, c->P2C, c->P2CL, conf);
  }
  return cudaErrorInvalidValue;
}

int read_state(askja_ctx* c, askja_traj_result* out) {
  if (!out) return sync_checked(c);
  CK(cudaMemcpyAsync(out, c->st, sizeof(TrajState), cudaMemcpyDeviceToHost, c->stream));
  return sync_checked(c);
}

int upload_conf(askja_ctx* c, const double* conf, void* dst, FieldKind kind = FieldKind::links) {
  const size_t bytes = (size_t)c->nl * c->N * c->N * 2 * sizeof(double);
  CK(cudaMemcpyAsync(c->staging, conf, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->nonfinite, 0, sizeof(unsigned long long), c->stream));
  askja::misc::k_count_nonfinite<<<4 * 148, 256, 0, c->stream>>>((const double*)c->staging,
                                                                  (long)(bytes / sizeof(double)), c->nonfinite);
  unsigned long long bad = 0;
  CK(cudaMemcpyAsync(&bad, c->nonfinite, sizeof bad, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (bad) return set_err(c, ASKJA_ERR_NONFINITE, "input buffer holds %llu non-finite values", bad);
  KL(from_conf_launch(c, c->staging, dst, kind), "from_conf");
  return ASKJA_OK;
}

int download_conf(askja_ctx* c, const void* src, double* conf, FieldKind kind = FieldKind::links) {
  const size_t bytes = (size_t)c->nl * c->N * c->N * 2 * sizeof(double);
  KL(to_conf_launch(c, src, c->staging, kind), "to_conf");
  CK(cudaMemcpyAsync(conf, c->staging, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

}  // namespace

// Lets entry points without a context (static_plaq.cu) report through
// askja_last_error(NULL).
void askja_internal_set_error(const char* msg) { g_last_error = msg; }

extern "C" {

const char* askja_version(void) { return "askja-b200 0.1 (sm_100a)"; }

const char* askja_last_error(const askja_ctx* c) { return c ? c->err.c_str() : g_last_error.c_str(); }

long askja_volume(const askja_ctx* c) { return c ? c->V : -1; }

void* askja_stream(askja_ctx* c) { return c ? (void*)c->stream : nullptr; }

int askja_sync(askja_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  return sync_checked(c);
}

void askja_destroy(askja_ctx* c) {
  if (!c) return;
  DevGuard g(c->p.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  drop_graphs(c);
  for (int b = 0; b < 2; b++) {
    if (c->up[b]) cudaFree(c->up[b]);
    if (c->up_copied[b]) cudaEventDestroy(c->up_copied[b]);
    if (c->up_free[b]) cudaEventDestroy(c->up_free[b]);
  }
  if (c->up_bad) cudaFree(c->up_bad);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  void* bufs[] = {c->U[0], c->U[1], c->P,      c->P2,      c->Uconf,     c->nbr,       c->partial, c->sums,
                  c->lines, c->st,  c->logbuf, c->staging, c->nonfinite, c->tc_status, c->eigs,    c->eigfail,
                  c->UL[0], c->UL[1], c->ULconf, c->PC, c->PCL, c->P2C, c->P2CL};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int askja_create(const askja_params* p, askja_ctx** out) {
  askja_ctx* c = nullptr;
  if (!p || !out) return set_err(nullptr, ASKJA_ERR_ARG, "null argument");
  *out = nullptr;
  if (p->nc < 2 || p->nc > ASKJA_MAX_NC) return set_err(nullptr, ASKJA_ERR_ARG, "NC=%d outside 2..%d", p->nc, ASKJA_MAX_NC);
  if (p->dim < 1 || p->dim > ASKJA_MAX_DIM)
    return set_err(nullptr, ASKJA_ERR_ARG, "DIM=%d outside 1..%d", p->dim, ASKJA_MAX_DIM);
  long V = 1;
  for (int i = 0; i < p->dim; i++) {
    if (p->n[i] < 1) return set_err(nullptr, ASKJA_ERR_ARG, "N%d=%d must be >= 1", i, p->n[i]);
    V *= p->n[i];
    if (V > (1L << 30)) return set_err(nullptr, ASKJA_ERR_ARG, "volume too large");
  }
  if (!(p->beta > 0.0) || !std::isfinite(p->beta)) return set_err(nullptr, ASKJA_ERR_ARG, "BETA must be > 0");
  if (p->precision != ASKJA_FP64 && p->precision != ASKJA_FP32 && p->precision != ASKJA_FP32_LEAN)
    return set_err(nullptr, ASKJA_ERR_ARG, "unknown precision %d", p->precision);
  if (p->kernel_path < 0 || p->kernel_path > 3)
    return set_err(nullptr, ASKJA_ERR_ARG, "unknown kernel path %d", p->kernel_path);
  if (p->kernel_path == 2 && !askja::tc_supported(p->nc, p->dim, p->precision == ASKJA_FP64))
    return set_err(nullptr, ASKJA_ERR_ARG, "tensor-core path needs FP32, NC = 32 or 64 and DIM >= 2");
  if (p->kernel_path == 3 && !askja::pair_supported(p->nc, p->dim, p->precision == ASKJA_FP64, p->n[p->dim - 1]))
    return set_err(nullptr, ASKJA_ERR_ARG, "site-pair path needs FP32, NC = 3, DIM >= 2 and an even N%d",
                   p->dim - 1);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(nullptr, ASKJA_ERR_NODEVICE, "no CUDA device available (the engine has no CPU fallback)");
  if (p->device < 0 || p->device >= ndev) return set_err(nullptr, ASKJA_ERR_ARG, "device %d not present", p->device);

  c = new askja_ctx();
  c->p = *p;
  DevGuard g(p->device);
  c->N = p->nc;
  c->D = p->dim;
  c->V = V;
  c->nl = V * p->dim;
  c->ks = p->precision == ASKJA_FP64 ? &askja::kernels_fp64 : &askja::kernels_fp32;
  // residual planes: ASKJA_FP32 on the thread-per-link mapping (NC <= 4, automatic kernel path)
  c->split = p->precision == ASKJA_FP32 && askja::splitk::supported(p->nc) && p->kernel_path == 0;
  const size_t elem = p->precision == ASKJA_FP64 ? 16 : 8;
  Lat& L = c->lat;
  L.V = (int)V;
  L.B = (int)((V + 31) / 32);
  L.D = p->dim;
  L.N = p->nc;
  c->field_bytes = askja::field_elems(L) * elem;
  for (int i = 0; i < p->dim; i++) {
    L.n[i] = p->n[i];
    long s = 1;
    for (int j = i + 1; j < p->dim; j++) s *= p->n[j];
    L.stride[i] = (int)s;
  }
  auto fail = [&](int rc) {
    g_last_error = c->err;
    askja_destroy(c);
    return rc;
  };
#define CKC(call)                                                                                          \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return fail(set_err(c, ASKJA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_))); \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  for (void** b : {&c->U[0], &c->U[1], &c->P, &c->P2, &c->Uconf}) CKC(cudaMalloc(b, c->field_bytes));
  std::vector<int> nbr;
  build_neighbours(*p, V, nbr);
  CKC(cudaMalloc(&c->nbr, nbr.size() * sizeof(int)));
  CKC(cudaMemcpy(c->nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice));
  L.nbr = c->nbr;
  CKC(cudaMalloc(&c->partial, askja::partial_doubles(L) * sizeof(double)));
  CKC(cudaMalloc(&c->sums, 64 * sizeof(double)));
  long maxlines = 1;
  for (int i = 0; i < p->dim; i++) maxlines = std::max(maxlines, (long)p->n[i]);
  CKC(cudaMalloc(&c->lines, (maxlines + 8) * sizeof(double)));
  if (p->dim >= 2) {
    CKC(cudaMalloc(&c->eigs, (size_t)(p->n[0] + p->n[1]) * p->nc * sizeof(double2)));
    CKC(cudaMalloc(&c->eigfail, sizeof(int)));
  }
  CKC(cudaMalloc(&c->st, sizeof(TrajState)));
  CKC(cudaMemset(c->st, 0, sizeof(TrajState)));
  c->logcap = 4096;
  CKC(cudaMalloc(&c->logbuf, (size_t)4 * c->logcap * sizeof(double)));
  CKC(cudaMalloc(&c->staging, (size_t)c->nl * c->N * c->N * 2 * sizeof(double)));
  CKC(cudaMalloc(&c->nonfinite, sizeof(unsigned long long)));
  for (void* b : {c->U[0], c->U[1], c->P, c->P2, c->Uconf}) CKC(cudaMemset(b, 0, c->field_bytes));
  if (c->split) {
    c->lo_bytes = askja::field_elems(L) * sizeof(uint32_t);
    c->coef_bytes = askja::splitk::coef_floats(L) * sizeof(float);
    c->coefl_bytes = askja::splitk::coef_words(L) * sizeof(uint32_t);
    for (void** b : {&c->UL[0], &c->UL[1], &c->ULconf}) {
      CKC(cudaMalloc(b, c->lo_bytes));
      CKC(cudaMemset(*b, 0, c->lo_bytes));
    }
    for (void** b : {&c->PC, &c->P2C}) {
      CKC(cudaMalloc(b, c->coef_bytes));
      CKC(cudaMemset(*b, 0, c->coef_bytes));
    }
    for (void** b : {&c->PCL, &c->P2CL}) {
      CKC(cudaMalloc(b, c->coefl_bytes));
      CKC(cudaMemset(*b, 0, c->coefl_bytes));
    }
  }
  c->lc.lat = L;
  c->lc.stream = c->stream;
  c->lc.order = askja::taylor_order(p->level);
  c->lc.reunit = p->reunitarise < 0 ? (p->precision == ASKJA_FP32) : (p->reunitarise != 0);
  c->lc.rows_ns = p->precision == ASKJA_FP32;
  CKC(cudaMalloc(&c->tc_status, sizeof(unsigned)));
  CKC(cudaMemset(c->tc_status, 0, sizeof(unsigned)));
  c->lc.scratch = c->staging;
  c->lc.status = c->tc_status;
  // untuned default: tensor cores for NC = 32 and 64, else thread-per-link for NC <= 4 (rows above);
  // NC = 16 on the tensor cores is an explicit path and an autotuner candidate
  c->lc.force_rows = p->kernel_path != 0 ? p->kernel_path
                     : (p->nc >= 32 && askja::tc_supported(p->nc, p->dim, p->precision == ASKJA_FP64)) ? 2
                                                                                                      : 0;
  c->lc.rows_groups = 0;
  c->lc.small_occ = 0;
  if (p->kernel_path == 0) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(std::make_tuple(p->nc, p->dim, p->precision));
    if (it != g_tune_cache.end() &&
        (it->second.path != 3 || askja::pair_supported(p->nc, p->dim, p->precision == ASKJA_FP64, p->n[p->dim - 1]))) {
      c->lc.force_rows = it->second.path;
      c->lc.rows_groups = it->second.groups;
      c->lc.small_occ = it->second.occupancy;
    }
  }
  // cold start by default
  if (c->ks->identity(c->lc, c->U[0]) != cudaSuccess) return fail(set_err(c, ASKJA_ERR_CUDA, "identity launch"));
  CKC(cudaMemcpyAsync(c->Uconf, c->U[0], c->field_bytes, cudaMemcpyDeviceToDevice, c->stream));
  CKC(cudaStreamSynchronize(c->stream));
#undef CKC
  *out = c;
  return ASKJA_OK;
}

int askja_set_links(askja_ctx* c, const double* conf) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_set_links");
  if (!conf) return set_err(c, ASKJA_ERR_ARG, "null buffer");
  DevGuard g(c->p.device);
  if (int rc = upload_conf(c, conf, cur_u(c))) return rc;
  CK(copy_saved(c, true));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_set_links_async(askja_ctx* c, const double* conf) {
  if (int rc = check_ctx(c)) return rc;
  if (!conf) return set_err(c, ASKJA_ERR_ARG, "null buffer");
  DevGuard g(c->p.device);
  const size_t bytes = (size_t)c->nl * c->N * c->N * 2 * sizeof(double);
  if (!c->copy_stream) {
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; b++) {
      CK(cudaMalloc(&c->up[b], bytes));
      CK(cudaEventCreateWithFlags(&c->up_copied[b], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->up_free[b], cudaEventDisableTiming));
    }
    CK(cudaMalloc(&c->up_bad, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(c->up_bad, 0, sizeof(unsigned long long), c->stream));
  }
  const int b = c->up_next;
  c->up_next ^= 1;
  // the copy waits for the conversion that last read this staging buffer (an
  // event never recorded counts as complete), then overlaps whatever the
  // engine's stream is running; the conversion is ordered after that work
  CK(cudaStreamWaitEvent(c->copy_stream, c->up_free[b], 0));
  CK(cudaMemcpyAsync(c->up[b], conf, bytes, cudaMemcpyHostToDevice, c->copy_stream));
  CK(cudaEventRecord(c->up_copied[b], c->copy_stream));
  CK(cudaStreamWaitEvent(c->stream, c->up_copied[b], 0));
  askja::misc::k_count_nonfinite<<<4 * 148, 256, 0, c->stream>>>((const double*)c->up[b],
                                                                  (long)(bytes / sizeof(double)), c->up_bad);
  KL(cudaGetLastError(), "non-finite check");
  KL(from_conf_launch(c, c->up[b], cur_u(c), FieldKind::links), "from_conf");
  CK(copy_saved(c, true));
  CK(cudaEventRecord(c->up_free[b], c->stream));
  return ASKJA_OK;
}

int askja_get_links(askja_ctx* c, double* conf) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_get_links");
  if (!conf) return set_err(c, ASKJA_ERR_ARG, "null buffer");
  DevGuard g(c->p.device);
  return download_conf(c, cur_u(c), conf);
}

int askja_get_saved_links(askja_ctx* c, double* conf) {
  if (int rc = check_ctx(c)) return rc;
  if (!conf) return set_err(c, ASKJA_ERR_ARG, "null buffer");
  DevGuard g(c->p.device);
  return download_conf(c, c->Uconf, conf, FieldKind::saved_links);
}

int askja_set_momenta(askja_ctx* c, int which, const double* conf) {
  if (int rc = check_ctx(c)) return rc;
  if (!conf || (which != 0 && which != 1)) return set_err(c, ASKJA_ERR_ARG, "bad momentum buffer selector");
  DevGuard g(c->p.device);
  if (int rc = upload_conf(c, conf, which ? c->P2 : c->P, which ? FieldKind::Pi : FieldKind::pi)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_get_momenta(askja_ctx* c, int which, double* conf) {
  if (int rc = check_ctx(c)) return rc;
  if (!conf || (which != 0 && which != 1)) return set_err(c, ASKJA_ERR_ARG, "bad momentum buffer selector");
  DevGuard g(c->p.device);
  return download_conf(c, which ? c->P2 : c->P, conf, which ? FieldKind::Pi : FieldKind::pi);
}

int askja_initializeU(askja_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  KL(c->ks->identity(c->lc, cur_u(c)), "identity");
  if (c->split) CK(cudaMemsetAsync(cur_ul(c), 0, c->lo_bytes, c->stream));
  CK(copy_saved(c, true));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_hot_start(askja_ctx* c, uint64_t seed) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  KL(c->ks->gauss_matrices(c->lc, cur_u(c), seed), "gaussian matrices");
  // Gram-Schmidt + determinant phase always, whatever the reunitarise setting
  if (c->split) {
    CK(cudaMemsetAsync(cur_ul(c), 0, c->lo_bytes, c->stream));
    KL(askja::splitk::reunit(c->lc, cur_u(c), cur_ul(c)), "reunitarise");
  } else {
    LaunchCtx lc = c->lc;
    KL(c->ks->reunit(lc, cur_u(c)), "reunitarise");
  }
  CK(copy_saved(c, true));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_initializeE(askja_ctx* c, uint64_t seed, uint64_t counter) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  KL(refresh_launch(c, seed, nullptr, (unsigned long long)counter), "refresh");
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_updateE(askja_ctx* c, double eps) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  KL(force_launch(c, 0, 0, 1, eps, 0.0), "updateE");
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_updateUandcopyDown(askja_ctx* c, double eps) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  KL(drift_launch(c, eps), "drift");
  CK(copy_down(c));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_copyDown(askja_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  CK(copy_down(c));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_takeconfiguration(askja_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  CK(copy_saved(c, true));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_loadconfiguration(askja_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  CK(copy_saved(c, false));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_reunitarise(askja_ctx* c) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  if (c->split)
    KL(askja::splitk::reunit(c->lc, cur_u(c), cur_ul(c)), "reunitarise");
  else
    KL(c->ks->reunit(c->lc, cur_u(c)), "reunitarise");
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_PlaqExp(askja_ctx* c, double* temporal, double* spatial) {
  if (int rc = check_ctx(c)) return rc;
  DevGuard g(c->p.device);
  KL(plaq_launch(c), "plaq");
  double h[2];
  if (int rc = scal(c, c->sums, h, 2)) return rc;
  if (temporal) *temporal = h[0];
  if (spatial) *spatial = h[1];
  return ASKJA_OK;
}

int askja_EnergyMag(askja_ctx* c, double* out) {
  double t = 0, s = 0;
  if (int rc = askja_PlaqExp(c, &t, &s)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  *out = t + s;
  return ASKJA_OK;
}

// pa / pb: 0 pi, 1 Pi, -1 none
static int linksums(askja_ctx* c, int pa, int pb, bool with_u, double h[3]) {
  DevGuard g(c->p.device);
  KL(linksums_launch(c, pa, pb, with_u), "linksums");
  return scal(c, c->sums + 2, h, 3);
}

int askja_simpleenergyEl(askja_ctx* c, int which, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out || (which != 0 && which != 1)) return set_err(c, ASKJA_ERR_ARG, "bad argument");
  double h[3];
  if (int rc = linksums(c, which, -1, false, h)) return rc;
  *out = h[0];
  return ASKJA_OK;
}

int askja_EnergyEl(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  double h[3];
  if (int rc = linksums(c, 0, 1, false, h)) return rc;
  *out = h[1];
  return ASKJA_OK;
}

int askja_UViol(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  double h[3];
  if (int rc = linksums(c, -1, -1, true, h)) return rc;
  *out = h[2];
  return ASKJA_OK;
}

int askja_TotalEnergy(askja_ctx* c, double* out) {
  double em = 0, el = 0;
  if (int rc = askja_EnergyMag(c, &em)) return rc;
  if (int rc = askja_EnergyEl(c, &el)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  *out = 2.0 * c->N * em + el;
  return ASKJA_OK;
}

int askja_GaussLaw(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  DevGuard g(c->p.device);
  KL(momenta_views(c), "momentum matrices");
  KL(c->ks->gauss(c->lc, cur_u(c), c->P2, c->partial, c->sums + 5), "gauss");
  return scal(c, c->sums + 5, out, 1);
}

static int line_mean(askja_ctx* c, int dir, int nlines, int start_stride, double* out) {
  DevGuard g(c->p.device);
  KL(c->ks->lines(c->lc, cur_u(c), dir, nlines, start_stride, c->lines), "lines");
  std::vector<double> h(nlines);
  if (int rc = scal(c, c->lines, h.data(), nlines)) return rc;
  double s = 0;
  for (double v : h) s += v;
  *out = s / nlines;
  return ASKJA_OK;
}

int askja_WilsonLoop(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  return line_mean(c, 0, 1, 0, out);
}

int askja_PolyakovLoop(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  if (c->D < 2) return set_err(c, ASKJA_ERR_ARG, "PolyakovLoop needs DIM >= 2");
  return line_mean(c, 0, c->lat.n[1], c->lat.stride[1], out);
}

int askja_WilsonLoopDir(askja_ctx* c, int dir, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out || dir < 1 || dir >= c->D) return set_err(c, ASKJA_ERR_ARG, "WilsonLoopDir needs 1 <= dir < DIM");
  return line_mean(c, dir, c->lat.n[0], c->lat.stride[0], out);
}

int askja_eigenphases(askja_ctx* c, double* w, double* p) {
  if (int rc = check_ctx(c)) return rc;
  if (!w || !p) return set_err(c, ASKJA_ERR_ARG, "null output");
  if (c->D < 2) return set_err(c, ASKJA_ERR_ARG, "eigenphases need DIM >= 2");
  DevGuard g(c->p.device);
  const int N = c->N, n0 = c->lat.n[0], n1 = c->lat.n[1];
  CK(cudaMemsetAsync(c->eigfail, 0, sizeof(int), c->stream));
  // Wilson lines along direction 1 through (x0, 0, ..), Polyakov lines along 0 through (0, x1, 0, ..)
  KL(c->ks->line_eigs(c->lc, cur_u(c), 1, n0, c->lat.stride[0], c->eigs, c->eigfail), "line eigenvalues");
  KL(c->ks->line_eigs(c->lc, cur_u(c), 0, n1, c->lat.stride[1], c->eigs + (size_t)n0 * N, c->eigfail),
     "line eigenvalues");
  std::vector<double2> ev((size_t)(n0 + n1) * N);
  int fail = 0;
  CK(cudaMemcpyAsync(ev.data(), c->eigs, ev.size() * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&fail, c->eigfail, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (fail) return set_err(c, ASKJA_ERR_CUDA, "line eigenvalues did not converge");
  // per line: phases, re-centred by the winding when |winding| > 0.1, sorted, summed; then averaged
  const double pi = 3.14159265358979323846;
  std::vector<double> ph(N);
  for (int i = 0; i < N; i++) w[i] = p[i] = 0.0;
  for (int q = 0; q < n0 + n1; q++) {
    double winding = 0.0;
    for (int i = 0; i < N; i++) {
      const double2 z = ev[(size_t)q * N + i];
      ph[i] = std::atan2(z.y, z.x);
      winding += ph[i] / (2 * pi);
    }
    if (winding > 0.1 || winding < -0.1)
      for (int i = 0; i < N; i++) ph[i] -= winding * 2 * pi / N;
    std::sort(ph.begin(), ph.end());
    double* acc = q < n0 ? w : p;
    for (int i = 0; i < N; i++) acc[i] += ph[i];
  }
  for (int i = 0; i < N; i++) {
    w[i] /= n0;
    p[i] /= n1;
  }
  return ASKJA_OK;
}

int askja_scalarLoopcorr(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  DevGuard g(c->p.device);
  KL(c->ks->slice_trace(c->lc, cur_u(c), c->lines), "slice trace");
  return scal(c, c->lines, out, c->lat.n[0]);
}

// Short names for the seam functions (same calls, same semantics).
int askja_force_step(askja_ctx* c, double eps) { return askja_updateE(c, eps); }
int askja_link_step(askja_ctx* c, double eps) { return askja_updateUandcopyDown(c, eps); }
int askja_action(askja_ctx* c, double* s_over_beta) { return askja_EnergyMag(c, s_over_beta); }
int askja_kinetic(askja_ctx* c, double* trp2) { return askja_simpleenergyEl(c, 0, trp2); }
int askja_refresh_momenta(askja_ctx* c, uint64_t seed, uint64_t counter) {
  return askja_initializeE(c, seed, counter);
}

int askja_measure(askja_ctx* c, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  if (c->D < 2) return set_err(c, ASKJA_ERR_ARG, "askja_measure needs DIM >= 2");
  if (int rc = askja_PlaqExp(c, out, out + 1)) return rc;
  if (int rc = askja_PolyakovLoop(c, out + 2)) return rc;
  for (int d = 1; d < c->D; d++)
    if (int rc = askja_WilsonLoopDir(c, d, out + 2 + d)) return rc;
  if (int rc = askja_GaussLaw(c, out + c->D + 2)) return rc;
  return askja_UViol(c, out + c->D + 3);
}

int askja_FourierTrafo(askja_ctx* c, double* coefficients) {
  if (int rc = check_ctx(c)) return rc;
  if (!coefficients) return set_err(c, ASKJA_ERR_ARG, "null output");
  if (c->N > 64) return set_err(c, ASKJA_ERR_ARG, "FourierTrafo: NC <= 64");
  DevGuard g(c->p.device);
  const int n = c->lat.n[0];
  KL(c->ks->fourier(c->lc, cur_u(c), n, c->partial, c->lines), "FourierTrafo");
  return scal(c, c->lines, coefficients, n);
}

// Tab of sites [site0, site0 + nsites) into the device buffer out (k*npt + m)
static int tab_range(askja_ctx* c, long site0, long nsites, int npt, double* out_dev) {
  if (c->D > 8 || c->N > 64) return set_err(c, ASKJA_ERR_ARG, "Tab: DIM <= 8 and NC <= 64");
  if (npt < 2 || npt > c->D + 2) return set_err(c, ASKJA_ERR_ARG, "Tab: Npt must be in 2..DIM+2 (got %d)", npt);
  KL(momenta_views(c), "momentum matrices");
  KL(c->ks->tab(c->lc, cur_u(c), c->P, c->P2, (int)site0, (int)nsites, npt, out_dev), "Tab");
  return ASKJA_OK;
}

int askja_Tab(askja_ctx* c, long site, double* mdata, int npt) {
  if (int rc = check_ctx(c)) return rc;
  if (!mdata) return set_err(c, ASKJA_ERR_ARG, "null output");
  if (site < 0 || site >= c->V) return set_err(c, ASKJA_ERR_ARG, "site %ld outside 0..%ld", site, c->V - 1);
  DevGuard g(c->p.device);
  if (int rc = tab_range(c, site, 1, npt, c->partial)) return rc;  // partial: >= 64 doubles
  double v[10];
  if (int rc = scal(c, c->partial, v, npt)) return rc;
  for (int m = 0; m < npt; m++) mdata[m] += v[m];  // the reference accumulates into mdata
  return ASKJA_OK;
}

int askja_Tab_all(askja_ctx* c, int npt, double* out) {
  if (int rc = check_ctx(c)) return rc;
  if (!out) return set_err(c, ASKJA_ERR_ARG, "null output");
  DevGuard g(c->p.device);
  // the staging buffer (V*DIM*NC*NC double2) holds V*(DIM+2) doubles
  if (int rc = tab_range(c, 0, c->V, npt, (double*)c->staging)) return rc;
  CK(cudaMemcpyAsync(out, c->staging, sizeof(double) * npt * (size_t)c->V, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_leapfrog(askja_ctx* c, int nsteps, double eps) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_leapfrog");
  if (nsteps < 1) return set_err(c, ASKJA_ERR_ARG, "nsteps must be >= 1");
  DevGuard g(c->p.device);
  if (int rc = fused_steps(c, nsteps, 0.5 * eps, eps)) return rc;
  KL(force_launch(c, 0, 0, 0, 0.5 * eps, 0.0), "kick");
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_md_steps(askja_ctx* c, int nsteps, double eps) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_md_steps");
  if (nsteps < 0) return set_err(c, ASKJA_ERR_ARG, "nsteps must be >= 0");
  if (nsteps == 0) return ASKJA_OK;
  DevGuard g(c->p.device);
  // D(eps) with Pi, pi = Pi ...
  KL(drift_launch(c, eps), "drift");
  CK(copy_down(c));
  // ... then (K D) fused, in place on pi ...
  if (int rc = fused_steps(c, nsteps - 1, eps, eps)) return rc;
  // ... and the last kick out of place: Pi = pi - eps F(u)
  KL(force_launch(c, 0, 0, 1, eps, 0.0), "kick");
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_trajectory(askja_ctx* c, int nsteps, askja_traj_result* out) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_trajectory");
  if (nsteps < 1) return set_err(c, ASKJA_ERR_ARG, "nsteps must be >= 1");
  DevGuard g(c->p.device);
  if (int rc = enqueue_trajectory(c, nsteps)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return read_state(c, out);
}

}  // extern "C"

namespace {

// Enqueue one trajectory, as a replay of the captured graph for this start
// buffer and step count when use_graph (captured on first use).
int launch_trajectory(askja_ctx* c, int nsteps, int use_graph) {
  if (!use_graph) return enqueue_trajectory(c, nsteps);
  const int start = c->cur;
  if (!c->gexec[start] || c->g_nsteps[start] != nsteps) {
    if (c->gexec[start]) cudaGraphExecDestroy(c->gexec[start]);
    c->gexec[start] = nullptr;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_trajectory(c, nsteps);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    c->cur = start;
    if (rc) return rc;
    if (ce != cudaSuccess) return set_err(c, ASKJA_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&c->gexec[start], graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return set_err(c, ASKJA_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    c->g_nsteps[start] = nsteps;
  }
  CK(cudaGraphLaunch(c->gexec[start], c->stream));
  c->cur = start ^ (nsteps & 1);
  return ASKJA_OK;
}

}  // namespace

extern "C" {

int askja_trajectory_async(askja_ctx* c, int nsteps, askja_traj_result* out) {
  if (int rc = check_ctx(c)) return rc;
  if (nsteps < 1) return set_err(c, ASKJA_ERR_ARG, "nsteps must be >= 1");
  DevGuard g(c->p.device);
  if (int rc = launch_trajectory(c, nsteps, 1)) return rc;
  if (out) CK(cudaMemcpyAsync(out, c->st, sizeof(TrajState), cudaMemcpyDeviceToHost, c->stream));
  return ASKJA_OK;
}

int askja_run_trajectories(askja_ctx* c, int ntraj, int nsteps, int use_graph, askja_traj_result* last,
                           double* log) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_run_trajectories");
  if (nsteps < 1 || ntraj < 0) return set_err(c, ASKJA_ERR_ARG, "bad trajectory counts");
  DevGuard g(c->p.device);
  TrajState st0;
  CK(cudaMemcpyAsync(&st0, c->st, sizeof st0, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int t = 0; t < ntraj; t++)
    if (int rc = launch_trajectory(c, nsteps, use_graph)) return rc;
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = read_state(c, last)) return rc;
  if (log && ntraj > 0) {
    std::vector<double> ring((size_t)4 * c->logcap);
    CK(cudaMemcpy(ring.data(), c->logbuf, ring.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int t = 0; t < ntraj; t++) {
      const unsigned long long k = (st0.traj + (unsigned long long)t) % (unsigned long long)c->logcap;
      // only the last logcap trajectories are kept
      if (ntraj - t > c->logcap) continue;
      memcpy(log + 4 * (size_t)t, ring.data() + 4 * k, 4 * sizeof(double));
    }
  }
  return ASKJA_OK;
}

int askja_set_tuning(askja_ctx* c, const askja_tuning* t) {
  if (int rc = check_ctx(c)) return rc;
  if (!t || t->path < 0 || t->path > 3 || (t->path == 0 && c->N > 4) || t->groups < 0 || (c->split && t->path != 0) ||
      (t->path == 2 && !askja::tc_supported(c->N, c->D, c->p.precision == ASKJA_FP64)) ||
      (t->path == 3 && !askja::pair_supported(c->N, c->D, c->p.precision == ASKJA_FP64, c->lat.n[c->D - 1])))
    return set_err(c, ASKJA_ERR_ARG, "invalid tuning");
  c->lc.force_rows = t->path;
  c->lc.rows_groups = t->groups;
  c->lc.small_occ = t->occupancy < 0 ? 0 : t->occupancy > 2 ? 2 : t->occupancy;
  drop_graphs(c);
  return ASKJA_OK;
}

int askja_autotune(askja_ctx* c, int reps, askja_tuning* out) {
  if (int rc = check_ctx(c)) return rc;
  Range range("askja_autotune");
  if (reps < 1) reps = 5;
  DevGuard g(c->p.device);
  struct Cand {
    int path, groups, occ;
  };
  std::vector<Cand> cands;
  const bool fp64 = c->p.precision == ASKJA_FP64;
  if (c->N <= 4) {
    cands.push_back({0, 0, 0});
    cands.push_back({0, 0, 1});
    cands.push_back({0, 0, 2});
  }
  if (askja::tc_supported(c->N, c->D, fp64)) cands.push_back({2, 0, 0});

  std::vector<int> seen;
  // the residual-plane mode has one mapping (thread per link); only its register budget is tuned
  for (int want : {0, 2, 4, 8, 16, 32, 64}) {
    if (c->split) break;
    const int eff = askja::rows_effective_groups(c->N, fp64, want);
    bool dup = false;
    for (int s : seen) dup |= s == eff;
    if (dup) continue;
    seen.push_back(eff);
    cands.push_back({1, eff, 0});
    // FP32 rows for 5 <= NC <= 8 (k_force8): the tighter register budgets at every sites-per-CTA choice
    if (!fp64 && c->N > 4 && c->N <= 8) {
      cands.push_back({1, eff, 1});
      cands.push_back({1, eff, 2});
    }
  }
  if (cands.size() > 24) cands.resize(24);
  // scratch: Pi holds a copy of pi, the partner link buffer receives the output
  CK(cudaMemcpyAsync(c->P2, c->P, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream));
  if (c->split) {
    CK(cudaMemcpyAsync(c->P2C, c->PC, c->coef_bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->P2CL, c->PCL, c->coefl_bytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  auto fused = [&](const askja::LaunchCtx& lc) -> cudaError_t {
    if (c->split)
      return askja::splitk::force(lc, 1, cur_u(c), cur_ul(c), c->P2C, c->P2CL, c->P2C, c->P2CL, c->U[1 - c->cur],
                                  c->UL[1 - c->cur], 0.5 * c->p.dt, c->p.dt);
    return c->ks->force(lc, 1, cur_u(c), c->P2, c->P2, c->U[1 - c->cur], 0.5 * c->p.dt, c->p.dt);
  };
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const askja::LaunchCtx saved = c->lc;
  askja_tuning res{};
  res.best_us = 1e300;
  int best = 0;
  for (size_t i = 0; i < cands.size(); i++) {
    askja::LaunchCtx lc = saved;
    lc.force_rows = cands[i].path;
    lc.rows_groups = cands[i].groups;
    lc.small_occ = cands[i].occ;
    // the site-pair candidate runs on the site-pair layout (swapped back below)
    const bool pl = cands[i].path == 3;
    cudaError_t e = cudaSuccess;
    if (pl) e = c->ks->pair_swap(lc, cur_u(c));
    if (pl && e == cudaSuccess) e = c->ks->pair_swap(lc, c->P2);
    if (e == cudaSuccess) e = fused(lc);
    if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = fused(lc);
    if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (pl && e == cudaSuccess) e = c->ks->pair_swap(lc, cur_u(c));
    if (pl && e == cudaSuccess) e = c->ks->pair_swap(lc, c->P2);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return set_err(c, ASKJA_ERR_CUDA, "autotune candidate %zu: %s", i, cudaGetErrorString(e));
    }
    const double us = 1e3 * ms / reps;
    res.cand_path[i] = cands[i].path;
    res.cand_groups[i] = cands[i].groups;
    res.cand_occ[i] = cands[i].occ;
    res.cand_us[i] = us;
    if (us < res.best_us) {
      res.best_us = us;
      best = (int)i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  res.ncand = (int)cands.size();
  res.path = cands[best].path;
  res.groups = cands[best].groups;
  res.occupancy = cands[best].occ;
  if (int rc = askja_set_tuning(c, &res)) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[std::make_tuple(c->N, c->D, c->p.precision)] = res;
  }
  if (out) *out = res;
  return ASKJA_OK;
}

int askja_set_reduction_range(askja_ctx* c, long s0, long s1) {
  if (int rc = check_ctx(c)) return rc;
  if (s0 < 0 || s1 <= s0 || s1 > c->V)
    return set_err(c, ASKJA_ERR_ARG, "reduction range [%ld, %ld) outside [0, %ld)", s0, s1, c->V);
  c->lat.r0 = (int)s0;
  c->lat.r1 = (int)s1;
  c->lc.lat.r0 = c->lat.r0;
  c->lc.lat.r1 = c->lat.r1;
  drop_graphs(c);  // the captured launches hold the geometry by value
  return ASKJA_OK;
}

int askja_slab(askja_ctx* c, long s0, long nsites, double* buf, int to_buf) {
  if (int rc = check_ctx(c)) return rc;
  if (!buf || s0 < 0 || nsites < 1 || s0 + nsites > c->V) return set_err(c, ASKJA_ERR_ARG, "bad slab");
  Range range("askja_slab");
  DevGuard g(c->p.device);
  const size_t bytes = (size_t)nsites * c->D * c->N * c->N * 2 * sizeof(double);
  const bool fp64 = c->p.precision == ASKJA_FP64;
  void* lo = c->split ? cur_ul(c) : nullptr;
  if (to_buf) {
    KL(askja::splitk::slab(c->lc, fp64, cur_u(c), lo, s0, nsites, c->staging, true), "slab");
    CK(cudaMemcpyAsync(buf, c->staging, bytes, cudaMemcpyDefault, c->stream));
  } else {
    CK(cudaMemcpyAsync(c->staging, buf, bytes, cudaMemcpyDefault, c->stream));
    KL(askja::splitk::slab(c->lc, fp64, cur_u(c), lo, s0, nsites, c->staging, false), "slab");
  }
  CK(cudaStreamSynchronize(c->stream));
  return ASKJA_OK;
}

int askja_tc_wait_selftest(askja_ctx* c, long long cycles) {
  if (int rc = check_ctx(c)) return rc;
  if (c->lc.force_rows != 2) return set_err(c, ASKJA_ERR_ARG, "the bounded-wait self-test needs the tensor-core path");
  if (cycles < 0) return set_err(c, ASKJA_ERR_ARG, "cycles must be >= 0");
  DevGuard g(c->p.device);
  KL(c->ks->wait_probe(c->lc, cycles), "bounded-wait self-test");
  return ASKJA_OK;
}

void* askja_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}

void askja_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

}  // extern "C"
