// Bench-only helper library (libaskja_peak.so, not part of the askja ABI):
// compute-pipe peaks measured on the running GPU, for the compute side of the
// roofline (the HBM and tensor peaks come from the pool's measured copy and
// cuBLAS figures).  Each kernel runs long chains of independent fused
// multiply-adds from registers: FP32 FFMA, FP32 packed FFMA2 (two lanes per
// instruction, sm_100), FP64 DFMA.  No memory traffic except one store per
// thread to keep the chains alive.
#include <cuda_runtime.h>

// status codes: 0 success, -1 bad argument, -2 a CUDA call failed
constexpr int kOk = 0, kErrArg = -1, kErrCuda = -2;


namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void k_ffma(float* out, float a, float b) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = threadIdx.x * 1e-3f + c;
  for (int i = 0; i < kIters; i++)
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = fmaf(x[c], a, b);
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_ffma2(float* out, float a, float b) {
  float2 x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = make_float2(threadIdx.x * 1e-3f + c, c);
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
  for (int i = 0; i < kIters; i++)
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = __ffma2_rn(x[c], a2, b2);
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c].x + x[c].y;
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_dfma(double* out, double a, double b) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = threadIdx.x * 1e-3 + c;
  for (int i = 0; i < kIters; i++)
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = fma(x[c], a, b);
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// which: 0 = FFMA, 1 = FFMA2, 2 = DFMA.  Returns GFLOP/s (2 flops per FMA
// lane) in *gflops, best of `repeats` timed launches.
extern "C" __attribute__((visibility("default"))) int askja_peak_flops(int device, int which, int repeats, double* gflops) {
  if (!gflops || which < 0 || which > 2 || repeats < 1) return kErrArg;
  if (cudaSetDevice(device) != cudaSuccess) return kErrCuda;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * 8;
  void* out = nullptr;
  if (cudaMalloc(&out, (size_t)threads * blocks * sizeof(double)) != cudaSuccess) return kErrCuda;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r < repeats + 1; r++) {
    cudaEventRecord(e0);
    if (which == 0) k_ffma<<<blocks, threads>>>((float*)out, 0.999f, 1e-4f);
    if (which == 1) k_ffma2<<<blocks, threads>>>((float*)out, 0.999f, 1e-4f);
    if (which == 2) k_dfma<<<blocks, threads>>>((double*)out, 0.999, 1e-4);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;  // first launch is warm-up
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return kErrCuda;
  const double lanes = which == 1 ? 2.0 : 1.0;
  const double fmas = (double)threads * blocks * kIters * kChains * lanes;
  *gflops = 2.0 * fmas / (best * 1e-3) / 1e9;
  return kOk;
}
