// Host interface of the residual-plane FP32 kernels (split.cuh, NC = 2..4):
// links as an FP32 field plus a bfloat16 residual plane (one uint32 per
// complex element, same index as the FP32 field), momenta as the N^2-1 real
// coordinates of the Hermitian traceless matrix in FP32 plus bfloat16
// residuals.  Every call enqueues on the context's stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include "launch.h"

namespace askja {
namespace splitk {

bool supported(int N);
// FP32 coordinates / residual words of one momentum field (padding included)
size_t coef_floats(const Lat& L);
size_t coef_words(const Lat& L);

// mode 0: Pout = Pin - ek F(U);  mode 1: also U' = U + (exp(i ed Pout) - 1) U into (Uout, ULout)
cudaError_t force(const LaunchCtx& c, int mode, const void* U, const void* UL, const void* Pin, const void* PLin,
                  void* Pout, void* PLout, void* Uout, void* ULout, double ek, double ed);
// U <- U + (exp(i eps P) - 1) U in place
cudaError_t drift(const LaunchCtx& c, void* U, void* UL, const void* P, const void* PL, double eps);
// projection onto SU(N) in FP64, in place and (Usave non-null) also into (Usave, ULsave)
cudaError_t reunit(const LaunchCtx& c, void* U, void* UL, void* Usave = nullptr, void* ULsave = nullptr);
// out[0] temporal, out[1] spatial plaquette sums
cudaError_t plaq(const LaunchCtx& c, const void* U, const void* UL, double* partial, double* out);
// out[0] sum tr(Pa^2), out[1] sum tr((Pa+Pb)^2)/4, out[2] sum ReTr((UU^dag-1)^2) (null arguments: skipped)
cudaError_t linksums(const LaunchCtx& c, const void* Pa, const void* PLa, const void* Pb, const void* PLb,
                     const void* U, const void* UL, double* partial, double* out);
cudaError_t refresh(const LaunchCtx& c, void* P, void* PL, uint64_t seed, const unsigned long long* traj_dev,
                    unsigned long long traj_host, double scale);
cudaError_t links_from_conf(const LaunchCtx& c, const void* conf, void* U, void* UL);
cudaError_t links_to_conf(const LaunchCtx& c, const void* U, const void* UL, void* conf);
cudaError_t momenta_from_conf(const LaunchCtx& c, const void* conf, void* P, void* PL);
cudaError_t momenta_to_conf(const LaunchCtx& c, const void* P, const void* PL, void* conf);
// links of the sites [s0, s0 + ns) to (to_buf) or from device memory buf in the
// U-conf order (FP64); any storage: FP64 (fp64), FP32 with (lo non-null) or
// without residual plane
cudaError_t slab(const LaunchCtx& c, bool fp64, void* f, void* lo, long s0, long ns, void* buf, bool to_buf);
// full FP32 matrices in the float2 field layout (for the matrix diagnostics)
cudaError_t momenta_to_matrix(const LaunchCtx& c, const void* P, const void* PL, void* F);

}  // namespace splitk
}  // namespace askja
