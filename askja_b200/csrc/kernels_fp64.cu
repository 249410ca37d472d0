// FP64 kernel table: the plain double-precision path (the reference's own
// arithmetic, used for parity against the oracle).
#include "kernels.cuh"

namespace askja {

const KernelSet kernels_fp64 = detail::make_set<double>();

size_t partial_doubles(const Lat& L) {
  const long nl = (long)L.V * L.D;
  const size_t plaq = 2 * ((L.V + misc::RED_THREADS - 1) / misc::RED_THREADS);
  const size_t links = 3 * ((nl + misc::RED_THREADS - 1) / misc::RED_THREADS);
  const size_t gauss =
      2 * (size_t)L.N * L.N * ((nl + detail::GAUSS_LINKS_PER_BLOCK - 1) / detail::GAUSS_LINKS_PER_BLOCK);
  // one partial per site / per link for the large-NC reductions
  const size_t big = L.N >= misc::BIG_NC ? std::max(2 * (size_t)L.V, 3 * (size_t)nl) : 0;
  const size_t fourier = 2 * (size_t)L.n[0];  // FourierTrafo: one plaquette partial per site 0..N0-1
  return std::max(std::max(std::max(plaq, big), std::max(links, gauss)), fourier) + 64;
}

int rows_effective_groups(int N, bool fp64, int want) {
  int G;
  size_t smem;
  if (fp64)
    detail::Rows<double>::shape(N, &G, &smem, want);
  else
    detail::Rows<float>::shape(N, &G, &smem, want);
  return G;
}

}  // namespace askja
