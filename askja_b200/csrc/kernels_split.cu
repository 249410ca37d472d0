// Host launchers of the residual-plane FP32 kernels (split.cuh), NC = 2..4.
#include "split.h"
#include "split.cuh"

namespace askja {
namespace splitk {

namespace {

constexpr int THREADS = 128;

inline long nlinks(const Lat& L) { return (long)L.V * L.D; }
inline unsigned blocks_for(long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <typename F>
cudaError_t by_nc(int N, F&& f) {
  switch (N) {
    case 2:
      return f(std::integral_constant<int, 2>{});
    case 3:
      return f(std::integral_constant<int, 3>{});
    case 4:
      return f(std::integral_constant<int, 4>{});
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace

bool supported(int N) { return N >= 2 && N <= 4; }

size_t coef_floats(const Lat& L) {
  const int nc = L.N * L.N - 1;
  return (size_t)L.D * L.B * 32 * nc;
}

size_t coef_words(const Lat& L) {
  const int nc = L.N * L.N - 1;
  return (size_t)L.D * L.B * 32 * ((nc + 1) / 2);
}

cudaError_t force(const LaunchCtx& c, int mode, const void* U, const void* UL, const void* Pin, const void* PLin,
                  void* Pout, void* PLout, void* Uout, void* ULout, double ek, double ed) {
  const unsigned grid = blocks_for(c.lat.V, 32);
  const int threads = 32 * std::min(c.lat.D, 4);
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    auto launch = [&](auto kern) {
      kern<<<grid, threads, 0, c.stream>>>(c.lat, (const float2*)U, (const uint32_t*)UL, (const float*)Pin,
                                           (const uint32_t*)PLin, (float*)Pout, (uint32_t*)PLout, (float2*)Uout,
                                           (uint32_t*)ULout, (float)ek, (float)ed, c.order);
      return cudaGetLastError();
    };
    if (mode == 0) {
      if (c.small_occ == 2) return launch(split::k_force<N, 0, 2>);
      if (c.small_occ == 1) return launch(split::k_force<N, 0, 1>);
      return launch(split::k_force<N, 0, 0>);
    }
    if (c.small_occ == 2) return launch(split::k_force<N, 1, 2>);
    if (c.small_occ == 1) return launch(split::k_force<N, 1, 1>);
    return launch(split::k_force<N, 1, 0>);
  });
}

cudaError_t drift(const LaunchCtx& c, void* U, void* UL, const void* P, const void* PL, double eps) {
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_drift<N><<<blocks_for(nlinks(c.lat), THREADS), THREADS, 0, c.stream>>>(
        c.lat, (float2*)U, (uint32_t*)UL, (const float*)P, (const uint32_t*)PL, (float)eps, c.order);
    return cudaGetLastError();
  });
}

cudaError_t reunit(const LaunchCtx& c, void* U, void* UL, void* Usave, void* ULsave) {
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_reunit<N><<<blocks_for(nlinks(c.lat), THREADS), THREADS, 0, c.stream>>>(
        c.lat, (float2*)U, (uint32_t*)UL, (float2*)Usave, (uint32_t*)ULsave);
    return cudaGetLastError();
  });
}

cudaError_t plaq(const LaunchCtx& c, const void* U, const void* UL, double* partial, double* out) {
  const unsigned nb = blocks_for(c.lat.V, misc::RED_THREADS);
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_plaq<N><<<nb, misc::RED_THREADS, 0, c.stream>>>(c.lat, (const float2*)U, (const uint32_t*)UL, partial);
    misc::k_finish<2><<<1, misc::RED_THREADS, 0, c.stream>>>(partial, (int)nb, out);
    return cudaGetLastError();
  });
}

cudaError_t linksums(const LaunchCtx& c, const void* Pa, const void* PLa, const void* Pb, const void* PLb,
                     const void* U, const void* UL, double* partial, double* out) {
  const unsigned nb = blocks_for(nlinks(c.lat), misc::RED_THREADS);
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_linksums<N><<<nb, misc::RED_THREADS, 0, c.stream>>>(
        c.lat, (const float*)Pa, (const uint32_t*)PLa, (const float*)Pb, (const uint32_t*)PLb, (const float2*)U,
        (const uint32_t*)UL, partial);
    misc::k_finish<3><<<1, misc::RED_THREADS, 0, c.stream>>>(partial, (int)nb, out);
    return cudaGetLastError();
  });
}

cudaError_t refresh(const LaunchCtx& c, void* P, void* PL, uint64_t seed, const unsigned long long* traj_dev,
                    unsigned long long traj_host, double scale) {
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_refresh<N><<<blocks_for(nlinks(c.lat), THREADS), THREADS, 0, c.stream>>>(
        c.lat, (float*)P, (uint32_t*)PL, seed, traj_dev, traj_host, scale);
    return cudaGetLastError();
  });
}

cudaError_t links_from_conf(const LaunchCtx& c, const void* conf, void* U, void* UL) {
  const long tot = (long)field_elems(c.lat);
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_links_from_conf<N><<<blocks_for(tot, 256), 256, 0, c.stream>>>(c.lat, (const double2*)conf, (float2*)U,
                                                                           (uint32_t*)UL);
    return cudaGetLastError();
  });
}

cudaError_t links_to_conf(const LaunchCtx& c, const void* U, const void* UL, void* conf) {
  const long tot = nlinks(c.lat) * c.lat.N * c.lat.N;
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_links_to_conf<N><<<blocks_for(tot, 256), 256, 0, c.stream>>>(c.lat, (const float2*)U,
                                                                         (const uint32_t*)UL, (double2*)conf);
    return cudaGetLastError();
  });
}

cudaError_t momenta_from_conf(const LaunchCtx& c, const void* conf, void* P, void* PL) {
  const long tot = (long)c.lat.D * c.lat.B * 32;
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_momenta_from_conf<N><<<blocks_for(tot, THREADS), THREADS, 0, c.stream>>>(c.lat, (const double2*)conf,
                                                                                      (float*)P, (uint32_t*)PL);
    return cudaGetLastError();
  });
}

cudaError_t momenta_to_conf(const LaunchCtx& c, const void* P, const void* PL, void* conf) {
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_momenta_to_conf<N><<<blocks_for(nlinks(c.lat), THREADS), THREADS, 0, c.stream>>>(
        c.lat, (const float*)P, (const uint32_t*)PL, (double2*)conf);
    return cudaGetLastError();
  });
}

cudaError_t momenta_to_matrix(const LaunchCtx& c, const void* P, const void* PL, void* F) {
  const long tot = (long)c.lat.D * c.lat.B * 32;
  return by_nc(c.lat.N, [&](auto n) {
    constexpr int N = decltype(n)::value;
    split::k_momenta_to_matrix<N><<<blocks_for(tot, THREADS), THREADS, 0, c.stream>>>(
        c.lat, (const float*)P, (const uint32_t*)PL, (float2*)F);
    return cudaGetLastError();
  });
}

cudaError_t slab(const LaunchCtx& c, bool fp64, void* f, void* lo, long s0, long ns, void* buf, bool to_buf) {
  const long tot = ns * c.lat.D * c.lat.N * c.lat.N;
  const unsigned grid = blocks_for(tot, 256);
  if (fp64) {
    if (to_buf)
      split::k_slab_get<double2><<<grid, 256, 0, c.stream>>>(c.lat, (const double2*)f, nullptr, (int)s0, (int)ns,
                                                             (double2*)buf);
    else
      split::k_slab_set<double2><<<grid, 256, 0, c.stream>>>(c.lat, (double2*)f, nullptr, (int)s0, (int)ns,
                                                             (const double2*)buf);
  } else {
    if (to_buf)
      split::k_slab_get<float2><<<grid, 256, 0, c.stream>>>(c.lat, (const float2*)f, (const uint32_t*)lo, (int)s0,
                                                            (int)ns, (double2*)buf);
    else
      split::k_slab_set<float2><<<grid, 256, 0, c.stream>>>(c.lat, (float2*)f, (uint32_t*)lo, (int)s0, (int)ns,
                                                            (const double2*)buf);
  }
  return cudaGetLastError();
}

}  // namespace splitk
}  // namespace askja
