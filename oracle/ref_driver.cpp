// ref_driver.cpp — TEST INFRASTRUCTURE ONLY. The reference's own
// clue::Clusterer<Ndim>::make_clusters, compiled from CLUEstering's unmodified
// headers on its serial CPU backend (against the alpaka stand-in in
// oracle/alpaka_shim), behind a small C ABI that the tests call through ctypes.
// oracle/Makefile builds it into oracle/_ref/ when the reference tree is
// present; the product never loads it.
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

#include "CLUEstering/CLUEstering.hpp"

namespace {

std::string g_error;

}  // namespace

extern "C" {

struct ref_params {
  float dc, rhoc, dm, seed_dc;
  int32_t kernel_kind;  // 0 flat, 1 exponential, 2 gaussian (the library's numbering)
  float kernel_params[2];
  int32_t metric_kind;  // 0 Euclidean, 1 weighted Euclidean, 2 periodic, 3 Manhattan, 4 Chebyshev,
                        // 5 weighted Chebyshev, 6 Mahalanobis
  float metric_params[10];
  uint8_t wrapped[10];
};

const char* ref_last_error() { return g_error.c_str(); }

}  // extern "C"

namespace {

template <std::size_t D, typename Fn>
void with_metric(const ref_params& p, Fn&& fn) {
  std::array<float, D> mp{};
  for (std::size_t d = 0; d < D; ++d)
    mp[d] = p.metric_params[d];
  switch (p.metric_kind) {
    case 1:
      fn(clue::WeightedEuclideanMetric<D, float>(mp));
      break;
    case 2:
      fn(clue::PeriodicEuclideanMetric<D, float>(mp));
      break;
    case 3:
      fn(clue::ManhattanMetric<D, float>{});
      break;
    case 4:
      fn(clue::ChebyshevMetric<D, float>{});
      break;
    case 5:
      fn(clue::WeightedChebyshevMetric<D, float>(mp));
      break;
    case 6:
      fn(clue::MahalanobisMetric<D, float>{});
      break;
    default:
      fn(clue::EuclideanMetric<D, float>{});
      break;
  }
}

template <typename Fn>
void with_kernel(const ref_params& p, Fn&& fn) {
  switch (p.kernel_kind) {
    case 1:
      fn(clue::ExponentialKernel<float>(p.kernel_params[0], p.kernel_params[1]));
      break;
    case 2:
      fn(clue::GaussianKernel<float>(p.kernel_params[0], p.kernel_params[1]));
      break;
    default:
      fn(clue::FlatKernel<float>(p.kernel_params[0]));
      break;
  }
}

template <std::size_t D>
int run(int32_t n, const float* coords, const float* weights, const ref_params& p, const float* sigma,
        const float* unc, const uint32_t* tags, const uint32_t* sizes, int32_t n_events,
        int32_t* cluster_index, int32_t* is_seed, float* rho, int32_t* nh) {
  clue::Queue queue(clue::get_device(0u));
  std::vector<float> c(coords, coords + (std::size_t)D * n), w(weights, weights + n);
  std::vector<int> out(n);
  clue::PointsHost<D> h(queue, n, c.data(), w.data(), out.data());
  std::vector<std::vector<float>> sig;
  if (sigma)
    for (std::size_t d = 0; d < D; ++d) {
      sig.emplace_back(sigma + d * n, sigma + (d + 1) * n);
      h.set_sigma(d, std::span<float>(sig.back().data(), n));
    }
  std::vector<float> u;
  if (unc) {
    u.assign(unc, unc + n);
    h.set_density_uncertainty(std::span<float>(u.data(), n));
  }
  std::vector<uint32_t> tg;
  if (tags) {
    tg.assign(tags, tags + n);
    h.set_tags(std::span<uint32_t>(tg.data(), n));
  }
  clue::PointsDevice<D> dev(queue, n);
  clue::Clusterer<D> algo(queue, p.dc, p.rhoc, p.dm, p.seed_dc);
  std::array<uint8_t, D> wr{};
  for (std::size_t d = 0; d < D; ++d)
    wr[d] = p.wrapped[d];
  algo.setWrappedCoordinates(wr);
  with_metric<D>(p, [&](const auto& metric) {
    with_kernel(p, [&](const auto& kernel) {
      if (sizes)
        algo.make_clusters(queue, h, dev, std::span<const uint32_t>(sizes, (std::size_t)n_events), metric,
                           kernel);
      else
        algo.make_clusters(queue, h, dev, metric, kernel);
    });
  });
  const auto& v = dev.view();
  std::memcpy(cluster_index, out.data(), sizeof(int32_t) * n);
  if (is_seed)
    std::memcpy(is_seed, v.m_is_seed, sizeof(int32_t) * n);
  if (rho)
    std::memcpy(rho, v.m_rho, sizeof(float) * n);
  if (nh)
    std::memcpy(nh, v.m_nearest_higher, sizeof(int32_t) * n);
  return 0;
}

}  // namespace

extern "C" {

// Clusters n points in ndim dimensions (coords: ndim planes of n floats) with
// the reference's make_clusters; event_sizes (n_events entries) selects its
// batched form. sigma (ndim planes), unc and tags may be null; is_seed, rho and
// nh may be null. Returns 0, or 1 with ref_last_error() set.
int ref_make_clusters(int32_t ndim, int32_t n, const float* coords, const float* weights,
                      const ref_params* p, const float* sigma, const float* unc, const uint32_t* tags,
                      const uint32_t* event_sizes, int32_t n_events, int32_t* cluster_index,
                      int32_t* is_seed, float* rho, int32_t* nh) {
  try {
    switch (ndim) {
#define CLUE_REF_CASE(D)                                                                              \
  case D:                                                                                             \
    return run<D>(n, coords, weights, *p, sigma, unc, tags, event_sizes, n_events, cluster_index,    \
                  is_seed, rho, nh);
      CLUE_REF_CASE(1)
      CLUE_REF_CASE(2)
      CLUE_REF_CASE(3)
      CLUE_REF_CASE(4)
#undef CLUE_REF_CASE
      default:
        g_error = "ndim outside 1..4";
        return 1;
    }
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

}  // extern "C"
