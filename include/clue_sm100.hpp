// clue_sm100.hpp — C++20 API of libclue_sm100.so with the names and behaviour of
// CLUEstering's clustering interface (namespace clue): Clusterer, PointsHost,
// PointsDevice, the convolutional kernels, the distance metrics,
// copyToDevice/copyToHost, get_queue/get_device and the association maps
// returned by getClusters/getSampleAssociations.
//
// Everything here is a thin inline layer over the C ABI in clue_sm100.h; no
// CUDA header is needed to use it. Coordinates and weights are float32 (the
// reference also instantiates double; this library computes in float only).
// Errors surface as the reference's exception types: std::invalid_argument,
// std::out_of_range and std::runtime_error.
#pragma once

#include <algorithm>
#include <array>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <optional>
#include <ranges>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "clue_sm100.h"

namespace clue {

namespace detail {

inline void check(clue_status s) {
  if (s == CLUE_OK)
    return;
  std::string msg = clue_last_error();
  if (msg.empty())
    msg = clue_status_string(s);
  switch (s) {
    case CLUE_ERR_INVALID_ARGUMENT:
      throw std::invalid_argument(msg);
    case CLUE_ERR_OUT_OF_RANGE:
      throw std::out_of_range(msg);
    default:
      throw std::runtime_error(msg);
  }
}

}  // namespace detail

// ---------------------------------------------------------------------------
// Devices and queues (utils/get_queue.hpp, utils/get_device.hpp)
// ---------------------------------------------------------------------------

struct Device {
  int32_t index = 0;
};

inline Device get_device(uint32_t index) { return Device{static_cast<int32_t>(index)}; }

// A CUDA stream on one device. Owns the stream it creates; wraps (without
// owning) a stream passed in from outside.
class Queue {
 public:
  explicit Queue(Device dev = {}) : device_{dev.index}, owned_{true} {
    detail::check(clue_stream_create(&stream_, device_));
  }
  Queue(void* cuda_stream, int32_t device) : stream_{cuda_stream}, device_{device}, owned_{false} {}
  Queue(const Queue&) = delete;
  Queue& operator=(const Queue&) = delete;
  Queue(Queue&& o) noexcept : stream_{o.stream_}, device_{o.device_}, owned_{o.owned_} { o.owned_ = false; }
  ~Queue() {
    if (owned_ && stream_)
      clue_stream_destroy(stream_);
  }
  void* stream() const { return stream_; }
  int32_t device() const { return device_; }
  void wait() const { detail::check(clue_stream_synchronize(stream_)); }

 private:
  void* stream_ = nullptr;
  int32_t device_ = 0;
  bool owned_ = false;
};

inline Queue get_queue(uint32_t device = 0) { return Queue(get_device(device)); }
// get_queue(cudaStream_t&): pass the stream as void*.
inline Queue get_queue(void* cuda_stream, int32_t device = 0) { return Queue(cuda_stream, device); }
inline void wait(const Queue& q) { q.wait(); }

// ---------------------------------------------------------------------------
// Convolutional kernels (core/ConvolutionalKernel.hpp)
// ---------------------------------------------------------------------------

template <typename TData = float>
class FlatKernel {
 public:
  using value_type = float;
  FlatKernel(value_type flat) : flat_{flat} {
    if (!(flat > 0))
      throw std::invalid_argument("Flat kernel parameter must be positive.");
  }
  void fill(clue_params& p) const {
    p.kernel_kind = CLUE_KERNEL_FLAT;
    p.kernel_params[0] = flat_;
    p.kernel_params[1] = 0.f;
  }

 private:
  value_type flat_;
};

template <typename TData = float>
class GaussianKernel {
 public:
  using value_type = float;
  GaussianKernel(value_type gaus_std, value_type gaus_amplitude) : std_{gaus_std}, amp_{gaus_amplitude} {
    if (!(gaus_std > 0) || !(gaus_amplitude > 0))
      throw std::invalid_argument("Gaussian kernel parameters must be positive.");
  }
  void fill(clue_params& p) const {
    p.kernel_kind = CLUE_KERNEL_GAUSSIAN;
    p.kernel_params[0] = std_;
    p.kernel_params[1] = amp_;
  }

 private:
  value_type std_, amp_;
};

template <typename TData = float>
class ExponentialKernel {
 public:
  using value_type = float;
  ExponentialKernel(value_type exp_avg, value_type exp_amplitude) : avg_{exp_avg}, amp_{exp_amplitude} {
    if (!(exp_avg > 0) || !(exp_amplitude > 0))
      throw std::invalid_argument("Exponential kernel parameters must be positive.");
  }
  void fill(clue_params& p) const {
    p.kernel_kind = CLUE_KERNEL_EXPONENTIAL;
    p.kernel_params[0] = avg_;
    p.kernel_params[1] = amp_;
  }

 private:
  value_type avg_, amp_;
};

// ---------------------------------------------------------------------------
// Distance metrics (core/DistanceMetrics.hpp)
// ---------------------------------------------------------------------------

template <std::size_t Ndim, int Kind>
class MetricBase {
 public:
  using value_type = float;
  void fill(clue_params& p) const {
    p.metric_kind = Kind;
    for (std::size_t d = 0; d < Ndim; ++d)
      p.metric_params[d] = params_[d];
  }

 protected:
  std::array<float, Ndim> params_{};
};

template <std::size_t Ndim, typename TData = float>
class EuclideanMetric : public MetricBase<Ndim, CLUE_METRIC_EUCLIDEAN> {};

template <std::size_t Ndim, typename TData = float>
class ManhattanMetric : public MetricBase<Ndim, CLUE_METRIC_MANHATTAN> {};

template <std::size_t Ndim, typename TData = float>
class ChebyshevMetric : public MetricBase<Ndim, CLUE_METRIC_CHEBYSHEV> {};

template <std::size_t Ndim, typename TData = float>
class MahalanobisMetric : public MetricBase<Ndim, CLUE_METRIC_MAHALANOBIS> {};

#define CLUE_PARAM_METRIC(Name, Kind)                                                   \
  template <std::size_t Ndim, typename TData = float>                                   \
  class Name : public MetricBase<Ndim, Kind> {                                          \
   public:                                                                              \
    Name(const std::array<float, Ndim>& v) { this->params_ = v; }                       \
    template <typename... T>                                                            \
      requires(sizeof...(T) == Ndim && (std::is_floating_point_v<T> && ...))            \
    Name(T... v) {                                                                      \
      this->params_ = {static_cast<float>(v)...};                                       \
    }                                                                                   \
  };
CLUE_PARAM_METRIC(WeightedEuclideanMetric, CLUE_METRIC_WEIGHTED_EUCLIDEAN)
CLUE_PARAM_METRIC(PeriodicEuclideanMetric, CLUE_METRIC_PERIODIC_EUCLIDEAN)
CLUE_PARAM_METRIC(WeightedChebyshevMetric, CLUE_METRIC_WEIGHTED_CHEBYSHEV)
#undef CLUE_PARAM_METRIC

template <typename T, std::size_t N>
PeriodicEuclideanMetric(std::array<T, N>) -> PeriodicEuclideanMetric<N, T>;
template <typename T, std::size_t N>
WeightedEuclideanMetric(std::array<T, N>) -> WeightedEuclideanMetric<N, T>;
template <typename T, std::size_t N>
WeightedChebyshevMetric(std::array<T, N>) -> WeightedChebyshevMetric<N, T>;

namespace metrics {
template <std::size_t Ndim, typename TData = float>
using Euclidean = EuclideanMetric<Ndim, TData>;
template <std::size_t Ndim, typename TData = float>
using WeightedEuclidean = WeightedEuclideanMetric<Ndim, TData>;
template <std::size_t Ndim, typename TData = float>
using PeriodicEuclidean = PeriodicEuclideanMetric<Ndim, TData>;
template <std::size_t Ndim, typename TData = float>
using Manhattan = ManhattanMetric<Ndim, TData>;
template <std::size_t Ndim, typename TData = float>
using Chebyshev = ChebyshevMetric<Ndim, TData>;
template <std::size_t Ndim, typename TData = float>
using WeightedChebyshev = WeightedChebyshevMetric<Ndim, TData>;
template <std::size_t Ndim, typename TData = float>
using Mahalanobis = MahalanobisMetric<Ndim, TData>;
}  // namespace metrics

// ---------------------------------------------------------------------------
// Association maps (data_structures/AssociationMap.hpp): key -> values CSR
// ---------------------------------------------------------------------------

class AssociationMapHost {
 public:
  using key_type = int32_t;
  using mapped_type = int32_t;
  using iterator = const mapped_type*;

  AssociationMapHost() = default;
  AssociationMapHost(std::vector<int32_t> offsets, std::vector<int32_t> values)
      : offsets_{std::move(offsets)}, values_{std::move(values)} {
    if (offsets_.empty())
      offsets_.push_back(0);
  }
  // Counting sort of values 0..n-1 by their key (negative keys are dropped);
  // values of one key stay ascending. Sized by the largest key + 1
  // (data_structures/internal/MakeAssociator.hpp:32-43).
  static AssociationMapHost from_keys(std::span<const int32_t> keys) {
    int32_t nkeys = 0;
    for (int32_t k : keys)
      nkeys = std::max(nkeys, k + 1);
    std::vector<int32_t> off(nkeys + 1, 0);
    for (int32_t k : keys)
      if (k >= 0)
        ++off[k + 1];
    std::partial_sum(off.begin(), off.end(), off.begin());
    std::vector<int32_t> vals(off.back());
    std::vector<int32_t> cur(off.begin(), off.end() - 1);
    for (int32_t i = 0; i < static_cast<int32_t>(keys.size()); ++i)
      if (keys[i] >= 0)
        vals[cur[keys[i]]++] = i;
    return AssociationMapHost(std::move(off), std::move(vals));
  }

  std::size_t size() const { return offsets_.size() - 1; }
  iterator begin() const { return values_.data(); }
  iterator end() const { return values_.data() + values_.size(); }
  std::span<const mapped_type> operator[](key_type key) const {
    if (key < 0 || static_cast<std::size_t>(key) >= size())
      throw std::out_of_range("key out of range in AssociationMap");
    return {values_.data() + offsets_[key], static_cast<std::size_t>(offsets_[key + 1] - offsets_[key])};
  }
  std::size_t count(key_type key) const { return (*this)[key].size(); }
  bool empty() const { return values_.empty(); }
  bool empty(key_type key) const { return count(key) == 0; }
  bool contains(key_type key) const { return key >= 0 && static_cast<std::size_t>(key) < size() && count(key) > 0; }
  iterator lower_bound(key_type key) const { return values_.data() + offsets_[key]; }
  iterator upper_bound(key_type key) const { return values_.data() + offsets_[key + 1]; }
  std::pair<iterator, iterator> equal_range(key_type key) const { return {lower_bound(key), upper_bound(key)}; }
  const std::vector<int32_t>& offsets() const { return offsets_; }
  const std::vector<int32_t>& values() const { return values_; }

 private:
  std::vector<int32_t> offsets_{0};
  std::vector<int32_t> values_;
};

// ---------------------------------------------------------------------------
// Points (data_structures/PointsHost.hpp, PointsDevice.hpp)
// ---------------------------------------------------------------------------

template <std::size_t Ndim, typename TData = float>
class PointsHost {
  static_assert(std::is_same_v<std::remove_cv_t<TData>, float>, "libclue_sm100 computes in float32");
  static_assert(Ndim >= 1 && Ndim <= CLUE_MAX_DIM, "Ndim must be in [1, 10]");

 public:
  using element_type = TData;
  using value_type = float;

  class Point {
   public:
    Point(const std::array<float, Ndim>& c, float w, int id) : c_{c}, w_{w}, id_{id} {}
    float operator[](std::size_t dim) const { return c_[dim]; }
    float weight() const { return w_; }
    int cluster_index() const { return id_; }

   private:
    std::array<float, Ndim> c_;
    float w_;
    int id_;
  };

  template <typename Q>
  PointsHost(Q&, int32_t n) : n_{n} {
    check_size();
    owned_.resize(static_cast<std::size_t>(n) * (Ndim + 1));
    owned_ids_.resize(n);
    bind(owned_.data(), owned_.data() + Ndim * n, owned_ids_.data());
  }
  template <typename Q>
  PointsHost(Q&, int32_t n, std::span<std::byte> buffer) : n_{n} {
    check_size();
    auto* f = reinterpret_cast<element_type*>(buffer.data());
    bind(f, f + Ndim * n, reinterpret_cast<int*>(f + (Ndim + 1) * n));
  }
  template <typename Q>
  PointsHost(Q&, int32_t n, element_type* input, int* output) : n_{n} {
    check_size();
    bind(input, input + Ndim * n, output);
  }
  template <typename Q>
  PointsHost(Q&, int32_t n, std::span<element_type> input, std::span<int> output) : n_{n} {
    check_size();
    bind(input.data(), input.data() + Ndim * n, output.data());
  }
  template <typename Q>
  PointsHost(Q&, int32_t n, element_type* coords, element_type* weights, int* output) : n_{n} {
    check_size();
    bind(coords, weights, output);
  }
  template <typename Q>
  PointsHost(Q&, int32_t n, std::span<element_type> coords, std::span<element_type> weights,
             std::span<int> output)
      : n_{n} {
    check_size();
    bind(coords.data(), weights.data(), output.data());
  }
  // One buffer per coordinate, then weights and cluster ids (Ndim + 2 pointers).
  template <typename Q, typename... P>
    requires(sizeof...(P) == Ndim + 2 && Ndim > 1 && (std::is_pointer_v<P> && ...))
  PointsHost(Q&, int32_t n, P... ptrs) : n_{n} {
    check_size();
    void* all[] = {const_cast<void*>(static_cast<const void*>(ptrs))...};
    for (std::size_t d = 0; d < Ndim; ++d)
      coords_[d] = static_cast<element_type*>(all[d]);
    weight_ = static_cast<element_type*>(all[Ndim]);
    ids_ = static_cast<int*>(all[Ndim + 1]);
  }
  PointsHost(const PointsHost&) = delete;
  PointsHost& operator=(const PointsHost&) = delete;
  PointsHost(PointsHost&&) = default;
  PointsHost& operator=(PointsHost&&) = default;

  int32_t size() const { return n_; }
  std::span<element_type> coords(std::size_t dim) const {
    if (dim >= Ndim)
      throw std::out_of_range("Dimension out of range in call to coords.");
    return {coords_[dim], static_cast<std::size_t>(n_)};
  }
  std::span<element_type> weights() const { return {weight_, static_cast<std::size_t>(n_)}; }
  std::span<const int> clusterIndexes() const { return {ids_, static_cast<std::size_t>(n_)}; }
  std::span<int> clusterIndexes() { return {ids_, static_cast<std::size_t>(n_)}; }
  bool clustered() const { return clustered_; }
  Point operator[](std::size_t i) const {
    if (i >= static_cast<std::size_t>(n_))
      throw std::out_of_range("Index out of range in PointsHost::operator[]");
    std::array<float, Ndim> c;
    for (std::size_t d = 0; d < Ndim; ++d)
      c[d] = coords_[d][i];
    return Point(c, weight_[i], ids_[i]);
  }
  // detail::compute_nclusters: largest id + 1.
  std::size_t n_clusters() const {
    int32_t m = -1;
    for (int32_t i = 0; i < n_; ++i)
      m = std::max(m, ids_[i]);
    return static_cast<std::size_t>(m + 1);
  }
  const AssociationMapHost& clusters() {
    if (!clusters_)
      clusters_ = AssociationMapHost::from_keys(clusterIndexes());
    return *clusters_;
  }
  std::vector<std::size_t> cluster_sizes() {
    const auto& c = clusters();
    std::vector<std::size_t> s(c.size());
    for (std::size_t k = 0; k < s.size(); ++k)
      s[k] = c.count(static_cast<int32_t>(k));
    return s;
  }
  void set_density_uncertainty(std::span<element_type> u) {
    if (u.size() != static_cast<std::size_t>(n_))
      throw std::invalid_argument("Size of density_uncertainty does not match the number of points");
    unc_ = u.data();
  }
  void set_sigma(std::size_t dim, std::span<element_type> s) {
    if (dim >= Ndim)
      throw std::out_of_range("Dimension out of range in set_sigma");
    if (s.size() != static_cast<std::size_t>(n_))
      throw std::invalid_argument("Size of sigma does not match the number of points");
    sigma_[dim] = s.data();
  }
  void set_tags(std::span<std::uint32_t> t) {
    if (t.size() != static_cast<std::size_t>(n_))
      throw std::invalid_argument("Size of tags does not match the number of points");
    tags_ = t.data();
  }

  // C ABI view of the points (host pointers).
  clue_points abi() const {
    clue_points p{};
    p.ndim = static_cast<int32_t>(Ndim);
    p.n = n_;
    for (std::size_t d = 0; d < Ndim; ++d) {
      p.coords[d] = coords_[d];
      p.sigma[d] = sigma_[d];
    }
    p.weight = weight_;
    p.density_uncertainty = unc_;
    p.tags = tags_;
    p.cluster_index = ids_;
    return p;
  }
  void mark_clustered() {
    clustered_ = true;
    clusters_.reset();
  }

 private:
  void check_size() const {
    if (n_ <= 0)
      throw std::invalid_argument("Number of points passed to PointsHost constructor must be positive.");
  }
  void bind(element_type* c, element_type* w, int* ids) {
    for (std::size_t d = 0; d < Ndim; ++d)
      coords_[d] = c + d * static_cast<std::size_t>(n_);
    weight_ = w;
    ids_ = ids;
  }

  int32_t n_;
  std::vector<float> owned_;
  std::vector<int> owned_ids_;
  std::array<element_type*, Ndim> coords_{};
  element_type* weight_ = nullptr;
  int* ids_ = nullptr;
  std::array<const float*, Ndim> sigma_{};
  const float* unc_ = nullptr;
  const uint32_t* tags_ = nullptr;
  bool clustered_ = false;
  std::optional<AssociationMapHost> clusters_;
};

template <std::size_t Ndim, typename TData = float>
using ConstPointsHost = PointsHost<Ndim, std::add_const_t<TData>>;

// Points in device memory. Owns its device buffers (allocated on the queue's
// device) unless constructed over caller buffers; keeps the internal outputs
// the reference's device points carry (is_seed, rho, nearest_higher).
template <std::size_t Ndim, typename TData = float>
class PointsDevice {
  static_assert(std::is_same_v<std::remove_cv_t<TData>, float>, "libclue_sm100 computes in float32");

 public:
  template <typename Q>
  PointsDevice(Q& q, int32_t n) : n_{n}, device_{q.device()} {
    check_size();
    coords_base_ = alloc<float>(static_cast<std::size_t>(n) * Ndim);
    for (std::size_t d = 0; d < Ndim; ++d)
      coords_[d] = coords_base_ + d * n;
    weight_ = alloc<float>(n);
    ids_ = alloc<int32_t>(n);
    alloc_internal();
  }
  template <typename Q>
  PointsDevice(Q& q, int32_t n, float* input, int* output) : n_{n}, device_{q.device()} {
    check_size();
    for (std::size_t d = 0; d < Ndim; ++d)
      coords_[d] = input + d * n;
    weight_ = input + Ndim * n;
    ids_ = output;
    alloc_internal();
  }
  template <typename Q>
  PointsDevice(Q& q, int32_t n, float* coords, float* weights, int* output) : n_{n}, device_{q.device()} {
    check_size();
    for (std::size_t d = 0; d < Ndim; ++d)
      coords_[d] = coords + d * n;
    weight_ = weights;
    ids_ = output;
    alloc_internal();
  }
  PointsDevice(const PointsDevice&) = delete;
  PointsDevice& operator=(const PointsDevice&) = delete;
  PointsDevice(PointsDevice&& o) noexcept { swap(o); }
  PointsDevice& operator=(PointsDevice&& o) noexcept {
    swap(o);
    return *this;
  }
  ~PointsDevice() {
    for (void* p : owned_)
      clue_device_free(p);
  }

  int32_t size() const { return n_; }
  float* coords(std::size_t dim) const {
    if (dim >= Ndim)
      throw std::out_of_range("Dimension out of range in call to coords.");
    return coords_[dim];
  }
  float* weights() const { return weight_; }
  int32_t* clusterIndexes() const { return ids_; }
  int32_t* is_seed() const { return seed_; }
  float* rho() const { return rho_; }
  int32_t* nearest_higher() const { return nh_; }
  bool clustered() const { return clustered_; }
  void mark_clustered() { clustered_ = true; }
  std::size_t n_clusters() const { return n_clusters_; }
  void set_n_clusters(std::size_t k) { n_clusters_ = k; }

  // Device spans (the reference takes std::span over device memory).
  void set_density_uncertainty(std::span<float> u) { unc_ = u.data(); }
  void set_sigma(std::size_t dim, std::span<float> s) {
    if (dim >= Ndim)
      throw std::out_of_range("Dimension out of range in set_sigma");
    sigma_[dim] = s.data();
  }
  void set_tags(std::span<std::uint32_t> t) { tags_ = t.data(); }

  clue_points abi() const {
    clue_points p{};
    p.ndim = static_cast<int32_t>(Ndim);
    p.n = n_;
    for (std::size_t d = 0; d < Ndim; ++d) {
      p.coords[d] = coords_[d];
      p.sigma[d] = sigma_[d];
    }
    p.weight = weight_;
    p.density_uncertainty = unc_;
    p.tags = tags_;
    p.cluster_index = ids_;
    p.is_seed = seed_;
    p.rho = rho_;
    p.nearest_higher = nh_;
    return p;
  }
  int32_t device() const { return device_; }
  // Device buffers the copies of host-side optional inputs go to.
  template <typename T>
  T* scratch(std::size_t count) { return alloc<T>(count); }

 private:
  template <typename T>
  T* alloc(std::size_t count) {
    void* p = nullptr;
    detail::check(clue_device_malloc(&p, std::max<std::size_t>(count, 1) * sizeof(T), device_));
    owned_.push_back(p);
    return static_cast<T*>(p);
  }
  void alloc_internal() {
    seed_ = alloc<int32_t>(n_);
    rho_ = alloc<float>(n_);
    nh_ = alloc<int32_t>(n_);
  }
  void check_size() const {
    if (n_ <= 0)
      throw std::invalid_argument("Number of points passed to PointsDevice constructor must be positive.");
  }
  void swap(PointsDevice& o) {
    std::swap(n_, o.n_);
    std::swap(device_, o.device_);
    std::swap(coords_base_, o.coords_base_);
    std::swap(coords_, o.coords_);
    std::swap(weight_, o.weight_);
    std::swap(ids_, o.ids_);
    std::swap(seed_, o.seed_);
    std::swap(rho_, o.rho_);
    std::swap(nh_, o.nh_);
    std::swap(sigma_, o.sigma_);
    std::swap(unc_, o.unc_);
    std::swap(tags_, o.tags_);
    std::swap(owned_, o.owned_);
    std::swap(clustered_, o.clustered_);
    std::swap(n_clusters_, o.n_clusters_);
  }

  int32_t n_ = 0;
  int32_t device_ = 0;
  float* coords_base_ = nullptr;
  std::array<float*, Ndim> coords_{};
  float* weight_ = nullptr;
  int32_t* ids_ = nullptr;
  int32_t* seed_ = nullptr;
  float* rho_ = nullptr;
  int32_t* nh_ = nullptr;
  std::array<const float*, Ndim> sigma_{};
  const float* unc_ = nullptr;
  const uint32_t* tags_ = nullptr;
  std::vector<void*> owned_;
  bool clustered_ = false;
  std::size_t n_clusters_ = 0;
};

template <std::size_t Ndim, typename TData = float>
using ConstPointsDevice = PointsDevice<Ndim, std::add_const_t<TData>>;

// data_structures/detail/PointsConversion.hpp:61-111: coordinates, weights and
// the optional per-point inputs to the device.
template <std::size_t Ndim, typename TH, typename TD>
void copyToDevice(Queue& q, PointsDevice<Ndim, TD>& d, const PointsHost<Ndim, TH>& h) {
  const clue_points hp = h.abi();
  const std::size_t n = static_cast<std::size_t>(h.size());
  for (std::size_t k = 0; k < Ndim; ++k)
    detail::check(clue_memcpy_async(d.coords(k), hp.coords[k], n * 4, 0, q.stream()));
  detail::check(clue_memcpy_async(d.weights(), hp.weight, n * 4, 0, q.stream()));
  for (std::size_t k = 0; k < Ndim; ++k)
    if (hp.sigma[k]) {
      float* s = d.template scratch<float>(n);
      detail::check(clue_memcpy_async(s, hp.sigma[k], n * 4, 0, q.stream()));
      d.set_sigma(k, std::span<float>(s, n));
    }
  if (hp.density_uncertainty) {
    float* u = d.template scratch<float>(n);
    detail::check(clue_memcpy_async(u, hp.density_uncertainty, n * 4, 0, q.stream()));
    d.set_density_uncertainty(std::span<float>(u, n));
  }
  if (hp.tags) {
    uint32_t* t = d.template scratch<uint32_t>(n);
    detail::check(clue_memcpy_async(t, hp.tags, n * 4, 0, q.stream()));
    d.set_tags(std::span<uint32_t>(t, n));
  }
  q.wait();
}

// data_structures/detail/PointsConversion.hpp:16-30: cluster ids back to the host.
template <std::size_t Ndim, typename TH, typename TD>
void copyToHost(Queue& q, PointsHost<Ndim, TH>& h, const PointsDevice<Ndim, TD>& d) {
  detail::check(clue_memcpy_async(h.clusterIndexes().data(), d.clusterIndexes(),
                                  static_cast<std::size_t>(h.size()) * 4, 1, q.stream()));
  q.wait();
  h.mark_clustered();
}

// ---------------------------------------------------------------------------
// Clusterer (core/Clusterer.hpp)
// ---------------------------------------------------------------------------

template <std::size_t Ndim, typename DataType = float>
class Clusterer {
  static_assert(std::is_same_v<DataType, float>, "libclue_sm100 computes in float32");

 public:
  using value_type = float;

  Clusterer(value_type density_radius, value_type min_density,
            std::optional<value_type> outlier_distance = std::nullopt,
            std::optional<value_type> seeding_distance = std::nullopt) {
    setParameters(density_radius, min_density, outlier_distance, seeding_distance);
  }
  Clusterer(Queue& q, value_type density_radius, value_type min_density,
            std::optional<value_type> outlier_distance = std::nullopt,
            std::optional<value_type> seeding_distance = std::nullopt)
      : device_{q.device()} {
    setParameters(density_radius, min_density, outlier_distance, seeding_distance);
  }
  Clusterer(const Clusterer&) = delete;
  Clusterer& operator=(const Clusterer&) = delete;
  ~Clusterer() {
    if (ws_)
      clue_workspace_destroy(ws_);
  }

  void setParameters(value_type density_radius, value_type min_density,
                     std::optional<value_type> outlier_distance = std::nullopt,
                     std::optional<value_type> seeding_distance = std::nullopt) {
    clue_params p = params_;
    p.dc = density_radius;
    p.rhoc = min_density;
    p.dm = outlier_distance.value_or(density_radius);
    p.seed_dc = seeding_distance.value_or(density_radius);
    p.kernel_kind = CLUE_KERNEL_FLAT;
    p.kernel_params[0] = 0.5f;
    detail::check(clue_validate_params(&p));
    params_ = p;
  }

  template <std::ranges::contiguous_range R>
    requires std::integral<std::ranges::range_value_t<R>>
  void setWrappedCoordinates(const R& wrapped) {
    std::size_t d = 0;
    for (auto v : wrapped) {
      if (d >= Ndim)
        break;
      params_.wrapped[d++] = static_cast<uint8_t>(v);
    }
  }
  template <std::integral... T>
  void setWrappedCoordinates(T... wrapped) {
    const uint8_t v[] = {static_cast<uint8_t>(wrapped)...};
    for (std::size_t d = 0; d < sizeof...(T) && d < Ndim; ++d)
      params_.wrapped[d] = v[d];
  }

  // make_clusters(Queue&, PointsHost&, metric, kernel): core/detail/Clusterer.hpp:90-105
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  void make_clusters(Queue& q, PointsHost<Ndim, TIn>& h, const Metric& metric = Metric{},
                     const Kernel& kernel = FlatKernel<>{.5f}) {
    const clue_params p = with(metric, kernel);
    const clue_points pts = h.abi();
    detail::check(clue_make_clusters_host(workspace(q.device()), &p, &pts, q.stream()));
    h.mark_clustered();
  }
  // make_clusters(PointsHost&, ...): a temporary queue on device 0 (:106-122)
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  void make_clusters(PointsHost<Ndim, TIn>& h, const Metric& metric = Metric{},
                     const Kernel& kernel = FlatKernel<>{.5f}) {
    Queue q(get_device(0));
    make_clusters(q, h, metric, kernel);
  }
  // make_clusters(Queue&, PointsHost&, PointsDevice&, ...): (:123-138)
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  void make_clusters(Queue& q, PointsHost<Ndim, TIn>& h, PointsDevice<Ndim, value_type>& d,
                     const Metric& metric = Metric{}, const Kernel& kernel = FlatKernel<>{.5f}) {
    copyToDevice(q, d, h);
    make_clusters(q, d, metric, kernel);
    copyToHost(q, h, d);
  }
  // make_clusters(Queue&, PointsDevice&, ...): (:139-151); returns synchronised
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  void make_clusters(Queue& q, PointsDevice<Ndim, TIn>& d, const Metric& metric = Metric{},
                     const Kernel& kernel = FlatKernel<>{.5f}) {
    const clue_params p = with(metric, kernel);
    const clue_points pts = d.abi();
    detail::check(clue_make_clusters_device(workspace(q.device()), &p, &pts, q.stream()));
    finish(q, d);
  }
  // Batched forms (:153-183). The reference builds one tile grid for the whole
  // batch; `grid_mode` CLUE_GRID_PER_EVENT gives each event its own grid.
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  void make_clusters(Queue& q, PointsHost<Ndim, TIn>& h, PointsDevice<Ndim, value_type>& d,
                     std::span<const uint32_t> batch_item_sizes, const Metric& metric = Metric{},
                     const Kernel& kernel = FlatKernel<>{.5f}, int32_t grid_mode = CLUE_GRID_SHARED) {
    copyToDevice(q, d, h);
    make_clusters(q, d, batch_item_sizes, metric, kernel, grid_mode);
    copyToHost(q, h, d);
  }
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  void make_clusters(Queue& q, PointsDevice<Ndim, TIn>& d, std::span<const uint32_t> batch_item_sizes,
                     const Metric& metric = Metric{}, const Kernel& kernel = FlatKernel<>{.5f},
                     int32_t grid_mode = CLUE_GRID_SHARED) {
    const clue_params p = with(metric, kernel);
    const clue_points pts = d.abi();
    detail::check(clue_make_clusters_batched_device(workspace(q.device()), &p, &pts,
                                                    batch_item_sizes.data(),
                                                    static_cast<int32_t>(batch_item_sizes.size()),
                                                    grid_mode, q.stream()));
    batch_size_ = static_cast<int32_t>(batch_item_sizes.size());
    finish(q, d);
  }

  // No reference counterpart: CUDA-graph replay of repeated identical device
  // runs, launch tuning and the autotuner (clue_workspace_set_graphs,
  // clue_workspace_{get,set}_tuning, clue_workspace_autotune). Results do not
  // depend on any of them.
  void set_graphs(Queue& q, bool enable) {
    detail::check(clue_workspace_set_graphs(workspace(q.device()), enable ? 1 : 0));
  }
  clue_tuning tuning(Queue& q) {
    clue_tuning t{};
    detail::check(clue_workspace_get_tuning(workspace(q.device()), &t));
    return t;
  }
  void set_tuning(Queue& q, const clue_tuning& t) {
    detail::check(clue_workspace_set_tuning(workspace(q.device()), &t));
  }
  template <typename TIn, typename Metric = EuclideanMetric<Ndim>, typename Kernel = FlatKernel<>>
  clue_tuning autotune(Queue& q, PointsDevice<Ndim, TIn>& d, const Metric& metric = Metric{},
                       const Kernel& kernel = FlatKernel<>{.5f}, int32_t reps = 3) {
    const clue_params p = with(metric, kernel);
    const clue_points pts = d.abi();
    clue_tuning t{};
    detail::check(clue_workspace_autotune(workspace(q.device()), &p, &pts, nullptr, 0, 0, q.stream(), reps,
                                          &t));
    finish(q, d);
    return t;
  }

  // getSeeds (:197-203): seed indices of the last run; cluster id k is seeds[k].
  std::span<const int32_t> getSeeds() {
    if (!ws_)
      throw std::runtime_error("Seeds are not available. Please run make_clusters first.");
    int32_t n = 0;
    detail::check(clue_get_seeds(ws_, nullptr, 0, &n));
    seeds_.resize(n);
    detail::check(clue_get_seeds(ws_, seeds_.data(), n, &n));
    return {seeds_.data(), seeds_.size()};
  }

  // getClusters (:205-217): cluster -> points.
  template <typename TIn>
  AssociationMapHost getClusters(const PointsHost<Ndim, TIn>& h) {
    return AssociationMapHost::from_keys(h.clusterIndexes());
  }

  // getSampleAssociations (:219-242): event -> cluster ids of the last batched run.
  template <typename TIn>
  AssociationMapHost getSampleAssociations(Queue&, PointsHost<Ndim, TIn>&) {
    return sample_associations();
  }
  template <typename TIn>
  AssociationMapHost getSampleAssociations(Queue&, PointsDevice<Ndim, TIn>&) {
    return sample_associations();
  }

 private:
  template <typename Metric, typename Kernel>
  clue_params with(const Metric& metric, const Kernel& kernel) const {
    clue_params p = params_;
    metric.fill(p);
    kernel.fill(p);
    detail::check(clue_validate_params(&p));
    return p;
  }
  clue_workspace* workspace(int32_t device) {
    if (!ws_) {
      detail::check(clue_workspace_create(&ws_, device));
      device_ = device;
    }
    return ws_;
  }
  template <typename D>
  void finish(Queue& q, D& d) {
    q.wait();
    int32_t k = 0;
    detail::check(clue_n_clusters(ws_, &k));
    d.set_n_clusters(static_cast<std::size_t>(k));
    d.mark_clustered();
  }
  AssociationMapHost sample_associations() {
    if (!ws_)
      throw std::runtime_error("Seeds are not available. Please run make_clusters first.");
    std::vector<int32_t> off(static_cast<std::size_t>(batch_size_) + 1);
    int32_t nkeys = 0;
    detail::check(clue_sample_associations(ws_, off.data(), batch_size_ + 1, &nkeys));
    off.resize(static_cast<std::size_t>(nkeys) + 1);
    std::vector<int32_t> ids(off.back());
    std::iota(ids.begin(), ids.end(), 0);
    return AssociationMapHost(std::move(off), std::move(ids));
  }

  clue_params params_{};
  clue_workspace* ws_ = nullptr;
  int32_t device_ = 0;
  int32_t batch_size_ = 1;
  std::vector<int32_t> seeds_;
};

// ---------------------------------------------------------------------------
// Validation utilities (utils/cluster_centroid.hpp, utils/scores.hpp): the
// reference's host functions over a clustered PointsHost, computed on GPU 0
// (clue_cluster_centroids_device, clue_silhouette_device) from temporary
// device copies of the points and of their cluster map.
// ---------------------------------------------------------------------------

template <std::size_t Ndim, typename ValueType = float>
using Centroid = std::array<std::remove_cv_t<ValueType>, Ndim>;
template <std::size_t Ndim, typename ValueType = float>
using Centroids = std::vector<Centroid<Ndim, ValueType>>;

namespace detail {

// Device copies of a clustered host point set (coordinates, weights, labels)
// and of its cluster map; released when the object goes.
template <std::size_t Ndim>
class DeviceClusters {
 public:
  template <typename T>
  explicit DeviceClusters(const PointsHost<Ndim, T>& h) : q_{get_device(0)} {
    if (!h.clustered())
      throw std::runtime_error("the points have not been clustered");
    const clue_points hp = h.abi();
    const std::size_t n = static_cast<std::size_t>(h.size());
    map_ = AssociationMapHost::from_keys(h.clusterIndexes());
    pts_.ndim = static_cast<int32_t>(Ndim);
    pts_.n = h.size();
    for (std::size_t d = 0; d < Ndim; ++d)
      pts_.coords[d] = static_cast<const float*>(upload(hp.coords[d], n * 4));
    pts_.weight = static_cast<const float*>(upload(hp.weight, n * 4));
    pts_.cluster_index = static_cast<int32_t*>(upload(h.clusterIndexes().data(), n * 4));
    offsets_ = static_cast<int32_t*>(upload(map_.offsets().data(), map_.offsets().size() * 4));
    members_ = static_cast<int32_t*>(upload(map_.values().data(), map_.values().size() * 4));
  }
  DeviceClusters(const DeviceClusters&) = delete;
  DeviceClusters& operator=(const DeviceClusters&) = delete;
  ~DeviceClusters() {
    clue_stream_synchronize(q_.stream());
    for (void* p : bufs_)
      clue_device_free(p);
  }

  int32_t n_clusters() const { return static_cast<int32_t>(map_.size()); }

  // n_clusters x Ndim, row-major
  std::vector<float> centroids(bool weighted) {
    const std::size_t k = static_cast<std::size_t>(n_clusters());
    std::vector<float> out(k * Ndim);
    if (k == 0)
      return out;
    auto* d_out = static_cast<float*>(alloc(out.size() * 4));
    check(clue_cluster_centroids_device(&pts_, offsets_, members_, n_clusters(), weighted ? 1 : 0, d_out,
                                        q_.stream()));
    check(clue_memcpy_async(out.data(), d_out, out.size() * 4, 1, q_.stream()));
    q_.wait();
    return out;
  }

  // per point; NaN where the reference's mean skips the point
  std::vector<float> silhouettes() {
    std::vector<float> out(static_cast<std::size_t>(pts_.n));
    auto* d_out = static_cast<float*>(alloc(out.size() * 4));
    check(clue_silhouette_device(&pts_, offsets_, members_, n_clusters(), d_out, q_.stream()));
    check(clue_memcpy_async(out.data(), d_out, out.size() * 4, 1, q_.stream()));
    q_.wait();
    return out;
  }

 private:
  void* alloc(std::size_t bytes) {
    void* p = nullptr;
    check(clue_device_malloc(&p, std::max<std::size_t>(bytes, 4), q_.device()));
    bufs_.push_back(p);
    return p;
  }
  void* upload(const void* src, std::size_t bytes) {
    void* p = alloc(bytes);
    if (bytes)
      check(clue_memcpy_async(p, src, bytes, 0, q_.stream()));
    return p;
  }

  Queue q_;
  AssociationMapHost map_;
  clue_points pts_{};
  int32_t* offsets_ = nullptr;
  int32_t* members_ = nullptr;
  std::vector<void*> bufs_;
};

template <std::size_t Ndim>
Centroids<Ndim> to_centroids(const std::vector<float>& flat) {
  Centroids<Ndim> out(flat.size() / Ndim);
  for (std::size_t c = 0; c < out.size(); ++c)
    std::copy_n(flat.begin() + static_cast<std::ptrdiff_t>(c * Ndim), Ndim, out[c].begin());
  return out;
}

}  // namespace detail

// cluster_centroids / weighted_cluster_centroids (utils/detail/cluster_centroid.hpp:86-140)
template <std::size_t Ndim, typename T>
Centroids<Ndim> cluster_centroids(const PointsHost<Ndim, T>& points) {
  detail::DeviceClusters<Ndim> dc(points);
  return detail::to_centroids<Ndim>(dc.centroids(false));
}
template <std::size_t Ndim, typename T>
Centroids<Ndim> weighted_cluster_centroids(const PointsHost<Ndim, T>& points) {
  detail::DeviceClusters<Ndim> dc(points);
  return detail::to_centroids<Ndim>(dc.centroids(true));
}
// cluster_centroid / weighted_cluster_centroid (:16-84): zeros for a cluster
// with no points.
template <std::size_t Ndim, typename T>
Centroid<Ndim> cluster_centroid(const PointsHost<Ndim, T>& points, std::size_t cluster_id) {
  const auto all = cluster_centroids(points);
  return cluster_id < all.size() ? all[cluster_id] : Centroid<Ndim>{};
}
template <std::size_t Ndim, typename T>
Centroid<Ndim> weighted_cluster_centroid(const PointsHost<Ndim, T>& points, std::size_t cluster_id) {
  const auto all = weighted_cluster_centroids(points);
  return cluster_id < all.size() ? all[cluster_id] : Centroid<Ndim>{};
}

// silhouette(points, point) and silhouette(points) (utils/detail/scores.hpp:33-100);
// the mean is the reference's std::reduce over the points it keeps.
template <std::size_t Ndim, typename T>
float silhouette(const PointsHost<Ndim, T>& points, std::size_t point) {
  detail::DeviceClusters<Ndim> dc(points);
  return dc.silhouettes().at(point);
}
template <std::size_t Ndim, typename T>
float silhouette(const PointsHost<Ndim, T>& points) {
  detail::DeviceClusters<Ndim> dc(points);
  const std::vector<float> all = dc.silhouettes();
  std::vector<float> scores;
  for (float s : all)
    if (s == s)
      scores.push_back(s);
  return std::reduce(scores.begin(), scores.end(), 0.0f) / static_cast<float>(scores.size());
}

}  // namespace clue
