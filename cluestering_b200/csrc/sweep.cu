// sweep.cu — local density (core/detail/ClusteringKernels.hpp:29-140) and
// nearest higher (:142-291) over the tile-contiguous layout.
//
// Summation order. The reference adds the contributions to rho_i tile by tile
// in the order of for_recursion (dimension 0 outermost, last dimension fastest)
// and, inside a tile, in the order the association map lists the tile's points
// — ascending index for the serial backend. The sorted layout stores every tile
// contiguously with its points in ascending index, and each thread walks its own
// search box in the same order, so every rho is bit-identical to the serial
// result. The nearest-higher choice is order-independent given identical rho and
// distances (the comparisons form a strict order on (distance, rho, tag)).
#include <cfloat>

#include "sweep.cuh"

namespace clue_impl {

namespace {

constexpr int kThreads = 256;
// sqrtf(2.0f), correctly rounded (the reference's math::sqrt(TData{2})).
constexpr float kSqrt2 = 1.41421356237309504880f;

int grid_for(int64_t n) {
  const int64_t b = (n + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

// Search box of point s: bins [inf, sup] per dimension (TilesView.hpp:77-87),
// half width max(r, r * sigma * sqrt(2)) (ClusteringKernels.hpp:112-118).
template <int D>
__device__ __forceinline__ void search_box(const GridDesc& g, const RunParams& p, const float* xi,
                                           const float* si, float radius, int* inf, int* sup) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float r = std_max(radius, __fmul_rn(__fmul_rn(radius, si[d]), kSqrt2));
    inf[d] = get_bin(g, p, __fsub_rn(xi[d], r), d);
    sup[d] = get_bin(g, p, __fadd_rn(xi[d], r), d);
    if (p.wrapped[d] && inf[d] > sup[d])
      sup[d] += g.k;
  }
}

// Advances the tile odometer (last dimension fastest); false when exhausted.
template <int D>
__device__ __forceinline__ bool next_tile(int* b, const int* inf, const int* sup) {
  bool carry = true;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    if (carry) {
      if (b[d] < sup[d]) {
        ++b[d];
        carry = false;
      } else {
        b[d] = inf[d];
      }
    }
  }
  return !carry;
}

template <int D>
__device__ __forceinline__ int tile_id(const GridDesc& g, const RunParams& p, int base, const int* b) {
  int t = base;
#pragma unroll
  for (int d = 0; d < D; ++d)
    t += g.stride[d] * wrap_bin(g, p, b[d], d);
  return t;
}

template <int D>
__global__ void __launch_bounds__(kThreads) k_density(const RunParams p, const SweepArgs a) {
  const int64_t n = a.n;
  const bool mahalanobis = p.metric_kind == CLUE_METRIC_MAHALANOBIS;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    float xi[D], si[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      xi[d] = a.sx[d * n + s];
      si[d] = ((p.has_sigma >> d) & 1) ? a.ssig[d * n + s] : 0.0f;
    }
    const int gi = a.perm[s];
    int inf[D], sup[D], b[D];
    search_box<D>(g, p, xi, si, p.dc, inf, sup);
#pragma unroll
    for (int d = 0; d < D; ++d)
      b[d] = inf[d];
    float rho = 0.0f;
    do {
      const int t = tile_id<D>(g, p, ev.tile_base, b);
      const int q1 = a.tile_offset[t + 1];
      for (int q = a.tile_offset[t]; q < q1; ++q) {
        float xj[D], sj[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          xj[d] = a.sx[d * n + q];
          sj[d] = mahalanobis ? a.ssig[d * n + q] : 0.0f;
        }
        const int gj = a.perm[q];
        const float dist = metric_finish(p, metric_inner<D>(p, xi, xj, si, sj));
        const float k = kernel_value(p, dist, gi == gj);
        // rho_i += static_cast<int>(distance <= density_radius) * k * w_j
        rho = __fadd_rn(rho, __fmul_rn(__fmul_rn((float)(int)(dist <= p.dc), k), a.sw[q]));
      }
    } while (next_tile<D>(b, inf, sup));
    a.srho[s] = rho;
    if (a.out_rho)
      a.out_rho[gi] = rho;
  }
}

template <int D>
__global__ void __launch_bounds__(kThreads) k_nearest_higher(const RunParams p, const SweepArgs a) {
  const int64_t n = a.n;
  const bool mahalanobis = p.metric_kind == CLUE_METRIC_MAHALANOBIS;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    float xi[D], si[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      xi[d] = a.sx[d * n + s];
      si[d] = ((p.has_sigma >> d) & 1) ? a.ssig[d * n + s] : 0.0f;
    }
    const int gi = a.perm[s];
    const float rho_i = a.srho[s];
    const float unc = p.has_unc ? a.sunc[s] : 1.0f;
    const float min_density = __fmul_rn(p.rhoc, unc);
    // ClusteringKernels.hpp:168
    const float eff = (rho_i >= min_density) ? p.seed_dc : p.dm;
    const uint32_t tag_i = p.has_tags ? a.stag[s] : (uint32_t)gi;
    int inf[D], sup[D], b[D];
    search_box<D>(g, p, xi, si, p.dm, inf, sup);
#pragma unroll
    for (int d = 0; d < D; ++d)
      b[d] = inf[d];
    float delta = FLT_MAX;
    int nh = -1;
    float rho_nh = 0.0f;
    uint32_t tag_nh = 0;
    do {
      const int t = tile_id<D>(g, p, ev.tile_base, b);
      const int q1 = a.tile_offset[t + 1];
      for (int q = a.tile_offset[t]; q < q1; ++q) {
        const float rho_j = a.srho[q];
        const int gj = a.perm[q];
        const uint32_t tag_j = p.has_tags ? a.stag[q] : (uint32_t)gj;
        // ClusteringKernels.hpp:180-182
        const bool higher =
            (rho_j > rho_i) || ((rho_j == rho_i) && (rho_j > 0.0f) && (tag_j > tag_i));
        if (!higher)
          continue;
        float xj[D], sj[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          xj[d] = a.sx[d * n + q];
          sj[d] = mahalanobis ? a.ssig[d * n + q] : 0.0f;
        }
        const float dist = metric_finish(p, metric_inner<D>(p, xi, xj, si, sj));
        // ClusteringKernels.hpp:195-202
        if (dist <= eff &&
            ((dist < delta) ||
             ((dist == delta) && (nh >= 0) &&
              ((rho_j > rho_nh) || ((rho_j == rho_nh) && (tag_j > tag_nh)))))) {
          delta = dist;
          nh = gj;
          rho_nh = rho_j;
          tag_nh = tag_j;
        }
      }
    } while (next_tile<D>(b, inf, sup));
    a.out_nh[gi] = nh;
    // KernelFindClusters, ClusteringKernels.hpp:301-313
    const int seed = (nh == -1) && (rho_i >= min_density);
    a.seed_flag[gi] = seed;
    if (a.out_seed)
      a.out_seed[gi] = seed;
  }
}


}  // namespace

#define CLUE_DISPATCH_D(D, KERNEL, ...)                                         \
  switch (D) {                                                                 \
    case 1: KERNEL<1><<<__VA_ARGS__>>>(p, a); break;                           \
    case 2: KERNEL<2><<<__VA_ARGS__>>>(p, a); break;                           \
    case 3: KERNEL<3><<<__VA_ARGS__>>>(p, a); break;                           \
    case 4: KERNEL<4><<<__VA_ARGS__>>>(p, a); break;                           \
    case 5: KERNEL<5><<<__VA_ARGS__>>>(p, a); break;                           \
    case 6: KERNEL<6><<<__VA_ARGS__>>>(p, a); break;                           \
    case 7: KERNEL<7><<<__VA_ARGS__>>>(p, a); break;                           \
    case 8: KERNEL<8><<<__VA_ARGS__>>>(p, a); break;                           \
    case 9: KERNEL<9><<<__VA_ARGS__>>>(p, a); break;                           \
    case 10: KERNEL<10><<<__VA_ARGS__>>>(p, a); break;                         \
    default: return cudaErrorInvalidValue;                                     \
  }

cudaError_t launch_density(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  if (a.n == 0)
    return cudaSuccess;
  CLUE_DISPATCH_D(D, k_density, grid_for(a.n), kThreads, 0, st)
  return cudaGetLastError();
}

cudaError_t launch_nearest_higher(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  if (a.n == 0)
    return cudaSuccess;
  CLUE_DISPATCH_D(D, k_nearest_higher, grid_for(a.n), kThreads, 0, st)
  return cudaGetLastError();
}

}  // namespace clue_impl
