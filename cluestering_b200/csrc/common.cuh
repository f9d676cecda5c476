// common.cuh — device-side building blocks shared by the clustering kernels.
//
// Every floating-point expression that decides a result restates the
// reference's expression with explicit round-to-nearest intrinsics, so the
// compiler can neither contract it into an FMA nor reorder it; the library is
// also compiled with -fmad=false. Citations are relative to the CLUEstering
// repository root.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "clue_expf.h"
#include "clue_sm100.h"

namespace clue_impl {

constexpr int kMaxDim = CLUE_MAX_DIM;
// Tiles of more points than this are "large": the tile sort lists them
// (DeviceBuffers::large_tiles) and the kernels that work tile by tile give
// each of them a whole block instead of one warp.
constexpr int kLargeTilePoints = 256;

// ---------------------------------------------------------------------------
// Tables the host builds for a run
// ---------------------------------------------------------------------------

// One tile grid (data_structures/internal/Tiles.hpp:141-280, TilesView.hpp:19-27).
// minv/maxv/tile are computed on the device from the points.
struct GridDesc {
  int32_t k;  // tiles per dimension (n_per_dim)
  int32_t T;  // k^D tiles per event
  int32_t stride[kMaxDim];  // k^(D-1-d)
  float minv[kMaxDim];
  float maxv[kMaxDim];
  float tile[kMaxDim];
};

// One event of a (possibly single-event) batch.
struct EventDesc {
  int32_t begin;      // first point (global index)
  int32_t n;          // number of points
  int32_t tile_base;  // first global tile id of this event
  int32_t grid;       // index into the grid table
  // Stable tile binning: the event's points form sort_chunks runs of sort_len
  // consecutive points, run c binned by warp sort_first + c; its count matrix
  // (runs x tiles, run-major: run c's counts are contiguous) starts at entry
  // sort_base.
  int32_t sort_first;
  int32_t sort_chunks;
  int32_t sort_len;
  int32_t sort_base;
  // The event at position e of the batch's events ordered by size, largest
  // first (so that per-event passes over a queue start with the longest).
  int32_t by_size;
};

// Tiles of one event the stable binning handles: each warp keeps a counter per
// tile of its event in shared memory (16 KB).
constexpr int kStableMaxTiles = 4096;
// Points per run of the stable binning (one warp, 32 rounds).
constexpr int kStableRun = 1024;

// A run of consecutive points of one event, processed by one block.
struct Chunk {
  int32_t event;
  int32_t begin;
  int32_t end;
};

// One cell of the nearest-higher layout: its members occupy [start, end) of
// the layout, and maxkey is the largest (density, tag) key among them.
struct alignas(16) CellInfo {
  int32_t start, end;
  unsigned long long maxkey;
};

// Scalar parameters of a run, passed by value to kernels.
struct RunParams {
  int32_t D;
  float dc, rhoc, dm, seed_dc;
  uint8_t wrapped[kMaxDim];
  int32_t kernel_kind;
  float kernel_p0, kernel_p1;
  int32_t metric_kind;
  float mparam[kMaxDim];
  // Largest squared distance whose correctly rounded square root is <= dc
  // (resp. dm, seed_dc): sqrt_rn is monotone, so `sqrt(d2) <= r` is exactly
  // `d2 <= thr`. Only meaningful for the square-root metrics.
  float dc2, dm2, seed2;
  int32_t has_sigma;  // bit d set when sigma[d] is present
  int32_t has_unc;
  int32_t has_tags;
  // Gaussian kernel: 2^-k when (2 * std) * std is the power of two 2^k, else 0.
  // Dividing by 2^k and multiplying by 2^-k round the same exact value once,
  // so the division can be a multiplication.
  float gauss_inv_den;
  // Nonzero when every exponent the kernel can see for an in-range pair
  // (distance <= dc) lies where clue_expf needs no special-case branch.
  int32_t exp_in_range;
  // Density sweep, warps whose lanes have different search boxes: the warp
  // streams the union of the boxes when the union holds at most
  // union_x16 / 16 times the candidates of its lanes' largest own box, else
  // each lane reads its own candidates (clue_tuning::density_union_x16_2d/3d).
  int32_t union_x16;
  // Pointer-jumping rounds before the label walk; -1: by size.
  int32_t jump_rounds;
  // Average points per cell of the sweeps' cell layout (1..8).
  int32_t cell_points;
  // Block shapes of the density sweep and of the nearest-higher cell search
  // (clue_tuning::density_shape, nh_shape).
  int32_t dens_shape;
  int32_t nh_shape;
  // Stable tile binning when the run's shape allows it (clue_tuning::tile_binning).
  int32_t stable_binning;
};

// ---------------------------------------------------------------------------
// Scalar semantics
// ---------------------------------------------------------------------------

// static_cast<int>(float) as the reference's serial backend executes it on
// x86-64 (cvttss2si): truncation, and INT_MIN for NaN or out-of-range values.
__device__ __forceinline__ int f2i_x86(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? __float2int_rz(v) : INT_MIN;
}

// std::max / std::min on floats.
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; }

// Order-preserving int image of a float (for atomicMin/atomicMax).
__device__ __forceinline__ int f2ord(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : (i ^ 0x7FFFFFFF);
}
__device__ __forceinline__ float ord2f(int i) { return __int_as_float(i >= 0 ? i : (i ^ 0x7FFFFFFF)); }

// ---------------------------------------------------------------------------
// Tile grid (data_structures/internal/TilesView.hpp)
// ---------------------------------------------------------------------------

// normalizeCoordinate, TilesView.hpp:96-104.
__device__ __forceinline__ float normalize_coordinate(const GridDesc& g, float coord, int dim) {
  const float range = __fsub_rn(g.maxv[dim], g.minv[dim]);
  const float q = (float)f2i_x86(__fdiv_rn(coord, range));
  float rem = __fsub_rn(coord, __fmul_rn(q, range));
  if (rem >= g.maxv[dim])
    rem = __fsub_rn(rem, range);
  else if (rem < g.minv[dim])
    rem = __fadd_rn(rem, range);
  return rem;
}

// getBin, TilesView.hpp:38-52.
__device__ __forceinline__ int get_bin(const GridDesc& g, const RunParams& p, float coord, int dim) {
  const float c = p.wrapped[dim] ? normalize_coordinate(g, coord, dim) : coord;
  int b = f2i_x86(__fdiv_rn(__fsub_rn(c, g.minv[dim]), g.tile[dim]));
  b = min(b, g.k - 1);
  b = max(b, 0);
  return b;
}

// Wrap of a search-box bin, TilesView.hpp:66-75 (`Bins[dim] % nperdim`).
__device__ __forceinline__ int wrap_bin(const GridDesc& g, const RunParams& p, int b, int dim) {
  return p.wrapped[dim] ? (b % g.k) : b;
}

// ---------------------------------------------------------------------------
// Distance metrics (core/DistanceMetrics.hpp). `acc` folds from the last
// dimension, which is meta::accumulate's right fold f0 + (f1 + (... + 0)).
// ---------------------------------------------------------------------------

// Squared-distance part of the square-root metrics, or the full distance of
// Manhattan/Chebyshev; `xi`/`xj` are the coordinates, `si`/`sj` the sigmas
// (Mahalanobis only).
template <int D>
__device__ __forceinline__ float metric_inner(const RunParams& p, const float* xi, const float* xj,
                                              const float* si, const float* sj) {
  float acc = 0.0f;
  switch (p.metric_kind) {
    case CLUE_METRIC_EUCLIDEAN:  // :108-113
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        const float diff = __fsub_rn(xi[d], xj[d]);
        acc = __fadd_rn(__fmul_rn(diff, diff), acc);
      }
      return acc;
    case CLUE_METRIC_WEIGHTED_EUCLIDEAN:  // :156-162
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        const float diff = __fsub_rn(xi[d], xj[d]);
        acc = __fadd_rn(__fmul_rn(__fmul_rn(p.mparam[d], diff), diff), acc);
      }
      return acc;
    case CLUE_METRIC_PERIODIC_EUCLIDEAN:  // :212-220
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        const float diff = fabsf(__fsub_rn(xi[d], xj[d]));
        const float pd = std_min(diff, __fsub_rn(p.mparam[d], diff));
        acc = __fadd_rn(__fmul_rn(pd, pd), acc);
      }
      return acc;
    case CLUE_METRIC_MANHATTAN:  // :241-245
#pragma unroll
      for (int d = D - 1; d >= 0; --d)
        acc = __fadd_rn(fabsf(__fsub_rn(xi[d], xj[d])), acc);
      return acc;
    case CLUE_METRIC_CHEBYSHEV:  // :266-270
#pragma unroll
      for (int d = 0; d < D; ++d)
        acc = std_max(acc, fabsf(__fsub_rn(xi[d], xj[d])));
      return acc;
    case CLUE_METRIC_WEIGHTED_CHEBYSHEV:  // :313-317
#pragma unroll
      for (int d = 0; d < D; ++d)
        acc = std_max(acc, __fmul_rn(p.mparam[d], fabsf(__fsub_rn(xi[d], xj[d]))));
      return acc;
    case CLUE_METRIC_MAHALANOBIS:  // :76-86
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        const float diff = __fsub_rn(xi[d], xj[d]);
        const float den = __fadd_rn(__fmul_rn(si[d], si[d]), __fmul_rn(sj[d], sj[d]));
        acc = __fadd_rn(__fdiv_rn(__fmul_rn(diff, diff), den), acc);
      }
      return acc;
    default:
      return __int_as_float(0x7fc00000);
  }
}

__device__ __forceinline__ bool metric_has_sqrt(int kind) {
  return kind != CLUE_METRIC_MANHATTAN && kind != CLUE_METRIC_CHEBYSHEV &&
         kind != CLUE_METRIC_WEIGHTED_CHEBYSHEV;
}

// Final distance from metric_inner's value.
__device__ __forceinline__ float metric_finish(const RunParams& p, float inner) {
  return metric_has_sqrt(p.metric_kind) ? __fsqrt_rn(inner) : inner;
}

// Convolutional kernel value, core/detail/ConvolutionalKernel.hpp:13-57.
__device__ __forceinline__ float kernel_value(const RunParams& p, float dist, bool self) {
  if (self)
    return 1.0f;
  switch (p.kernel_kind) {
    case CLUE_KERNEL_FLAT:
      return p.kernel_p0;
    case CLUE_KERNEL_GAUSSIAN: {
      // amp * exp(-d * d / (2 * std * std))
      const float num = __fmul_rn(-dist, dist);
      const float den = __fmul_rn(__fmul_rn(2.0f, p.kernel_p0), p.kernel_p0);
      return __fmul_rn(p.kernel_p1, clue_expf(__fdiv_rn(num, den)));
    }
    case CLUE_KERNEL_EXPONENTIAL:
      // amp * exp(-avg * d)
      return __fmul_rn(p.kernel_p1, clue_expf(__fmul_rn(-p.kernel_p0, dist)));
    default:
      return __int_as_float(0x7fc00000);
  }
}

// Kernel value of an in-range pair for the fast sweep: the same operations as
// kernel_value, with the Gaussian division replaced by the exact power-of-two
// multiplication when available and clue_expf's range branches dropped when the
// host proved they cannot trigger (RunParams::exp_in_range).
__device__ __forceinline__ float kernel_value_in_range(const RunParams& p, float dist, bool self) {
  if (self)
    return 1.0f;
  if (p.kernel_kind == CLUE_KERNEL_GAUSSIAN) {
    const float num = __fmul_rn(-dist, dist);
    const float den = __fmul_rn(__fmul_rn(2.0f, p.kernel_p0), p.kernel_p0);
    const float x = p.gauss_inv_den != 0.0f ? __fmul_rn(num, p.gauss_inv_den) : __fdiv_rn(num, den);
    return __fmul_rn(p.kernel_p1, p.exp_in_range ? clue_expf_core(x) : clue_expf(x));
  }
  if (p.kernel_kind == CLUE_KERNEL_EXPONENTIAL) {
    const float x = __fmul_rn(-p.kernel_p0, dist);
    return __fmul_rn(p.kernel_p1, p.exp_in_range ? clue_expf_core(x) : clue_expf(x));
  }
  return p.kernel_p0;
}

// ---------------------------------------------------------------------------
// Exact-sum events (flat kernel)
//
// The reference adds a point's density contributions in its tile order, and
// float addition rounds, so in general only that order reproduces its bits.
// When every contribution of an event (fl(flat * w_j) for a neighbour, w_i for
// the point itself) is a non-negative integer multiple of u = 2^min_lsb and
// their total over the event is at most 2^24 u, every partial sum of any subset
// is an integer multiple of u no larger than 2^24 u, which binary32 represents
// exactly: no addition rounds, and the ordered sum equals the exact sum in any
// order (unit weights are the common case: multiples of 1/2). k_bin records per
// event (4 ints): the smallest lowest-set-bit exponent of any contribution, the
// largest neighbour contribution and the largest weight (float bits), and a
// flag for a negative, -0, NaN or infinite one.
// ---------------------------------------------------------------------------

// Exponent of the lowest set bit of a positive finite float: x = m * 2^e with
// m odd returns e.
__device__ __forceinline__ int lsb_exponent(float x) {
  const uint32_t bits = __float_as_uint(x);
  const uint32_t ex = (bits >> 23) & 0xffu;
  const uint32_t m = ex ? ((bits & 0x7fffffu) | 0x800000u) : (bits & 0x7fffffu);
  return (ex ? (int)ex - 150 : -149) + (__ffs(m) - 1);
}

// The bound is checked in double: the true bound n * max_v + max_w and 2^24 u
// are multiples of u, so a true bound above 2^24 u is at least (2^24 + 1) u,
// which the double product cannot round down to 2^24 u.
__device__ __forceinline__ bool event_sums_exact(const int32_t* event_exact, int e, int n_points) {
  const int4 st = reinterpret_cast<const int4*>(event_exact)[e];
  if (st.w != 0)
    return false;
  if (st.x == INT_MAX)
    return true;  // every contribution is zero
  const double bound = (double)n_points * (double)__int_as_float(st.y) + (double)__int_as_float(st.z);
  return bound <= ldexp(1.0, 24 + st.x);
}

// Status word bits written by kernels whose waits are bounded.
enum : uint32_t {
  kStatusScanTimeout = 1u << 0,
  kStatusSortOverflow = 1u << 1,
  kStatusLabelTimeout = 1u << 2,
  kStatusCopyTimeout = 1u << 3,
  kStatusLabelRange = 1u << 4,  // a nearest-higher chain left its event
};

}  // namespace clue_impl
