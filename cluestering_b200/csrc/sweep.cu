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
//
// Warp-uniform work. The thread -> point assignment is free: each sweep
// processes points in an order where the points of one tile are grouped by the
// shape of their search box (launch_work_order). The 32 lanes of a warp then
// walk the same tiles and read the same candidate at the same time, so every
// candidate load is one broadcast and the loops do not diverge.
#include <cfloat>

#include "engine.h"
#include "sweep.cuh"

namespace clue_impl {

namespace {

constexpr int kThreads = 256;
constexpr unsigned kFullMask = 0xffffffffu;
// sqrtf(2.0f), correctly rounded (the reference's math::sqrt(TData{2})).
constexpr float kSqrt2 = 1.41421356237309504880f;

int grid_for(int64_t n) {
  const int64_t b = (n + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count() * 16));
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
__device__ __forceinline__ void load_point(const RunParams& p, const SweepArgs& a, int64_t s, float* x,
                                           float* sg) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    x[d] = a.sx[d * a.n + s];
    sg[d] = ((p.has_sigma >> d) & 1) ? a.ssig[d * a.n + s] : 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Work order: within each tile, points grouped by search-box class
// ---------------------------------------------------------------------------

template <int D>
__host__ __device__ constexpr int box_classes() {
  return D == 1 ? 9 : D == 2 ? 81 : D == 3 ? 729 : 1;
}

// Class of a search box relative to the point's own tile: per dimension
// (own - inf, sup - own) each capped at 2, so points of one tile with equal
// class have equal boxes whenever the box spans at most 3 tiles per dimension.
template <int D>
__device__ __forceinline__ int box_class(const GridDesc& g, const int* own, const int* inf,
                                         const int* sup) {
  if (box_classes<D>() == 1)
    return 0;
  int c = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int lo = min(max(own[d] - inf[d], 0), 2);
    const int hi = min(max(sup[d] - own[d], 0), 2);
    c = c * 9 + lo * 3 + hi;
  }
  return c;
}

// Exclusive scan of cnt[0..E) in place by one warp.
template <int E>
__device__ void warp_scan_counts(int* cnt) {
  const int lane = threadIdx.x & 31;
  constexpr int per = (E + 31) / 32;
  int local[per];
  int sum = 0;
#pragma unroll
  for (int j = 0; j < per; ++j) {
    const int k = lane * per + j;
    local[j] = k < E ? cnt[k] : 0;
    sum += local[j];
  }
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o)
      incl += y;
  }
  int run = incl - sum;
#pragma unroll
  for (int j = 0; j < per; ++j) {
    const int k = lane * per + j;
    if (k < E)
      cnt[k] = run;
    run += local[j];
  }
}

template <int D>
__global__ void __launch_bounds__(kThreads) k_work_order(const RunParams p, const SweepArgs a) {
  constexpr int E = box_classes<D>();
  __shared__ int cnt[2][E];
  for (int64_t t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
    const int begin = a.tile_offset[t], end = a.tile_offset[t + 1];
    if (end - begin == 0)
      continue;
    if (end - begin == 1 || E == 1) {
      for (int s = begin + threadIdx.x; s < end; s += blockDim.x) {
        a.work_dens[s] = s;
        a.work_nh[s] = s;
      }
      continue;
    }
    for (int i = threadIdx.x; i < 2 * E; i += blockDim.x)
      (&cnt[0][0])[i] = 0;
    __syncthreads();
    const EventDesc ev = a.events[a.sevt[begin]];
    const GridDesc& g = a.grids[ev.grid];
    int own[D];
    {
      int local = (int)t - ev.tile_base;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        own[d] = local / g.stride[d];
        local -= own[d] * g.stride[d];
      }
    }
    // the cell search of the nearest higher visits points in layout order and
    // needs no work order of its own
    const bool nh_order = !a.nh_cells;
    for (int s = begin + threadIdx.x; s < end; s += blockDim.x) {
      float xi[D], si[D];
      load_point<D>(p, a, s, xi, si);
      int inf[D], sup[D];
      search_box<D>(g, p, xi, si, p.dc, inf, sup);
      const int cd = box_class<D>(g, own, inf, sup);
      a.cls_dens[s] = cd;
      atomicAdd(&cnt[0][cd], 1);
      if (nh_order) {
        search_box<D>(g, p, xi, si, p.dm, inf, sup);
        const int cn = box_class<D>(g, own, inf, sup);
        a.cls_nh[s] = cn;
        atomicAdd(&cnt[1][cn], 1);
      }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    if (warp < (nh_order ? 2 : 1))
      warp_scan_counts<E>(cnt[warp]);
    __syncthreads();
    for (int s = begin + threadIdx.x; s < end; s += blockDim.x) {
      a.work_dens[begin + atomicAdd(&cnt[0][a.cls_dens[s]], 1)] = s;
      if (nh_order)
        a.work_nh[begin + atomicAdd(&cnt[1][a.cls_nh[s]], 1)] = s;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Generic sweeps: any D, metric, kernel and option
// ---------------------------------------------------------------------------

template <int D>
__global__ void __launch_bounds__(kThreads) k_density(const RunParams p, const SweepArgs a) {
  const int64_t n = a.n;
  const bool mahalanobis = p.metric_kind == CLUE_METRIC_MAHALANOBIS;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int s = a.work_dens[w];
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    float xi[D], si[D];
    load_point<D>(p, a, s, xi, si);
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
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int s = a.work_nh[w];
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    float xi[D], si[D];
    load_point<D>(p, a, s, xi, si);
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
    int nh = -1, nh_pos = s;
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
          nh_pos = q;
          rho_nh = rho_j;
          tag_nh = tag_j;
        }
      }
    } while (next_tile<D>(b, inf, sup));
    a.out_nh[gi] = nh;
    a.parent[s] = nh_pos;
    // KernelFindClusters, ClusteringKernels.hpp:301-313
    const int seed = (nh == -1) && (rho_i >= min_density);
    a.seed_flag[gi] = seed;
    if (a.out_seed)
      a.out_seed[gi] = seed;
  }
}

// ---------------------------------------------------------------------------
// Fast path: D = 2 or 3, Euclidean, no sigma, no wrapped coordinate.
// Candidates are packed float4 records; `sqrt(d2) <= r` is tested as
// `d2 <= thr` with the exact threshold computed on the host; the tiles of one
// row of the search box (last dimension) are contiguous and read as one range.
// ---------------------------------------------------------------------------

// Order-preserving image of a density: key(a) > key(b) iff a > b and equal
// densities give equal keys. NaN maps to 0, below every number, so a NaN
// density is never "higher" (every comparison with NaN is false). Densities
// are never -0 (they start at +0 and round-to-nearest sums of opposite values
// give +0), so no other pair of equal values has different keys.
__device__ __forceinline__ uint32_t rho_key(float rho) {
  if (rho != rho)
    return 0u;
  const uint32_t b = __float_as_uint(rho);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// (x_i - x_j)^2 and (y_i - y_j)^2 with one packed subtract and one packed
// multiply (sm_100 f32x2): each half is the IEEE round-to-nearest result of
// the scalar operation, so the values equal __fsub_rn / __fmul_rn.
__device__ __forceinline__ void sq_diff_xy(float xi, float yi, float xj, float yj, float& sx,
                                           float& sy) {
  asm("{\n\t.reg .b64 a, b, d, s;\n\t"
      "mov.b64 a, {%2, %3};\n\t"
      "mov.b64 b, {%4, %5};\n\t"
      "sub.rn.f32x2 d, a, b;\n\t"
      "mul.rn.f32x2 s, d, d;\n\t"
      "mov.b64 {%0, %1}, s;\n\t}"
      : "=f"(sx), "=f"(sy)
      : "f"(xi), "f"(yi), "f"(xj), "f"(yj));
}

template <int D>
__device__ __forceinline__ float sq_dist(const float* xi, const float4& r) {
  // meta::accumulate right fold: dx^2 + (dy^2 [+ dz^2])
  float sx, sy;
  sq_diff_xy(xi[0], xi[1], r.x, r.y, sx, sy);
  if (D == 2)
    return __fadd_rn(sx, sy);
  const float dz = __fsub_rn(xi[2], r.z);
  return __fadd_rn(sx, __fadd_rn(sy, __fmul_rn(dz, dz)));
}

// Row iteration shared by both fast sweeps: calls body(q) for every candidate
// of the search box in the reference's order.
template <int D, typename Body>
__device__ __forceinline__ void for_each_candidate(const SweepArgs& a, const GridDesc& g, int base,
                                                   const int* inf, const int* sup, Body&& body) {
  if (D == 2) {
    for (int b0 = inf[0]; b0 <= sup[0]; ++b0) {
      const int row = base + b0 * g.stride[0];
      const int qe = a.tile_offset[row + sup[1] + 1];
#pragma unroll 4
      for (int q = a.tile_offset[row + inf[1]]; q < qe; ++q)
        body(q);
    }
  } else {
    for (int b0 = inf[0]; b0 <= sup[0]; ++b0)
      for (int b1 = inf[1]; b1 <= sup[1]; ++b1) {
        const int row = base + b0 * g.stride[0] + b1 * g.stride[1];
        const int qe = a.tile_offset[row + sup[2] + 1];
#pragma unroll 4
        for (int q = a.tile_offset[row + inf[2]]; q < qe; ++q)
          body(q);
      }
  }
}

// ---------------------------------------------------------------------------
// Cell layout (fast path).
//
// Every tile of m points is split into s^D cells, s the largest value with
// s^D * kCellTarget <= m (at least 1, at most cell_dim_max). A point's cell
// comes from cell_coord, which is monotone in the coordinate; a search
// therefore finds every point of [a, b] in the cells cell_coord(a) ..
// cell_coord(b), whatever rounding placed it there. Each cell records the
// bounding box of its members and (for the nearest-higher search) their
// largest key. The density sweep uses the cells to skip candidates no lane of
// a warp can reach; the nearest-higher search visits them nearest-first.
// ---------------------------------------------------------------------------

// Average points per cell: a launch tuning (clue_tuning::cell_points, 1..8,
// default 2). Cells only order and prune the candidates of the sweeps, so the
// choice never changes a result.
constexpr int kCellSlots = 2048;   // cells per tile at most (45^2, 12^3)
constexpr int kCellWarps = 8;      // warps per block of k_cells

template <int D>
__host__ __device__ constexpr int cell_dim_max() {
  return D == 2 ? 45 : 12;
}

template <int D>
__device__ __forceinline__ int cells_per_dim(int m, int target) {
  int s = 1;
  while (s < cell_dim_max<D>()) {
    const int u = s + 1;
    const int vol = D == 2 ? u * u : u * u * u;
    if (vol * target > m)
      break;
    s = u;
  }
  return s;
}

// Cell coordinate of x in a tile with origin lo and inverse cell width inv
// (0 for a degenerate tile): monotone non-decreasing in x for every non-NaN x,
// clamped to [0, s); NaN lands in cell 0.
__device__ __forceinline__ int cell_coord(float x, float lo, float inv, int s) {
  float u = __fmul_rn(__fsub_rn(x, lo), inv);
  u = fminf(fmaxf(u, 0.0f), (float)(s - 1));
  return (int)u;
}

// Origin and inverse cell width of the tiles' cells, dimension d.
__device__ __forceinline__ void cell_axis(const GridDesc& g, int b, int s, int d, float& lo,
                                          float& inv) {
  lo = __fadd_rn(g.minv[d], __fmul_rn((float)b, g.tile[d]));
  const float v = __fdiv_rn((float)s, g.tile[d]);
  inv = (g.tile[d] > 0.0f && v < INFINITY) ? v : 0.0f;
}

template <int D>
__device__ __forceinline__ void load_geom(const SweepArgs& a, int t, float* lo, float* inv) {
  const float4 g0 = a.cell_geom[D == 2 ? t : 2 * t];
  if (D == 2) {
    lo[0] = g0.x, lo[1] = g0.y, inv[0] = g0.z, inv[1] = g0.w;
  } else {
    const float4 g1 = a.cell_geom[2 * t + 1];
    lo[0] = g0.x, lo[1] = g0.y, lo[D - 1] = g0.z, inv[0] = g0.w, inv[1] = g1.x, inv[D - 1] = g1.y;
  }
}

template <int D>
__device__ __forceinline__ void load_box(const SweepArgs& a, int slot, float* mn, float* mx) {
  const float4 b0 = a.cell_box[D == 2 ? slot : 2 * slot];
  if (D == 2) {
    mn[0] = b0.x, mn[1] = b0.y, mx[0] = b0.z, mx[1] = b0.w;
  } else {
    const float4 b1 = a.cell_box[2 * slot + 1];
    mn[0] = b0.x, mn[1] = b0.y, mn[D - 1] = b0.z, mx[0] = b0.w, mx[1] = b1.x, mx[D - 1] = b1.y;
  }
}

// Lower bound of the squared distance from xi to any member of a cell, with
// the operations of sq_dist: per dimension the gap to the box is at most
// |fl(x_i - x_j)| of every member (rounding is monotone), and squares and the
// right fold are monotone too.
template <int D>
__device__ __forceinline__ float box_lower_bound(const float* xi, const float* mn, const float* mx) {
  float gap[D];
#pragma unroll
  for (int d = 0; d < D; ++d)
    gap[d] = fmaxf(fmaxf(__fsub_rn(mn[d], xi[d]), __fsub_rn(xi[d], mx[d])), 0.0f);
  if (D == 2)
    return __fadd_rn(__fmul_rn(gap[0], gap[0]), __fmul_rn(gap[1], gap[1]));
  return __fadd_rn(__fmul_rn(gap[0], gap[0]),
                   __fadd_rn(__fmul_rn(gap[1], gap[1]), __fmul_rn(gap[D - 1], gap[D - 1])));
}

// |x_j - x_i| <= reach(bound2) in every coordinate for every point with
// fl(d2) <= bound2: each square and sum is rounded to nearest, so
// |x_j - x_i| <= sqrt(bound2) (1 + 2^-22); the factor 1 + 10^-6 and the
// absolute 10^-19 (square roots near the smallest normal) cover that, rounded up.
__device__ __forceinline__ float reach(float bound2) {
  return __fadd_ru(__fmul_ru(__fsqrt_ru(bound2), 1.000001f), 1e-19f);
}

// Asynchronous 16-byte global -> shared copies (per thread, completion by
// commit groups).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Bulk copies (the copy engine inside each SM) into this CTA's shared memory,
// completed on an mbarrier by transaction bytes. Sources are this GPU's own
// memory; nothing is multicast.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier shared-memory accesses before later bulk copies
// into the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of `bar` with this parity, at most kCopyWaitLimit polls
// (each poll itself bounded by the hardware's try-wait time limit). On giving
// up it records kStatusCopyTimeout, so the host call reports CLUE_ERR_TIMEOUT.
constexpr int kCopyWaitLimit = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, uint32_t* status) {
  for (int it = 0; it < kCopyWaitLimit; ++it)
    if (mbar_try_wait(bar, parity))
      return true;
  atomicOr(status, kStatusCopyTimeout);
  return false;
}

// Contribution of candidate record r (sorted position q) to rho_i.
template <int D, int KIND>
__device__ __forceinline__ void density_add(const RunParams& p, const float* xi, const float4& r,
                                            bool self, float wi, float& rho) {
  const float d2 = sq_dist<D>(xi, r);
  if (d2 <= p.dc2) {
    const float v = D == 2 ? r.z : r.w;
    if (KIND == CLUE_KERNEL_FLAT) {
      rho = __fadd_rn(rho, self ? wi : v);
    } else {
      const float k = kernel_value_in_range(p, __fsqrt_rn(d2), self);
      rho = __fadd_rn(rho, __fmul_rn(k, v));
    }
  }
}

// (a, b) as one 64-bit register pair, the operand of the f32x2 instructions.
__device__ __forceinline__ unsigned long long pack2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}

// Squared distance and contribution weight of a streamed record: xi_xy holds
// (x_i, y_i) packed, the record arrives as two packed halves {(x, y), (z or v,
// v or w)}; the arithmetic is that of sq_dist.
template <int D>
__device__ __forceinline__ float packed_d2(unsigned long long xi_xy, float zi, const ulonglong2& r,
                                           float& v) {
  float sx, sy;
  asm("{\n\t.reg .b64 d, s;\n\t"
      "sub.rn.f32x2 d, %2, %3;\n\t"
      "mul.rn.f32x2 s, d, d;\n\t"
      "mov.b64 {%0, %1}, s;\n\t}"
      : "=f"(sx), "=f"(sy)
      : "l"(xi_xy), "l"(r.x));
  float hi_lo, hi_hi;  // the record's second half: D = 2 {v, w}; D = 3 {z, v}
  asm("mov.b64 {%0, %1}, %2;" : "=f"(hi_lo), "=f"(hi_hi) : "l"(r.y));
  v = D == 2 ? hi_lo : hi_hi;
  if (D == 2)
    return __fadd_rn(sx, sy);
  const float dz = __fsub_rn(zi, hi_lo);
  return __fadd_rn(sx, __fadd_rn(sy, __fmul_rn(dz, dz)));
}

// Streamed form of density_add (same arithmetic).
template <int D, int KIND>
__device__ __forceinline__ void density_add_packed(const RunParams& p, unsigned long long xi_xy,
                                                   float zi, const ulonglong2& r, bool self,
                                                   float wi, float& rho) {
  float v;
  const float d2 = packed_d2<D>(xi_xy, zi, r, v);
  if (KIND == CLUE_KERNEL_FLAT) {
    if (d2 <= p.dc2)
      rho = __fadd_rn(rho, self ? wi : v);
  } else if (d2 <= p.dc2) {
    const float k = kernel_value_in_range(p, __fsqrt_rn(d2), self);
    rho = __fadd_rn(rho, __fmul_rn(k, v));
  }
}

constexpr int kRing = 4;       // chunks of candidate records in flight per warp
constexpr int kChunk = 32;     // records per chunk (kChunk / 32 per lane)
constexpr int kMaxRows = 32;   // rows of a search box the streamed path handles

// Copies stream positions c * kChunk + lane + 32 k (row table off/qa, row
// cursor rr) into ring slot c % kRing, then closes the lane's commit group for
// chunk c.
__device__ __forceinline__ void stream_issue(float4 (*ring)[kChunk], const int* off, const int* qa,
                                             const float4* rec, int c, int lane, int total,
                                             int& rr) {
#pragma unroll
  for (int k = 0; k < kChunk / 32; ++k) {
    const int pp = c * kChunk + k * 32 + lane;
    if (pp < total) {
      while (pp >= off[rr + 1])
        ++rr;
      cp_async16(&ring[c % kRing][k * 32 + lane], &rec[qa[rr] + (pp - off[rr])]);
    }
  }
  cp_async_commit();
}

// One streamed chunk through masks: each lane marks the records of the chunk
// that are in range and in its own search box (`acc`: a warp streaming the
// union of its lanes' boxes passes each lane the positions of its own box;
// all ones when the boxes are equal), then adds its marked records lowest
// first: the same additions in the same order as density_add_packed. For the
// kernels with an exponential this also evaluates the kernel only on the
// records the lane takes: the lanes of a warp seldom have the same candidates
// in range, and a kernel evaluated inside the candidate loop would run
// whenever any lane is in range.
template <int D, int KIND>
__device__ __forceinline__ void density_chunk_masked(const RunParams& p, unsigned long long xi_xy,
                                                     float zi, const ulonglong2* chunk, int cnt,
                                                     unsigned acc, int jself, float wi,
                                                     float& rho) {
  static_assert(kChunk == 32, "one mask bit per record of a chunk");
  if (acc == 0)
    return;
  unsigned m = 0;
  if (cnt == kChunk) {
#pragma unroll 8
    for (int j = 0; j < kChunk; ++j) {
      float v;
      if (packed_d2<D>(xi_xy, zi, chunk[j], v) <= p.dc2)
        m |= 1u << j;
    }
  } else {
    for (int j = 0; j < cnt; ++j) {
      float v;
      if (packed_d2<D>(xi_xy, zi, chunk[j], v) <= p.dc2)
        m |= 1u << j;
    }
  }
  m &= acc;
  while (m) {
    const int j = __ffs(m) - 1;
    m &= m - 1;
    float v;
    const float d2 = packed_d2<D>(xi_xy, zi, chunk[j], v);
    if (KIND == CLUE_KERNEL_FLAT) {
      rho = __fadd_rn(rho, j == jself ? wi : v);
    } else {
      const float k = kernel_value_in_range(p, __fsqrt_rn(d2), j == jself);
      rho = __fadd_rn(rho, __fmul_rn(k, v));
    }
  }
}

// Bits [lo, hi) of a 32-bit mask, 0 <= lo < hi <= 32.
__device__ __forceinline__ unsigned range_bits(int lo, int hi) {
  return (hi - lo == 32 ? 0xffffffffu : ((1u << (hi - lo)) - 1u)) << lo;
}

// ---------------------------------------------------------------------------
// Exact-sum density (flat kernel; event_sums_exact in common.cuh). For an
// event whose sums are exact in any order, a warp streams only the cells
// within reach of its 32 points, and each lane adds its in-range candidates
// from its own box's tiles, the same candidate set as the reference's.
// ---------------------------------------------------------------------------

constexpr int kMaxSegs = 64;        // cell-row segments an exact-sum warp streams (2 per lane)
constexpr int kMaxUnionTiles = 32;  // tiles of the warp's union box (one per lane)
constexpr int kMaxStream = kMaxSegs > kMaxRows ? kMaxSegs : kMaxRows;

// One warp, exact-sum event. Returns false (nothing done) when the warp's
// reach needs more than kMaxSegs segments or kMaxUnionTiles tiles; the caller
// then takes the ordered stream. Warp-uniform: every lane calls it.
template <int D>
__device__ bool density_exact(const RunParams& p, const SweepArgs& a, const EventDesc& ev,
                              const GridDesc& g, const float* xi, int s, float wi, const int* inf,
                              const int* sup, bool ordered, const int* uinf, const int* usup,
                              float4 (*ring)[kChunk], int* off, int* qa, int* seg,
                              float& rho, int& tested) {
  const int lane = threadIdx.x & 31;
  int nu[D];
  int64_t n_union = 1;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    nu[d] = usup[d] - uinf[d] + 1;
    n_union *= nu[d];
  }
  if (n_union > kMaxUnionTiles)
    return false;
  // bounding box of the warp's points, widened by the reach of dc: every
  // candidate in range of a lane lies in a cell that meets it
  const float R = reach(p.dc2);
  float qlo[D], qhi[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    float lo = xi[d], hi = xi[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(kFullMask, lo, o));
      hi = fmaxf(hi, __shfl_xor_sync(kFullMask, hi, o));
    }
    qlo[d] = __fsub_rd(lo, R);
    qhi[d] = __fadd_ru(hi, R);
  }
  // lane t < n_union: tile t of the union box (last dimension fastest) and
  // its rows of cells within reach
  int rows_t = 0, tb = 0, ts = 1;
  int clo[D], chi[D];
#pragma unroll
  for (int d = 0; d < D; ++d)
    clo[d] = chi[d] = 0;
  if (lane < n_union) {
    int rem = lane, tile = ev.tile_base;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      tile += (uinf[d] + rem % nu[d]) * g.stride[d];
      rem /= nu[d];
    }
    tb = a.tile_offset[tile];
    if (a.tile_offset[tile + 1] > tb) {
      ts = a.cell_s[tile];
      float glo[D], ginv[D];
      load_geom<D>(a, tile, glo, ginv);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        clo[d] = cell_coord(qlo[d], glo[d], ginv[d], ts);
        chi[d] = cell_coord(qhi[d], glo[d], ginv[d], ts);
      }
      rows_t = (chi[0] - clo[0] + 1) * (D == 3 ? chi[1] - clo[1] + 1 : 1);
    }
  }
  // tiles of the union box inside this lane's box, as a mask over union tiles
  uint32_t tmask = 0;
  if (ordered) {
    if (D == 2) {
      const uint32_t row = (uint32_t)((1ull << (sup[1] - inf[1] + 1)) - 1) << (inf[1] - uinf[1]);
      for (int b0 = inf[0]; b0 <= sup[0]; ++b0)
        tmask |= row << ((b0 - uinf[0]) * nu[1]);
    } else {
      const uint32_t row = (uint32_t)((1ull << (sup[2] - inf[2] + 1)) - 1) << (inf[2] - uinf[2]);
      for (int b0 = inf[0]; b0 <= sup[0]; ++b0)
        for (int b1 = inf[1]; b1 <= sup[1]; ++b1)
          tmask |= row << (((b0 - uinf[0]) * nu[1] + (b1 - uinf[1])) * nu[2]);
    }
  }
  const uint32_t all_tiles = (uint32_t)((1ull << n_union) - 1);
  // The tiles in every lane's box stream first (any order sums exactly here):
  // every lane takes all their records, with no per-lane test.
  const uint32_t common = __reduce_and_sync(kFullMask, tmask) & all_tiles;
  const bool is_common = (common >> lane) & 1u;
  int incl_c = is_common ? rows_t : 0, incl_o = is_common ? 0 : rows_t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int yc = __shfl_up_sync(kFullMask, incl_c, o);
    const int yo = __shfl_up_sync(kFullMask, incl_o, o);
    if (lane >= o) {
      incl_c += yc;
      incl_o += yo;
    }
  }
  const int K_common = __shfl_sync(kFullMask, incl_c, 31);
  const int K = K_common + __shfl_sync(kFullMask, incl_o, 31);
  if (K > kMaxSegs)
    return false;
  const int first = is_common ? incl_c - rows_t : K_common + incl_o - rows_t;
  const int n1c = D == 3 ? chi[1] - clo[1] + 1 : 1;
  if (lane < n_union) {
    for (int r = 0; r < rows_t; ++r) {
      const int c0 = clo[0] + r / n1c;
      const int row_cell = D == 2 ? c0 * ts : (c0 * ts + clo[1] + r % n1c) * ts;
      const int q0 = a.cell_info[tb + row_cell + clo[D - 1]].start;
      off[first + r] = a.cell_info[tb + row_cell + chi[D - 1]].end - q0;  // length for now
      qa[first + r] = q0;
      seg[first + r] = lane;
    }
  }
  __syncwarp();
  // stream offsets of the segments
  const int l0 = 2 * lane < K ? off[2 * lane] : 0;
  const int l1 = 2 * lane + 1 < K ? off[2 * lane + 1] : 0;
  int run = l0 + l1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFullMask, run, o);
    if (lane >= o)
      run += y;
  }
  const int total = __shfl_sync(kFullMask, run, 31);
  tested = total;
  __syncwarp();
  if (2 * lane < K)
    off[2 * lane] = run - l0 - l1;
  if (2 * lane + 1 < K)
    off[2 * lane + 1] = run - l1;
  if (lane == 0)
    off[K] = total;
  __syncwarp();
  const int p_common = off[K_common];  // stream positions [0, p_common): common tiles
  // Whether the point's own record is among its candidates: a finite point
  // inside its own box (its cell is within reach of the warp's points and its
  // tile is in the union); a point with a non-finite coordinate has nothing in
  // range, itself included.
  bool self_in = ordered;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int own = get_bin(g, p, xi[d], d);
    self_in &= inf[d] <= own && own <= sup[d] && isfinite(xi[d]);
  }
  // cursor over this lane's accepted segments past the common ones: [ilo,
  // ihi) in stream positions
  int kc = K_common, ilo = INT_MAX, ihi = INT_MAX;
  auto next_accepted = [&]() {
    while (kc < K && !((tmask >> seg[kc]) & 1u))
      ++kc;
    if (kc < K) {
      ilo = off[kc];
      ihi = off[kc + 1];
      ++kc;
    } else {
      ilo = ihi = INT_MAX;
    }
  };
  const bool take_all = tmask == all_tiles;
  if (!take_all)
    next_accepted();
  const int chunks = (total + kChunk - 1) / kChunk;
  const unsigned long long xi_xy = pack2(xi[0], xi[1]);
  const float4* __restrict__ rec = a.rec_cell;
  int rr = 0;
#pragma unroll
  for (int c = 0; c < kRing - 1; ++c)
    stream_issue(ring, off, qa, rec, c, lane, total, rr);
  for (int c = 0; c < chunks; ++c) {
    stream_issue(ring, off, qa, rec, c + kRing - 1, lane, total, rr);
    cp_async_wait<kRing - 1>();
    __syncwarp();
    const ulonglong2* chunk = reinterpret_cast<const ulonglong2*>(ring[c % kRing]);
    const int base = c * kChunk;
    const int cnt = min(kChunk, total - base);
    unsigned acc = 0xffffffffu;
    if (!take_all && base + cnt > p_common) {
      const int cend = base + cnt;
      acc = base < p_common ? range_bits(0, p_common - base) : 0u;
      while (ilo < cend) {
        const int lo = max(ilo, base), hi = min(ihi, cend);
        if (lo < hi)
          acc |= range_bits(lo - base, hi - base);
        if (ihi > cend)
          break;
        next_accepted();
      }
    }
    // Any order is exact here. Every record in range adds its v_j, the
    // point's own record included; the own term is corrected once at the end.
    if (cnt == kChunk && __all_sync(kFullMask, acc == 0xffffffffu)) {
      // two running sums (exact, so their split and final sum change
      // nothing): measured 3 % faster than one
      float rho_b = 0.0f;
#pragma unroll 8
      for (int j = 0; j < kChunk; j += 2) {
        float v, v1;
        const float d2 = packed_d2<D>(xi_xy, xi[2], chunk[j], v);
        const float d2b = packed_d2<D>(xi_xy, xi[2], chunk[j + 1], v1);
        if (d2 <= p.dc2)
          rho = __fadd_rn(rho, v);
        if (d2b <= p.dc2)
          rho_b = __fadd_rn(rho_b, v1);
      }
      rho = __fadd_rn(rho, rho_b);
    } else {
      for (int j = 0; j < cnt; ++j) {
        float v;
        const float d2 = packed_d2<D>(xi_xy, xi[2], chunk[j], v);
        if (((acc >> j) & 1u) && d2 <= p.dc2)
          rho = __fadd_rn(rho, v);
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();
  __syncwarp();
  // The own record (d2 = 0, in range) added v_i = fl(flat * w_i) where the
  // reference adds w_i: (rho - v_i) + w_i, both steps exact (multiples of u,
  // between 0 and the event bound).
  if (self_in)
    rho = __fadd_rn(__fsub_rn(rho, __fmul_rn(p.kernel_p0, wi)), wi);
  return true;
}

// Local density, one point per lane. When the 32 lanes of a warp share one
// search box (the work order groups each tile's points by box), the warp
// streams the box's candidate records through a shared-memory ring of kRing
// chunks of kChunk records, copied asynchronously kRing - 1 chunks ahead; every
// lane reads each record from shared memory. The stream is the box's rows in
// order, each a contiguous range of sorted positions, i.e. the reference's
// summation order. Other warps read candidates from global memory.
template <int D, int KIND, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_density_fast(const RunParams p, const SweepArgs a) {
  __shared__ __align__(16) float4 s_ring[NT / 32][kRing][kChunk];
  __shared__ int s_off[NT / 32][kMaxStream + 1];
  __shared__ int s_qa[NT / 32][kMaxStream];
  __shared__ int s_seg[NT / 32][kMaxSegs];
  const int64_t n = a.n;
  const float4* __restrict__ rec = a.rec_dens;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4(*ring)[kChunk] = s_ring[warp];
  int* off = s_off[warp];
  int* qa = s_qa[warp];
  const int64_t n_items = (n + 31) / 32;
  for (;;) {
    // next item of 32 work positions: warps of light boxes take more items
    int64_t item = 0;
    if (lane == 0)
      item = atomicAdd(reinterpret_cast<unsigned*>(&a.queue[0]), 1u);
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= n_items)
      break;
    const int64_t w = item * 32 + lane;
    const bool active = w < n;
    int s = active ? a.work_dens[w] : 0;
    // idle lanes shadow lane 0 (the shuffle runs on every lane: a full-mask
    // shuffle that only some lanes reach never completes)
    const int s_lane0 = __shfl_sync(kFullMask, s, 0);
    s = active ? s : s_lane0;
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    const float4 ri = rec[s];
    const float xi[3] = {ri.x, ri.y, ri.z};
    const float zero[3] = {0.0f, 0.0f, 0.0f};
    const float wi = a.sw[s];
    int inf[D], sup[D];
    search_box<D>(g, p, xi, zero, p.dc, inf, sup);
    bool ordered = true;
#pragma unroll
    for (int d = 0; d < D; ++d)
      ordered &= inf[d] <= sup[d];
    // The warp's stream is the union U of its lanes' boxes (lanes of one event
    // grid only). Each lane's box is a sub-box of U, and the reference's order
    // over U restricted to a sub-box is the sub-box's own order, so every lane
    // takes its own candidates from the shared stream in its own order.
    const bool one_grid =
        __all_sync(kFullMask, __shfl_sync(kFullMask, ev.tile_base, 0) == ev.tile_base);
    int uinf[D], usup[D];
    bool same = ordered, u_ordered = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      uinf[d] = __reduce_min_sync(kFullMask, ordered ? inf[d] : INT_MAX);
      usup[d] = __reduce_max_sync(kFullMask, ordered ? sup[d] : INT_MIN);
      same &= (inf[d] == uinf[d]) & (sup[d] == usup[d]);
      u_ordered &= uinf[d] <= usup[d];
    }
    const bool uniform = __all_sync(kFullMask, same);
    const int64_t n1 = (D == 3 && u_ordered) ? (int64_t)usup[1] - uinf[1] + 1 : 1;
    const int64_t rows64 = u_ordered ? ((int64_t)usup[0] - uinf[0] + 1) * n1 : 0;
    // U-row index of (b0, b1) (row table in off/qa) and this lane's part of
    // that row as stream positions
    auto u_row = [&](int b0, int b1) {
      return (b0 - uinf[0]) * (int)n1 + (D == 3 ? b1 - uinf[1] : 0);
    };
    auto lane_part = [&](int b0, int b1, int& lo, int& hi) {
      const int r = u_row(b0, b1);
      int row = ev.tile_base + b0 * g.stride[0];
      if (D == 3)
        row += b1 * g.stride[1];
      lo = off[r] + (a.tile_offset[row + inf[D - 1]] - qa[r]);
      hi = off[r] + (a.tile_offset[row + sup[D - 1] + 1] - qa[r]);
    };
    float rho = 0.0f;
    // events whose sums are exact in any order stream only the cells in reach
    const bool exact = KIND == CLUE_KERNEL_FLAT && a.rec_cell != nullptr && one_grid && u_ordered &&
                       __all_sync(kFullMask, event_sums_exact(a.event_exact, a.sevt[s], ev.n));
    bool done = false;  // warp-uniform: the exact-sum path handled the warp
    int tested = 0;     // candidate records this lane tests
    if (exact)
      done = density_exact<D>(p, a, ev, g, xi, s, wi, inf, sup, ordered, uinf, usup, ring, off, qa,
                              s_seg[warp], rho, tested);
    bool streamed = false;  // warp-uniform: the ordered stream handles the warp
    if (!done && one_grid && rows64 >= 1 && rows64 <= kMaxRows) {
      const int rows = (int)rows64;
      // row table: lane r holds row r of U
      int len = 0, start = 0;
      if (lane < rows) {
        const int b0 = uinf[0] + lane / (int)n1;
        int row = ev.tile_base + b0 * g.stride[0];
        if (D == 3)
          row += (uinf[1] + lane % (int)n1) * g.stride[1];
        start = a.tile_offset[row + uinf[D - 1]];
        len = a.tile_offset[row + usup[D - 1] + 1] - start;
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= o)
          incl += y;
      }
      const int total = __shfl_sync(kFullMask, incl, 31);
      if (lane < rows) {
        off[lane] = incl - len;
        qa[lane] = start;
      }
      if (lane == 0)
        off[rows] = total;
      __syncwarp();
      // Lanes with different boxes: every lane pays for the whole union, so
      // the union is streamed only while it is not much larger than the
      // largest own box; otherwise each lane reads its own candidates below.
      if (!uniform) {
        int own_len = 0;
        if (ordered)
          for (int b0 = inf[0]; b0 <= sup[0]; ++b0)
            for (int b1 = D == 3 ? inf[1] : 0; b1 <= (D == 3 ? sup[1] : 0); ++b1) {
              int lo, hi;
              lane_part(b0, b1, lo, hi);
              own_len += hi - lo;
            }
        const int max_own = __reduce_max_sync(kFullMask, own_len);
        streamed = (int64_t)total * 16 <= (int64_t)p.union_x16 * max_own;
      } else {
        streamed = true;
      }
    }
    if (streamed) {
      const int rows = (int)rows64;
      const int total = off[rows];
      tested = total;
      // stream position of the point itself (its own tile is in the box unless
      // get_bin's clamping left it out)
      int p_self = -1;
      {
        int own[D];
        bool in = ordered;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          own[d] = get_bin(g, p, xi[d], d);
          in &= inf[d] <= own[d] && own[d] <= sup[d];
        }
        if (in) {
          const int r = u_row(own[0], D == 3 ? own[1] : 0);
          p_self = off[r] + (s - qa[r]);
        }
      }
      // cursor over this lane's rows of U (last dimension excluded): the
      // current row (cb0, cb1) and its stream positions [ilo, ihi)
      int cb0 = inf[0], cb1 = D == 3 ? inf[1] : 0, ilo = INT_MAX, ihi = INT_MAX;
      if (!uniform && ordered)
        lane_part(cb0, cb1, ilo, ihi);
      const int chunks = (total + kChunk - 1) / kChunk;
      const unsigned long long xi_xy = pack2(xi[0], xi[1]);
      int rr = 0;  // row cursor of this lane's copies
#pragma unroll
      for (int c = 0; c < kRing - 1; ++c)
        stream_issue(ring, off, qa, rec, c, lane, total, rr);
      for (int c = 0; c < chunks; ++c) {
        stream_issue(ring, off, qa, rec, c + kRing - 1, lane, total, rr);
        cp_async_wait<kRing - 1>();
        __syncwarp();
        const ulonglong2* chunk = reinterpret_cast<const ulonglong2*>(ring[c % kRing]);
        const int base = c * kChunk;
        const int cnt = min(kChunk, total - base);
        const int jself = p_self - base;  // own record's place in this chunk, if any
        if (uniform) {
          if (KIND != CLUE_KERNEL_FLAT) {
            density_chunk_masked<D, KIND>(p, xi_xy, xi[2], chunk, cnt, 0xffffffffu, jself, wi, rho);
          } else if (cnt == kChunk) {
#pragma unroll 8
            for (int j = 0; j < kChunk; ++j)
              density_add_packed<D, KIND>(p, xi_xy, xi[2], chunk[j], j == jself, wi, rho);
          } else {
            for (int j = 0; j < cnt; ++j)
              density_add_packed<D, KIND>(p, xi_xy, xi[2], chunk[j], j == jself, wi, rho);
          }
        } else {
          // positions of this chunk inside this lane's box
          const int cend = base + cnt;
          unsigned acc = 0;
          while (ilo < cend) {
            const int lo = max(ilo, base), hi = min(ihi, cend);
            if (lo < hi)
              acc |= range_bits(lo - base, hi - base);
            if (ihi > cend)
              break;  // the row goes on in the next chunk
            // next row of this lane's box
            if (D == 3 && cb1 < sup[1]) {
              ++cb1;
            } else {
              cb1 = D == 3 ? inf[1] : 0;
              ++cb0;
            }
            if (cb0 > sup[0]) {
              ilo = ihi = INT_MAX;
              break;
            }
            lane_part(cb0, cb1, ilo, ihi);
          }
          density_chunk_masked<D, KIND>(p, xi_xy, xi[2], chunk, cnt, acc, jself, wi, rho);
        }
        __syncwarp();
      }
      cp_async_wait<0>();
      __syncwarp();
    }
    if (!streamed && !done)
      for_each_candidate<D>(a, g, ev.tile_base, inf, sup, [&](int q) {
        density_add<D, KIND>(p, xi, __ldg(&rec[q]), q == s, wi, rho);
        ++tested;
      });
    if (a.stats) {  // warp-uniform
      const int sum = __reduce_add_sync(kFullMask, active ? tested : 0);
      if (lane == 0) {
        atomicAdd(&a.stats[0], (unsigned long long)sum);
        atomicAdd(&a.stats[1], 1ull);
      }
    }
    if (!active)
      continue;
    a.srho[s] = rho;
    const int gi = a.perm[s];
    if (a.out_rho)
      a.out_rho[gi] = rho;
    const uint32_t tag = p.has_tags ? a.stag[s] : (uint32_t)gi;
    const uint32_t kbits = rho_key(rho);
    const float key = __uint_as_float(kbits);
    int pos = s;
    if (a.nh_cells) {
      pos = a.nh_pos[s];
      atomicMax(&a.cell_info[a.cell_slot[s]].maxkey, ((unsigned long long)kbits << 32) | tag);
    }
    if (D == 2) {
      a.rec_nh[pos] = make_float4(xi[0], xi[1], key, __uint_as_float(tag));
    } else {
      a.rec_nh[pos] = make_float4(xi[0], xi[1], xi[2], key);
      a.rec_tag[pos] = tag;
    }
  }
}

__device__ __forceinline__ float next_up(float x) {  // x >= 0, finite
  return __uint_as_float(__float_as_uint(x) + 1u);
}
__device__ __forceinline__ float next_down(float x) {  // x >= 0; next_down(0) = -denorm_min
  return x > 0.0f ? __uint_as_float(__float_as_uint(x) - 1u) : __uint_as_float(0x80000001u);
}

// Squared distances that bracket the rounding class of `delta` (a correctly
// rounded square root): every d2 <= lo has sqrt_rn(d2) < delta and every
// d2 >= hi has sqrt_rn(d2) > delta. With a = the float below delta,
// lo = next_down(fl(a*a)) <= a^2 and, with b = the float above, hi =
// next_up(fl(b*b)) >= b^2; sqrt_rn is monotone, which gives both claims.
__device__ __forceinline__ void bracket(float delta, float& lo, float& hi) {
  const float a = next_down(delta);
  lo = next_down(__fmul_rn(a, a));
  const float b = next_up(delta);
  const float bb = __fmul_rn(b, b);
  hi = isinf(bb) ? bb : next_up(bb);
}

// Best candidate of a nearest-higher search: its squared distance d2b, key and
// position, and a bracket (lo, hi) around d2b: every d2 <= lo has
// sqrt_rn(d2) < sqrt_rn(d2b) and every d2 >= hi has sqrt_rn(d2) > sqrt_rn(d2b).
struct NhBest {
  float d2b, lo, hi;
  int best;
  uint64_t key_b;
};

__device__ __forceinline__ NhBest nh_none() {
  const float inf = __int_as_float(0x7f800000);
  return NhBest{inf, inf, inf, -1, 0ull};  // no best yet: every eligible candidate wins
}

// For d2b >= 2^-100 the bracket is d2b * (1 -+ 2^-20): with round-to-nearest
// errors of at most 2^-24 in the product and in sqrt_rn, d2 <= fl(d2b (1 - 2^-20))
// gives sqrt_rn(d2) <= sqrt(d2b)(1 - 6.5 * 2^-24) < sqrt_rn(d2b), and
// symmetrically above (an overflowing hi is +inf, which only sends more
// candidates to the exact comparison). Smaller d2b (0 for coincident points)
// takes the exact rounding class of sqrt_rn(d2b).
__device__ __forceinline__ void nh_take(NhBest& st, float d2, int q, uint64_t key) {
  st.d2b = d2;
  st.best = q;
  st.key_b = key;
  if (d2 >= 0x1p-100f) {
    st.lo = __fmul_rn(d2, 0.99999904632568359375f);   // 1 - 2^-20
    st.hi = __fmul_rn(d2, 1.00000095367431640625f);   // 1 + 2^-20
  } else {
    bracket(__fsqrt_rn(d2), st.lo, st.hi);
  }
}

// ClusteringKernels.hpp:195-202 for one eligible candidate (higher key, d2 <=
// eff2): it wins when its distance is smaller, or equal with a larger key.
// Only squared distances inside the bracket take the exact square roots.
__device__ __forceinline__ void nh_consider(NhBest& st, float d2, int q, uint64_t key) {
  if (d2 <= st.lo) {
    nh_take(st, d2, q, key);
  } else if (d2 < st.hi) {
    const float dist = __fsqrt_rn(d2), delta = __fsqrt_rn(st.d2b);
    if ((dist < delta) || ((dist == delta) && (key > st.key_b)))
      nh_take(st, d2, q, key);
  }
}

// Nearest higher with (density, tag) as one ordered 64-bit key and distances
// compared as squared distances. A candidate j of point i is eligible when it is
// "higher" (key_j > key_i, which is rho_j > rho_i, or equal densities above zero
// and tag_j > tag_i) and sqrt(d2) <= the effective distance (d2 <= eff2). Against
// the current best (distance delta) it wins when sqrt(d2) < delta, or when
// sqrt(d2) == delta and key_j > key_best (ClusteringKernels.hpp:195-202). The
// bracket decides all but the candidates whose squared distance falls in
// (lo, hi); those take the exact square root.
template <int D>
__global__ void __launch_bounds__(kThreads, 4) k_nearest_higher_fast(const RunParams p,
                                                                  const SweepArgs a) {
  const int64_t n = a.n;
  const float4* __restrict__ rec = a.rec_nh;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int s = a.work_nh[w];
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    const float4 ri = rec[s];
    const float xi[3] = {ri.x, ri.y, ri.z};
    const float zero[3] = {0.0f, 0.0f, 0.0f};
    const float rho_i = a.srho[s];
    const uint32_t tag_i = D == 2 ? __float_as_uint(ri.w) : a.rec_tag[s];
    const float unc = p.has_unc ? a.sunc[s] : 1.0f;
    const float min_density = __fmul_rn(p.rhoc, unc);
    const bool seedlike = rho_i >= min_density;  // ClusteringKernels.hpp:168
    const float eff2 = seedlike ? p.seed2 : p.dm2;
    // rho_j == rho_i && rho_j > 0 && tag_j > tag_i: with rho_i <= 0 (or NaN)
    // equal densities never count, so the tag part of the key is saturated.
    const bool nan_i = rho_i != rho_i;
    const uint64_t key_i =
        ((uint64_t)(nan_i ? 0xffffffffu : rho_key(rho_i)) << 32) |
        ((nan_i || !(rho_i > 0.0f)) ? 0xffffffffu : tag_i);
    int inf[D], sup[D];
    search_box<D>(g, p, xi, zero, p.dm, inf, sup);
    NhBest bs = nh_none();
    for_each_candidate<D>(a, g, ev.tile_base, inf, sup, [&](int q) {
      const float4 r = __ldg(&rec[q]);
      const uint32_t tag_j = D == 2 ? __float_as_uint(r.w) : __ldg(&a.rec_tag[q]);
      const uint64_t key_j = ((uint64_t)__float_as_uint(D == 2 ? r.z : r.w) << 32) | tag_j;
      const float d2 = sq_dist<D>(xi, r);
      if ((key_j > key_i) && (d2 <= eff2))
        nh_consider(bs, d2, q, key_j);
    });
    const int best = bs.best;
    const int gi = a.perm[s];
    const int nh = best >= 0 ? a.perm[best] : -1;
    a.out_nh[gi] = nh;
    a.parent[s] = best >= 0 ? best : s;
    const int seed = (nh == -1) && seedlike;
    a.seed_flag[gi] = seed;
    if (a.out_seed)
      a.out_seed[gi] = seed;
  }
}


// Exclusive scan of cnt[0..S) in place by one warp (any S).
__device__ void warp_scan_range(int* cnt, int S) {
  const int lane = threadIdx.x & 31;
  const int per = (S + 31) / 32;
  const int lo = min(lane * per, S), hi = min(lo + per, S);
  int sum = 0;
  for (int k = lo; k < hi; ++k)
    sum += cnt[k];
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o)
      incl += y;
  }
  int run = incl - sum;
  for (int k = lo; k < hi; ++k) {
    const int v = cnt[k];
    cnt[k] = run;
    run += v;
  }
}

__device__ __forceinline__ unsigned lane_mask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <int NT>
__device__ __forceinline__ void group_sync() {
  if (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}

// Walk order of a tile's cells: strips of kStripRows rows of cells, each
// strip column by column (3-D: z-slice by z-slice, each slice in strips), a
// bijection onto 0 .. s^D - 1. Consecutive cells form compact patches (about
// 4 x 4 cells for the 16 cells that hold 32 points on average).
constexpr int kStripRows = 4;
template <int D>
__device__ __forceinline__ int strip_position(int c, int s) {
  int c0, c1, z = 0;
  if (D == 2) {
    c0 = c / s;
    c1 = c - c0 * s;
  } else {
    z = c % s;
    const int c01 = c / s;
    c0 = c01 / s;
    c1 = c01 - c0 * s;
  }
  const int r0 = c0 - c0 % kStripRows;
  const int rows = min(kStripRows, s - r0);
  const int p2 = r0 * s + c1 * rows + (c0 - r0);
  return D == 2 ? p2 : z * s * s + p2;
}

// Cell layout of tile t by a group of NT threads (one warp, or the whole block
// for a large tile): cell of every point, the layout positions (a counting
// sort by cell inside the tile's range), cell ranges and member boxes, the
// walk order (strip_position) and the density sweep's work order for the
// tile. cnt and cnt2 hold s^D cell counters each, ccnt box_classes<D>() class
// counters.
template <int D, int NT>
__device__ void tile_cells(const RunParams& p, const SweepArgs& a, int64_t t, int* cnt, int* ccnt,
                           int* cnt2) {
  constexpr int E = box_classes<D>();
  const int tid = NT == 32 ? (threadIdx.x & 31) : (int)threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int64_t n = a.n;
  group_sync<NT>();  // the previous tile of this group is done with cnt/ccnt
  const int begin = a.tile_offset[t], end = a.tile_offset[t + 1];
  const int m = end - begin;
  if (m == 0)
    return;
  const EventDesc ev = a.events[a.sevt[begin]];
  const GridDesc& g = a.grids[ev.grid];
  const int s = cells_per_dim<D>(m, p.cell_points);
  float lo[D], inv[D];
  int own[D];
  {
    int local = (int)t - ev.tile_base;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      own[d] = local / g.stride[d];
      local -= own[d] * g.stride[d];
      cell_axis(g, own[d], s, d, lo[d], inv[d]);
    }
  }
  if (tid == 0) {
    a.cell_s[t] = s;
    if (D == 2) {
      a.cell_geom[t] = make_float4(lo[0], lo[1], inv[0], inv[1]);
    } else {
      a.cell_geom[2 * t] = make_float4(lo[0], lo[1], lo[D - 1], inv[0]);
      a.cell_geom[2 * t + 1] = make_float4(inv[1], inv[D - 1], 0.0f, 0.0f);
    }
  }
  const int S = D == 2 ? s * s : s * s * s;
  for (int c = tid; c < S; c += NT)
    cnt[c] = 0;
  for (int c = tid; c < E; c += NT)
    ccnt[c] = 0;
  group_sync<NT>();
  for (int i = tid; i < m; i += NT) {
    const int q = begin + i;
    int c = 0;
#pragma unroll
    for (int d = 0; d < D; ++d)
      c = c * s + cell_coord(a.sx[d * n + q], lo[d], inv[d], s);
    atomicAdd(&cnt[c], 1);
    a.cell_slot[q] = begin + c;
  }
  group_sync<NT>();
  if (tid < 32)
    warp_scan_range(cnt, S);
  group_sync<NT>();
  for (int c = tid; c < S; c += NT) {
    CellInfo ci;
    ci.start = begin + cnt[c];
    ci.end = begin + (c + 1 < S ? cnt[c + 1] : m);
    ci.maxkey = 0ull;
    a.cell_info[begin + c] = ci;
  }
  group_sync<NT>();
  for (int i = tid; i < m; i += NT) {
    const int q = begin + i;
    const int pos = begin + atomicAdd(&cnt[a.cell_slot[q] - begin], 1);
    a.nh_pos[q] = pos;
    a.nh_q[pos] = q;
    a.rec_cell[pos] = a.rec_dens[q];  // the density record in cell-layout order
  }
  group_sync<NT>();
  // Member boxes. A point with a NaN coordinate is never within reach and
  // is left out; a cell without other members gets an empty box (+inf, -inf).
  for (int c = tid; c < S; c += NT) {
    const int c_end = c + 1 < S ? cnt[c] : m;  // cursors now hold the cell ends
    const int c_begin = c > 0 ? cnt[c - 1] : 0;
    float mn[D], mx[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      mn[d] = INFINITY;
      mx[d] = -INFINITY;
    }
    for (int k = c_begin; k < c_end; ++k) {
      const int q = a.nh_q[begin + k];
      float x[D];
      bool ok = true;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        x[d] = a.sx[d * n + q];
        ok &= x[d] == x[d];
      }
      if (ok) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
          mn[d] = fminf(mn[d], x[d]);
          mx[d] = fmaxf(mx[d], x[d]);
        }
      }
    }
    if (D == 2) {
      a.cell_box[begin + c] = make_float4(mn[0], mn[1], mx[0], mx[1]);
    } else {
      a.cell_box[2 * (begin + c)] = make_float4(mn[0], mn[1], mn[D - 1], mx[0]);
      a.cell_box[2 * (begin + c) + 1] = make_float4(mx[1], mx[D - 1], 0.0f, 0.0f);
    }
  }
  // Walk order: the layout positions with the cells taken in strip order,
  // walk[begin + k] = layout position of the k-th point.
  for (int c = tid; c < S; c += NT) {
    const int c_end = c + 1 < S ? cnt[c] : m;  // cursors hold the cell ends
    const int c_begin = c > 0 ? cnt[c - 1] : 0;
    cnt2[strip_position<D>(c, s)] = c_end - c_begin;
  }
  group_sync<NT>();
  if (tid < 32)
    warp_scan_range(cnt2, S);
  group_sync<NT>();
  for (int i = tid; i < m; i += NT) {
    const int c = a.cell_slot[a.nh_q[begin + i]] - begin;
    const int c_begin = c > 0 ? cnt[c - 1] : 0;
    a.walk[begin + cnt2[strip_position<D>(c, s)] + (i - c_begin)] = begin + i;
  }
  group_sync<NT>();
  // Density work order: the tile's points grouped by search-box class (the
  // lanes of a warp share one box) and in walk order inside a class (they are
  // neighbours). A counting sort by class: rounds of 32 walk positions per
  // warp, grouped within a round by __match_any_sync; one warp keeps the walk
  // order inside a class, several warps interleave their rounds (any order
  // inside a class is correct: it only decides which lane computes which
  // point). The class only groups points, so it comes from boxes computed
  // with a multiplication by the inverse tile size instead of get_bin's
  // division (a point near a tile boundary may land in a neighbouring class);
  // the density sweep computes every box exactly.
  float inv_tile[D];
#pragma unroll
  for (int d = 0; d < D; ++d)
    inv_tile[d] = g.tile[d] > 0.0f ? 1.0f / g.tile[d] : 0.0f;
  for (int i = tid; i < m; i += NT) {
    const int q = a.nh_q[a.walk[begin + i]];
    int inf[D], sup[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const float x = a.sx[d * n + q];
      const float u0 = (x - p.dc - g.minv[d]) * inv_tile[d];
      const float u1 = (x + p.dc - g.minv[d]) * inv_tile[d];
      inf[d] = u0 >= 0.0f ? min((int)fminf(u0, (float)g.k), g.k - 1) : 0;  // NaN and below: 0
      sup[d] = u1 >= 0.0f ? min((int)fminf(u1, (float)g.k), g.k - 1) : 0;
    }
    const int c = box_class<D>(g, own, inf, sup);
    a.cls_dens[begin + i] = c;
    atomicAdd(&ccnt[c], 1);
  }
  group_sync<NT>();
  if (tid < 32)
    warp_scan_range(ccnt, E);
  group_sync<NT>();
  for (int base = 0; base < m; base += NT) {
    const int i = base + tid;
    const bool valid = i < m;
    const int c = valid ? a.cls_dens[begin + i] : -1;
    const unsigned grp = __match_any_sync(kFullMask, c);
    const int leader = __ffs(grp) - 1;
    int first = 0;
    if (valid && lane == leader)
      first = atomicAdd(&ccnt[c], __popc(grp));
    first = __shfl_sync(kFullMask, first, leader);
    if (valid)
      a.work_dens[begin + first + __popc(grp & lane_mask_lt())] = a.nh_q[a.walk[begin + i]];
  }
}

// Cell layouts of all tiles. Blocks [0, large_blocks) take the tiles of more
// than kLargeTilePoints points, which the tile sort listed, one block each, so
// a dense tile of thousands of points does not hold up the launch on one warp;
// they come first so that the heaviest tiles do not run as a tail. The other
// blocks give one warp to each smaller tile. The kernel waits on dependent
// loads, so it trades registers for resident blocks: in 2-D 6 blocks per SM
// (40 registers, 8 bytes spilled) took 2.2 ms of the 46.5 M-point batch
// against 2.7 ms at the compiler's 64 registers (4 blocks); the 3-D form keeps
// 4, where 5 spills more and measured slower.
constexpr int kWarpCellSlots = kLargeTilePoints;  // s^D <= m <= 256 (at least 1 point per cell)
template <int D>
__global__ void __launch_bounds__(kCellWarps * 32, D == 2 ? 6 : 4) k_cells(const RunParams p, const SweepArgs a,
                                                          int large_blocks) {
  constexpr int E = box_classes<D>();
  static_assert(kWarpCellSlots * kCellWarps <= kCellSlots, "warp counters fit the block's");
  __shared__ int s_cnt[kCellSlots];
  __shared__ int s_cnt2[kCellSlots];
  __shared__ int s_cls[kCellWarps][E];
  const int warp = threadIdx.x >> 5;
  if ((int)blockIdx.x >= large_blocks) {
    const int64_t wb = (int64_t)blockIdx.x - large_blocks;
    const int64_t stride = ((int64_t)gridDim.x - large_blocks) * kCellWarps;
    for (int64_t t = wb * kCellWarps + warp; t < a.n_tiles; t += stride) {
      if (a.tile_offset[t + 1] - a.tile_offset[t] > kLargeTilePoints)
        continue;
      tile_cells<D, 32>(p, a, t, s_cnt + warp * kWarpCellSlots, s_cls[warp],
                        s_cnt2 + warp * kWarpCellSlots);
    }
  } else {
    const int n_large = *a.large_count;
    for (int k = (int)blockIdx.x; k < n_large; k += large_blocks)
      tile_cells<D, kCellWarps * 32>(p, a, a.large_tiles[k], s_cnt, s_cls[0], s_cnt2);
  }
}

// Tests the members of one cell unless the cell is empty, holds no higher
// key, or its box is out of reach.
// `cnt` counts cells checked, cells entered and members tested (statistics).
template <int D, bool STATS>
__device__ __forceinline__ void visit_cell(const SweepArgs& a, int slot, const float* xi,
                                           uint64_t key_i, float eff2, NhBest& st, int* cnt) {
  if (STATS)
    ++cnt[0];
  const CellInfo ci = a.cell_info[slot];
  if (ci.start == ci.end || ci.maxkey <= key_i)
    return;
  float mn[D], mx[D];
  load_box<D>(a, slot, mn, mx);
  const float lb2 = box_lower_bound<D>(xi, mn, mx);
  if (lb2 > eff2 || lb2 >= st.hi)
    return;
  if (STATS) {
    ++cnt[1];
    cnt[2] += ci.end - ci.start;
  }
  const float4* __restrict__ rec = a.rec_nh;
#pragma unroll 4
  for (int q = ci.start; q < ci.end; ++q) {
    const float4 r = __ldg(&rec[q]);
    const uint32_t tag_j = D == 2 ? __float_as_uint(r.w) : __ldg(&a.rec_tag[q]);
    const uint64_t key_j = ((uint64_t)__float_as_uint(D == 2 ? r.z : r.w) << 32) | tag_j;
    const float d2 = sq_dist<D>(xi, r);
    if ((key_j > key_i) && (d2 <= eff2))
      nh_consider(st, d2, q, key_j);
  }
}

// Nearest higher over the cell layout. Thread w takes the w-th point of the
// walk order, so a warp holds neighbouring points. The own cell and its neighbours in the own
// tile come first, which usually fixes a small delta; then every tile of the
// reference's search box is visited, but only its cells that can hold a point
// within the current bound. The result is the eligible candidate of least
// distance, ties to the larger key (ClusteringKernels.hpp:195-202), as in
// k_nearest_higher_fast, over exactly the same candidates.
// The search is bound by the latency of its dependent loads (cell info, box,
// members), so the 2-D form trades registers for resident warps: 8 blocks of
// 256 threads per SM measured 8.3 ms on the 46.5 M-point batch against 9.4 ms
// at 5 and 10.8 ms at 4, small spills included. The 3-D form, with more state
// per lane, stays at 4.
// STATS: the profiling instantiation, which also counts the candidates tested
// (SweepArgs::stats); the counters cost registers, so timed runs go without.
template <int D, int NT, int MINB, bool STATS>
__global__ void __launch_bounds__(NT, MINB) k_nearest_higher_cells(const RunParams p, const SweepArgs a) {
  const int64_t n = a.n;
  const float4* __restrict__ rec = a.rec_nh;
  const int lane = threadIdx.x & 31;
  const int64_t n_items = (n + 31) / 32;
  for (;;) {
    // next item of 32 layout positions (work per point varies a lot: points
    // in dense cells test many more candidates)
    int64_t item = 0;
    if (lane == 0)
      item = atomicAdd(reinterpret_cast<unsigned*>(&a.queue[1]), 1u);
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= n_items)
      break;
    const int64_t w = item * 32 + lane;
    // lanes past the end shadow lane 0 (the warp-wide steps below need every
    // lane) and write nothing
    const bool active = w < n;
    const int pi = a.walk[active ? w : item * 32];  // neighbouring points in neighbouring lanes
    const int s = a.nh_q[pi];
    int cnt[3] = {0, 0, 0};  // cells checked, cells entered, members tested
    const float4 ri = rec[pi];
    const float xi[3] = {ri.x, ri.y, ri.z};
    const float zero[3] = {0.0f, 0.0f, 0.0f};
    const float rho_i = a.srho[s];
    const uint32_t tag_i = D == 2 ? __float_as_uint(ri.w) : a.rec_tag[pi];
    const float unc = p.has_unc ? a.sunc[s] : 1.0f;
    const float min_density = __fmul_rn(p.rhoc, unc);
    const bool seedlike = rho_i >= min_density;  // ClusteringKernels.hpp:168
    const float eff2 = seedlike ? p.seed2 : p.dm2;
    const bool nan_i = rho_i != rho_i;
    const uint64_t key_i =
        ((uint64_t)(nan_i ? 0xffffffffu : rho_key(rho_i)) << 32) |
        ((nan_i || !(rho_i > 0.0f)) ? 0xffffffffu : tag_i);
    const EventDesc ev = a.events[a.sevt[s]];
    const GridDesc& g = a.grids[ev.grid];
    int inf[D], sup[D], own[D];
    search_box<D>(g, p, xi, zero, p.dm, inf, sup);
#pragma unroll
    for (int d = 0; d < D; ++d)
      own[d] = get_bin(g, p, xi[d], d);
    const int t0 = tile_id<D>(g, p, ev.tile_base, own);

    // no best yet: every eligible candidate wins
    NhBest bs = nh_none();

    // Phase 0: the own cell and its neighbours in the own tile. Phase 1: every
    // tile of the search box, cells within reach only, less those of phase 0.
    // The own tile is skipped when the box leaves it out: get_bin sends a
    // coordinate beyond the int range to bin 0 (x86 conversion), so a huge
    // radius can give a box that misses the point's own tile.
    int c0[D], b[D];
    bool first = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      b[d] = inf[d];
      c0[d] = 0;
      first &= inf[d] <= own[d] && own[d] <= sup[d];
    }
    for (;;) {
      const int t = first ? t0 : tile_id<D>(g, p, ev.tile_base, b);
      const int base = a.tile_offset[t];
      if (a.tile_offset[t + 1] != base) {
        const int st = a.cell_s[t];
        float glo[D], ginv[D];
        load_geom<D>(a, t, glo, ginv);
        // |x_j - x_i| <= R for every member that can still win (d2 <= bound2)
        const float R = reach(fminf(eff2, bs.hi));
        int c_lo[D], c_hi[D], c[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          if (first) {
            c0[d] = cell_coord(xi[d], glo[d], ginv[d], st);
            c_lo[d] = c0[d] - 1;
            c_hi[d] = c0[d] + 1;
          } else {
            c_lo[d] = cell_coord(__fsub_rd(xi[d], R), glo[d], ginv[d], st);
            c_hi[d] = cell_coord(__fadd_ru(xi[d], R), glo[d], ginv[d], st);
          }
          c[d] = c_lo[d];
        }
        const bool own_tile = !first && t == t0;
        do {
          int lin = 0;
          bool seen = own_tile, valid = true;
#pragma unroll
          for (int d = 0; d < D; ++d) {
            int cd = c[d];
            if (first) {
              // offsets -1, 0, 1 visited as 0, 1, -1: the own cell comes
              // first and its nearest higher bounds the neighbours
              cd = c0[d] + (cd - c0[d] + 2) % 3 - 1;
              valid &= cd >= 0 && cd < st;
            }
            lin = lin * st + cd;
            seen &= abs(cd - c0[d]) <= 1;
          }
          if (valid && !seen)
            visit_cell<D, STATS>(a, base + lin, xi, key_i, eff2, bs, cnt);
        } while (next_tile<D>(c, c_lo, c_hi));
      }
      if (first)
        first = false;
      else if (!next_tile<D>(b, inf, sup))
        break;
    }

    if (STATS) {  // every lane gets here
      const int members = __reduce_add_sync(kFullMask, active ? cnt[2] : 0);
      const int checked = __reduce_add_sync(kFullMask, active ? cnt[0] : 0);
      const int entered = __reduce_add_sync(kFullMask, active ? cnt[1] : 0);
      if (lane == 0) {
        atomicAdd(&a.stats[2], (unsigned long long)members);
        atomicAdd(&a.stats[3], (unsigned long long)checked);
        atomicAdd(&a.stats[4], (unsigned long long)entered);
      }
    }
    if (!active)
      continue;
    const int gi = a.perm[s];
    const int qb = bs.best >= 0 ? a.nh_q[bs.best] : s;
    const int nh = bs.best >= 0 ? a.perm[qb] : -1;
    a.out_nh[gi] = nh;
    a.parent[s] = qb;
    const int seed = (nh == -1) && seedlike;
    a.seed_flag[gi] = seed;
    if (a.out_seed)
      a.out_seed[gi] = seed;
  }
}

}  // namespace

bool sweep_fast_path(const RunParams& p) {
  if ((p.D != 2 && p.D != 3) || p.metric_kind != CLUE_METRIC_EUCLIDEAN || p.has_sigma)
    return false;
  for (int d = 0; d < p.D; ++d)
    if (p.wrapped[d])
      return false;
  return true;
}

bool sweep_cells_path(const RunParams& p) { return sweep_fast_path(p) && !p.has_tags; }

#define CLUE_DISPATCH_D(D, KERNEL, ...)                \
  switch (D) {                                        \
    case 1: KERNEL<1><<<__VA_ARGS__>>>(p, a); break;  \
    case 2: KERNEL<2><<<__VA_ARGS__>>>(p, a); break;  \
    case 3: KERNEL<3><<<__VA_ARGS__>>>(p, a); break;  \
    case 4: KERNEL<4><<<__VA_ARGS__>>>(p, a); break;  \
    case 5: KERNEL<5><<<__VA_ARGS__>>>(p, a); break;  \
    case 6: KERNEL<6><<<__VA_ARGS__>>>(p, a); break;  \
    case 7: KERNEL<7><<<__VA_ARGS__>>>(p, a); break;  \
    case 8: KERNEL<8><<<__VA_ARGS__>>>(p, a); break;  \
    case 9: KERNEL<9><<<__VA_ARGS__>>>(p, a); break;  \
    case 10: KERNEL<10><<<__VA_ARGS__>>>(p, a); break; \
    default: return cudaErrorInvalidValue;            \
  }

cudaError_t launch_work_order(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  if (a.n == 0)
    return cudaSuccess;
  // With cells, k_cells writes the density work order; k_work_order is still
  // needed for the nearest-higher order when the cell search is off (tags).
  if (!a.nh_cells) {
    const int blocks = (int)std::min<int64_t>(a.n_tiles, (int64_t)sm_count() * 16);
    CLUE_DISPATCH_D(D, k_work_order, blocks, kThreads, 0, st)
    count_launches(1);
  }
  if (a.nh_pos) {
    const int warp_blocks =
        (int)std::max<int64_t>(1, std::min<int64_t>((a.n_tiles + kCellWarps - 1) / kCellWarps, (int64_t)sm_count() * 32));
    // blocks for the large tiles: at most one per tile that can be large
    const int large_blocks =
        (int)std::max<int64_t>(1, std::min<int64_t>(a.n / (kLargeTilePoints + 1), (int64_t)sm_count() * 24));
    if (D == 2)
      k_cells<2><<<large_blocks + warp_blocks, kCellWarps * 32, 0, st>>>(p, a, large_blocks);
    else
      k_cells<3><<<large_blocks + warp_blocks, kCellWarps * 32, 0, st>>>(p, a, large_blocks);
    count_launches(1);
  }
  return cudaGetLastError();
}

// Grid of a persistent sweep: enough blocks of nt threads to cover n points,
// at most `per_sm` per SM (the kernels take work items from a queue).
int sweep_grid(int64_t n, int nt, int per_sm) {
  const int64_t b = (n + nt - 1) / nt;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count() * per_sm));
}

// Block shapes of the density sweep (clue_tuning::density_shape):
// 0: 256 threads, 4 blocks per SM; 1: 128 threads, 8 per SM; 2: 256 threads, 3 per SM.
template <int D, int KIND>
void launch_density_kind(const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  switch (p.dens_shape) {
    case 1:
      k_density_fast<D, KIND, 128, 8><<<sweep_grid(a.n, 128, 32), 128, 0, st>>>(p, a);
      break;
    case 2:
      k_density_fast<D, KIND, 256, 3><<<sweep_grid(a.n, 256, 16), 256, 0, st>>>(p, a);
      break;
    default:
      k_density_fast<D, KIND, 256, 4><<<sweep_grid(a.n, 256, 16), 256, 0, st>>>(p, a);
      break;
  }
}

template <int D>
cudaError_t launch_density_fast(const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  count_launches(1);  // the density kernel below; k_gather wrote its records
  switch (p.kernel_kind) {
    case CLUE_KERNEL_FLAT:
      launch_density_kind<D, CLUE_KERNEL_FLAT>(p, a, st);
      break;
    case CLUE_KERNEL_GAUSSIAN:
      launch_density_kind<D, CLUE_KERNEL_GAUSSIAN>(p, a, st);
      break;
    default:
      launch_density_kind<D, CLUE_KERNEL_EXPONENTIAL>(p, a, st);
      break;
  }
  return cudaGetLastError();
}

// Block shapes of the nearest-higher cell search (clue_tuning::nh_shape):
// 0: 256 threads with 8 blocks per SM in 2-D, 4 in 3-D; 1: 256 threads, 6 per
// SM; 2: 128 threads with 16 blocks per SM in 2-D, 8 in 3-D.
template <int D, bool STATS>
void launch_nh_cells(const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  switch (p.nh_shape) {
    case 1:
      k_nearest_higher_cells<D, 256, 6, STATS><<<sweep_grid(a.n, 256, 16), 256, 0, st>>>(p, a);
      break;
    case 2:
      k_nearest_higher_cells<D, 128, D == 2 ? 16 : 8, STATS><<<sweep_grid(a.n, 128, 32), 128, 0, st>>>(p, a);
      break;
    default:
      k_nearest_higher_cells<D, 256, D == 2 ? 8 : 4, STATS><<<sweep_grid(a.n, 256, 16), 256, 0, st>>>(p, a);
      break;
  }
}

cudaError_t launch_density(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  if (a.n == 0)
    return cudaSuccess;
  if (sweep_fast_path(p))
    return D == 2 ? launch_density_fast<2>(p, a, st) : launch_density_fast<3>(p, a, st);
  CLUE_DISPATCH_D(D, k_density, grid_for(a.n), kThreads, 0, st)
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_nearest_higher(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st) {
  if (a.n == 0)
    return cudaSuccess;
  count_launches(1);  // one kernel on every path below
  if (a.nh_cells) {
    if (D == 2)
      a.stats ? launch_nh_cells<2, true>(p, a, st) : launch_nh_cells<2, false>(p, a, st);
    else
      a.stats ? launch_nh_cells<3, true>(p, a, st) : launch_nh_cells<3, false>(p, a, st);
    return cudaGetLastError();
  }
  if (sweep_fast_path(p)) {
    if (D == 2)
      k_nearest_higher_fast<2><<<grid_for(a.n), kThreads, 0, st>>>(p, a);
    else
      k_nearest_higher_fast<3><<<grid_for(a.n), kThreads, 0, st>>>(p, a);
    return cudaGetLastError();
  }
  CLUE_DISPATCH_D(D, k_nearest_higher, grid_for(a.n), kThreads, 0, st)
  return cudaGetLastError();
}

}  // namespace clue_impl
