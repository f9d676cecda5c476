// kernels.cu — the CUDA kernels of one clustering run and the launch sequence.
//
// Pipeline (all on one stream, no host round trip between stages):
//   grid extents  : per-grid min/max of the coordinates, tile size (max-min)/k
//   tile binning  : counting sort of point ids by tile — warp-aggregated
//                   histogram, single-pass decoupled-look-back scan, warp-
//                   aggregated scatter, then each tile's ids put in ascending
//                   order (the order the reference's serial fill produces)
//   gather        : tile-contiguous SoA copy of coordinates, weights, options
//   density sweep : rho per point, summed in the reference's exact order
//   NH sweep      : nearest higher, the reference's comparisons and tie-breaks
//   seeds/labels  : exclusive scan of the seed flags (seed k = k-th seed in
//                   index order gets cluster id k), roots by pointer jumping
//                   (per event in shared memory when every event has its own
//                   grid and at most 65,536 points; else over the whole run).
#include <atomic>
#include <cfloat>
#include <cuda/atomic>

#include "engine.h"
#include "sweep.cuh"

namespace clue_impl {

namespace {

constexpr int kThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kThreads * kScanItems;  // elements per scan block
constexpr int kSortCap = 4096;                    // tile sizes sorted in one shared-memory pass
constexpr int kSpinLimit = 1 << 21;               // bounded waits (~0.2 s) before flagging
constexpr unsigned kFull = 0xffffffffu;

struct CoordPtrs {
  const float* p[kMaxDim];
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T block_reduce(T v, T (*op)(T, T), T* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = op(v, __shfl_xor_sync(kFull, v, o));
  if (lane == 0)
    smem[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? smem[lane] : smem[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v = op(v, __shfl_xor_sync(kFull, v, o));
  }
  __syncthreads();
  return v;  // valid in warp 0
}

__device__ float fmin_op(float a, float b) { return fminf(a, b); }
__device__ float fmax_op(float a, float b) { return fmaxf(a, b); }

// ---------------------------------------------------------------------------
// Grid extents: core/detail/ComputeTiles.hpp:16-62, SetupTiles.hpp:19-96
// ---------------------------------------------------------------------------

__global__ void k_grid_init(int32_t* grid_minmax, int n_grids, int32_t* event_exact, int n_events) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_grids * kMaxDim) {
    grid_minmax[2 * i] = f2ord(FLT_MAX);       // min starts at numeric_limits::max()
    grid_minmax[2 * i + 1] = f2ord(-FLT_MAX);  // max starts at numeric_limits::lowest()
  }
  // exact-sum bounds (common.cuh), filled by k_bin
  if (event_exact && i < 4 * n_events)
    event_exact[i] = (i & 3) == 0 ? INT_MAX : 0;
}

// 2-D and 3-D: one pass over the chunk loads every coordinate of a point, and
// one shared-memory round reduces all 2 D extremes of the block.
template <int DD>
__device__ __forceinline__ void minmax_fixed(CoordPtrs x, const Chunk& c, int g, int32_t* grid_minmax) {
  __shared__ float red[2 * DD][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float mn[DD], mx[DD];
#pragma unroll
  for (int d = 0; d < DD; ++d) {
    mn[d] = FLT_MAX;
    mx[d] = -FLT_MAX;
  }
  for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) {
#pragma unroll
    for (int d = 0; d < DD; ++d) {
      const float v = x.p[d][i];
      if (v == v) {  // NaN never becomes an extreme
        mn[d] = fminf(mn[d], v);
        mx[d] = fmaxf(mx[d], v);
      }
    }
  }
#pragma unroll
  for (int d = 0; d < DD; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = fminf(mn[d], __shfl_xor_sync(kFull, mn[d], o));
      mx[d] = fmaxf(mx[d], __shfl_xor_sync(kFull, mx[d], o));
    }
    if (lane == 0) {
      red[2 * d][warp] = mn[d];
      red[2 * d + 1][warp] = mx[d];
    }
  }
  __syncthreads();
  if (warp == 0) {
    const bool in = lane < (int)(blockDim.x >> 5);
#pragma unroll
    for (int d = 0; d < DD; ++d) {
      float lo = in ? red[2 * d][lane] : FLT_MAX, hi = in ? red[2 * d + 1][lane] : -FLT_MAX;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(kFull, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(kFull, hi, o));
      }
      if (lane == 0) {
        atomicMin(&grid_minmax[2 * (g * kMaxDim + d)], f2ord(lo));
        atomicMax(&grid_minmax[2 * (g * kMaxDim + d) + 1], f2ord(hi));
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_minmax(int D, CoordPtrs x, const Chunk* chunks,
                                                     const EventDesc* events, int32_t* grid_minmax) {
  __shared__ float red[32];
  const Chunk c = chunks[blockIdx.x];
  const int g = events[c.event].grid;
  if (D == 2)
    return minmax_fixed<2>(x, c, g, grid_minmax);
  if (D == 3)
    return minmax_fixed<3>(x, c, g, grid_minmax);
  for (int d = 0; d < D; ++d) {
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int i = c.begin + threadIdx.x; i < c.end; i += blockDim.x) {
      const float v = x.p[d][i];
      if (v == v) {  // NaN never becomes an extreme
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
      }
    }
    mn = block_reduce(mn, fmin_op, red);
    mx = block_reduce(mx, fmax_op, red);
    if (threadIdx.x == 0) {
      atomicMin(&grid_minmax[2 * (g * kMaxDim + d)], f2ord(mn));
      atomicMax(&grid_minmax[2 * (g * kMaxDim + d) + 1], f2ord(mx));
    }
  }
}

__global__ void k_grid_finalize(int D, GridDesc* grids, int n_grids, const int32_t* grid_minmax) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_grids)
    return;
  for (int d = 0; d < D; ++d) {
    const float mn = ord2f(grid_minmax[2 * (g * kMaxDim + d)]);
    const float mx = ord2f(grid_minmax[2 * (g * kMaxDim + d) + 1]);
    grids[g].minv[d] = mn;
    grids[g].maxv[d] = mx;
    grids[g].tile[d] = __fdiv_rn(__fsub_rn(mx, mn), (float)grids[g].k);
  }
}

// ---------------------------------------------------------------------------
// Tile binning: data_structures/detail/AssociationMap.hpp:20-61 with
// Tiles::GetGlobalBin (Tiles.hpp:208-227, TilesView.hpp:54-64)
// ---------------------------------------------------------------------------

// Also the exact-sum bounds of the chunk's event (flat kernel, when
// event_exact is given): lowest-bit exponent, largest contributions, and a flag
// for a negative, -0, NaN or infinite weight, one atomic per warp.
__global__ void __launch_bounds__(kThreads) k_bin(RunParams p, CoordPtrs x, const Chunk* chunks,
                                                  const EventDesc* events, const GridDesc* grids,
                                                  int32_t* tile_of, int32_t* point_event,
                                                  int32_t* tile_count, const float* weight,
                                                  int32_t* event_exact) {
  __shared__ GridDesc sg;
  const Chunk c = chunks[blockIdx.x];
  const EventDesc ev = events[c.event];
  if (threadIdx.x == 0)
    sg = grids[ev.grid];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const bool bounds = event_exact && p.kernel_kind == CLUE_KERNEL_FLAT;  // block-uniform
  int lsb = INT_MAX, bad = 0;
  uint32_t vb = 0, wb = 0;
  // 2-D: the coordinates of four rounds are loaded ahead of their binning
  constexpr int U = 4;
  float px[U], py[U];
  for (int base = c.begin; base < c.end; base += blockDim.x) {
    const int k = ((base - c.begin) / (int)blockDim.x) % U;
    if (p.D == 2 && k == 0) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int iu = base + u * (int)blockDim.x + (int)threadIdx.x;
        px[u] = iu < c.end ? x.p[0][iu] : 0.0f;
        py[u] = iu < c.end ? x.p[1][iu] : 0.0f;
      }
    }
    const int i = base + threadIdx.x;
    const bool valid = i < c.end;
    int t = -1;
    if (valid) {
      int b = ev.tile_base;
      if (p.D == 2) {
        float vx = px[0], vy = py[0];
#pragma unroll
        for (int u = 1; u < U; ++u)
          if (k == u) {
            vx = px[u];
            vy = py[u];
          }
        b += sg.stride[0] * get_bin(sg, p, vx, 0) + sg.stride[1] * get_bin(sg, p, vy, 1);
      } else {
        for (int d = 0; d < p.D; ++d)
          b += sg.stride[d] * get_bin(sg, p, x.p[d][i], d);
      }
      t = b;
      tile_of[i] = t;
      point_event[i] = c.event;
      if (bounds) {
        const float w = weight[i];
        const float v = __fmul_rn(p.kernel_p0, w);  // a neighbour's fl(flat * w_j)
        const int bd = !(w >= 0.0f) || signbit(w) || isinf(w) || isinf(v);
        bad |= bd;
        if (!bd) {
          if (v > 0.0f)
            lsb = min(lsb, lsb_exponent(v));
          if (w > 0.0f)
            lsb = min(lsb, lsb_exponent(w));
          vb = max(vb, __float_as_uint(v));
          wb = max(wb, __float_as_uint(w));
        }
      }
    }
    const unsigned mask = __match_any_sync(kFull, t);
    const int leader = __ffs(mask) - 1;
    if (valid && lane == leader)
      atomicAdd(&tile_count[t], __popc(mask));
  }
  // the chunk's bounds, one set of atomics per block
  if (bounds) {
    __shared__ int s_b[4];
    if (threadIdx.x == 0) {
      s_b[0] = INT_MAX;
      s_b[1] = s_b[2] = s_b[3] = 0;
    }
    __syncthreads();
    lsb = __reduce_min_sync(kFull, lsb);
    vb = __reduce_max_sync(kFull, vb);
    wb = __reduce_max_sync(kFull, wb);
    bad = __any_sync(kFull, bad);
    if (lane == 0) {
      atomicMin(&s_b[0], lsb);
      atomicMax(reinterpret_cast<unsigned*>(&s_b[1]), vb);
      atomicMax(reinterpret_cast<unsigned*>(&s_b[2]), wb);
      atomicOr(&s_b[3], bad);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int32_t* st = event_exact + 4 * c.event;
      atomicMin(&st[0], s_b[0]);
      atomicMax(reinterpret_cast<unsigned*>(&st[1]), (unsigned)s_b[1]);
      atomicMax(reinterpret_cast<unsigned*>(&st[2]), (unsigned)s_b[2]);
      if (s_b[3])
        atomicOr(&st[3], 1);
    }
  }
}

// ---------------------------------------------------------------------------
// Stable tile binning: one warp per run of consecutive points of one event,
// runs of an event in index order. Binning counts each run's points per tile
// into the event's count matrix (runs x tiles, run-major); a pass per tile
// turns its column into exclusive prefixes over the runs and the tile's
// total; a scan of the totals gives the tile offsets; the scatter then places
// each run's points in index order from offset + prefix. Every tile thus
// lists its points in ascending index, the order the reference's serial fill
// produces (data_structures/detail/AssociationMap.hpp:63-81), with no sort.
// ---------------------------------------------------------------------------

// Event of stable-binning warp w: the last event whose first warp is <= w.
__device__ __forceinline__ int sort_event_of(const EventDesc* events, int n_events, int w) {
  int lo = 0, hi = n_events - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (events[mid].sort_first <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Tile ids and per-run tile counts; also the exact-sum bounds of the event
// (flat kernel, when event_exact is given), as in k_bin. s_col holds one
// counter per tile of the warp's event (max_tiles per warp).
__global__ void __launch_bounds__(kThreads) k_bin_stable(RunParams p, CoordPtrs x, const EventDesc* events,
                                                         int n_events, int n_warps, const GridDesc* grids,
                                                         int32_t* tile_of, int32_t* point_event,
                                                         int32_t* matrix, int max_tiles,
                                                         const float* weight, int32_t* event_exact,
                                                         int32_t* tile_event) {
  extern __shared__ int s_col[];
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= n_warps)
    return;  // whole warps only: nothing below synchronises the block
  int* col = s_col + (threadIdx.x >> 5) * max_tiles;
  const int e = sort_event_of(events, n_events, w);
  const EventDesc ev = events[e];
  const GridDesc& g = grids[ev.grid];
  const int c = w - ev.sort_first;
  const int T = g.T;
  for (int t = lane; t < T; t += 32)
    col[t] = 0;
  __syncwarp();
  const int begin = ev.begin + c * ev.sort_len;
  const int end = min(ev.begin + ev.n, begin + ev.sort_len);
  const bool bounds = event_exact && p.kernel_kind == CLUE_KERNEL_FLAT;
  int lsb = INT_MAX, bad = 0;
  uint32_t vb = 0, wb = 0;
#pragma unroll 4
  for (int base = begin; base < end; base += 32) {
    const int i = base + lane;
    const bool valid = i < end;
    int t = -1;
    if (valid) {
      int b = 0;
      for (int d = 0; d < p.D; ++d)
        b += g.stride[d] * get_bin(g, p, x.p[d][i], d);
      t = b;
      tile_of[i] = ev.tile_base + t;
      point_event[i] = e;
      if (bounds) {
        const float wt = weight[i];
        const float v = __fmul_rn(p.kernel_p0, wt);  // a neighbour's fl(flat * w_j)
        const int bd = !(wt >= 0.0f) || signbit(wt) || isinf(wt) || isinf(v);
        bad |= bd;
        if (!bd) {
          if (v > 0.0f)
            lsb = min(lsb, lsb_exponent(v));
          if (wt > 0.0f)
            lsb = min(lsb, lsb_exponent(wt));
          vb = max(vb, __float_as_uint(v));
          wb = max(wb, __float_as_uint(wt));
        }
      }
    }
    const unsigned mask = __match_any_sync(kFull, t);
    if (valid && lane == __ffs(mask) - 1)
      atomicAdd(&col[t], __popc(mask));  // ordered with later rounds' leaders, no barrier
  }
  __syncwarp();
  int32_t* row = matrix + (int64_t)ev.sort_base + (int64_t)c * T;
  if (c == 0)  // the event of each of its tiles, for the prefix pass
    for (int t = lane; t < T; t += 32)
      tile_event[ev.tile_base + t] = e;
  for (int t = lane; t < T; t += 32)
    row[t] = col[t];
  if (bounds) {
    lsb = __reduce_min_sync(kFull, lsb);
    vb = __reduce_max_sync(kFull, vb);
    wb = __reduce_max_sync(kFull, wb);
    bad = __any_sync(kFull, bad);
    if (lane == 0) {
      int32_t* st = event_exact + 4 * e;
      atomicMin(&st[0], lsb);
      atomicMax(reinterpret_cast<unsigned*>(&st[1]), vb);
      atomicMax(reinterpret_cast<unsigned*>(&st[2]), wb);
      if (bad)
        atomicOr(&st[3], 1);
    }
  }
}

// One thread per tile: the tile's counts over the runs of its event become
// exclusive prefixes (in place), and the total goes to tile_count. Threads of
// consecutive tiles read consecutive entries of each run's row.
__global__ void __launch_bounds__(kThreads) k_tile_prefix(const EventDesc* events, const GridDesc* grids,
                                                          int64_t n_tiles, const int32_t* tile_event,
                                                          int32_t* matrix, int32_t* tile_count) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_tiles;
       g += (int64_t)gridDim.x * blockDim.x) {
    const EventDesc ev = events[tile_event[g]];
    const int64_t T = grids[ev.grid].T;
    int32_t* m = matrix + (int64_t)ev.sort_base + (g - ev.tile_base);
    int run = 0;
#pragma unroll 8
    for (int c = 0; c < ev.sort_chunks; ++c) {
      const int v = m[c * T];
      m[c * T] = run;
      run += v;
    }
    tile_count[g] = run;
  }
}

// Places each run's points at tile offset + the run's prefix in that tile.
// The first run of each event lists the event's tiles of more than
// kLargeTilePoints points (for k_cells).
__global__ void __launch_bounds__(kThreads) k_scatter_stable(const EventDesc* events, int n_events,
                                                             int n_warps, const GridDesc* grids,
                                                             const int32_t* tile_of, const int32_t* matrix,
                                                             int max_tiles, const int32_t* tile_offset,
                                                             const int32_t* tile_count, int32_t* perm,
                                                             int32_t* large, int32_t* large_count) {
  extern __shared__ int s_col[];
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= n_warps)
    return;
  int* col = s_col + (threadIdx.x >> 5) * max_tiles;
  const int e = sort_event_of(events, n_events, w);
  const EventDesc ev = events[e];
  const int c = w - ev.sort_first;
  const int T = grids[ev.grid].T;
  const int32_t* row = matrix + (int64_t)ev.sort_base + (int64_t)c * T;
  for (int t = lane; t < T; t += 32) {
    col[t] = tile_offset[ev.tile_base + t] + row[t];
    if (c == 0 && tile_count[ev.tile_base + t] > kLargeTilePoints)
      large[atomicAdd(large_count, 1)] = ev.tile_base + t;
  }
  __syncwarp();
  const int begin = ev.begin + c * ev.sort_len;
  const int end = min(ev.begin + ev.n, begin + ev.sort_len);
  // Rounds of 32 points in index order; the next round's tile ids are loaded
  // before this round's cursor updates, so the load latency overlaps them.
  int t_next = begin + lane < end ? tile_of[begin + lane] - ev.tile_base : -1;
  for (int base = begin; base < end; base += 32) {
    const int i = base + lane;
    const bool valid = i < end;
    const int t = t_next;
    t_next = base + 32 + lane < end ? tile_of[base + 32 + lane] - ev.tile_base : -1;
    const unsigned mask = __match_any_sync(kFull, t);
    const int leader = __ffs(mask) - 1;
    int pos = 0;
    if (valid && lane == leader) {
      pos = col[t];
      col[t] = pos + __popc(mask);
    }
    pos = __shfl_sync(kFull, pos, leader);
    if (valid)
      perm[pos + __popc(mask & lanemask_lt())] = i;
    __syncwarp();  // the next round's leaders read these cursors
  }
}

// ---------------------------------------------------------------------------
// Single-pass exclusive scan with decoupled look-back.
// Each block takes a ticket (so every predecessor is already running), scans
// kScanTile elements, publishes its aggregate, then walks back over its
// predecessors' descriptors until it finds an inclusive prefix.
// ---------------------------------------------------------------------------

constexpr unsigned long long kFlagAggregate = 1ull << 62;
constexpr unsigned long long kFlagInclusive = 2ull << 62;
constexpr unsigned long long kValueMask = 0xffffffffull;

__device__ __forceinline__ void publish(unsigned long long* d, unsigned long long v) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*d);
  r.store(v, cuda::memory_order_release);
}
__device__ __forceinline__ unsigned long long peek(unsigned long long* d) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*d);
  return r.load(cuda::memory_order_acquire);
}

// Waits until descriptor d carries a flag, at most kSpinLimit polls; on giving
// up it records kStatusScanTimeout in the status word and returns an
// inclusive zero, so the scan finishes (with a wrong prefix the host then
// reports as CLUE_ERR_TIMEOUT) instead of hanging.
__device__ __forceinline__ unsigned long long await_descriptor(unsigned long long* d, uint32_t* status) {
  int spins = 0;
  unsigned long long dsc = peek(d);
  while ((dsc >> 62) == 0) {
    if (++spins > kSpinLimit) {
      atomicOr(status, kStatusScanTimeout);
      return kFlagInclusive;
    }
    __nanosleep(64);
    dsc = peek(d);
  }
  return dsc;
}

// Failure-detection self-test: the scan's wait on a descriptor nothing
// publishes must give up and flag it.
__global__ void k_wait_probe(unsigned long long* desc, uint32_t* status) {
  if (threadIdx.x == 0 && blockIdx.x == 0)
    (void)await_descriptor(desc, status);
}

// Clears and copies of a run are kernels rather than cudaMemsetAsync /
// cudaMemcpyAsync: a run then never waits in a copy engine's queue behind the
// point uploads of a pipelined host batch.
__global__ void k_fill32(uint32_t* p, int64_t n, uint32_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void k_copy32(uint32_t* dst, const uint32_t* src, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// Zeroes the scan's look-back descriptors and its block ticket.
__global__ void k_scan_reset(unsigned long long* desc, int blocks, int32_t* ticket) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < blocks; i += gridDim.x * blockDim.x)
    desc[i] = 0ull;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    *ticket = 0;
}

__global__ void __launch_bounds__(kThreads) k_scan(const int32_t* in, int32_t* out, int64_t n,
                                                   unsigned long long* desc, int32_t* ticket,
                                                   int32_t* total, uint32_t* status) {
  __shared__ int s_data[kScanTile + kScanTile / 32];
  __shared__ int s_warp[kThreads / 32];
  __shared__ int s_bid;
  __shared__ int s_prefix;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0)
    s_bid = atomicAdd(ticket, 1);
  __syncthreads();
  const int bid = s_bid;
  const int64_t base = (int64_t)bid * kScanTile;
  auto pad = [](int k) { return k + (k >> 5); };
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const int k = j * kThreads + tid;
    const int64_t g = base + k;
    s_data[pad(k)] = (g < n) ? in[g] : 0;
  }
  __syncthreads();
  int v[kScanItems];
  int sum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = s_data[pad(tid * kScanItems + j)];
    sum += v[j];
  }
  // inclusive scan of thread sums
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o)
      incl += y;
  }
  if (lane == 31)
    s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < kThreads / 32) ? s_warp[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, wi, o);
      if (lane >= o)
        wi += y;
    }
    if (lane < kThreads / 32)
      s_warp[lane] = wi - w;  // exclusive warp offsets
    const int aggregate = __shfl_sync(kFull, wi, kThreads / 32 - 1);
    // publish and look back
    int exclusive = 0;
    if (bid == 0) {
      if (lane == 0)
        publish(&desc[0], kFlagInclusive | (unsigned)aggregate);
    } else {
      if (lane == 0)
        publish(&desc[bid], kFlagAggregate | (unsigned)aggregate);
      int pred = bid - 1;
      bool done = false;
      while (!done) {
        const int idx = pred - lane;
        unsigned long long dsc = kFlagInclusive;  // lanes beyond block 0 contribute nothing
        if (idx >= 0)
          dsc = await_descriptor(&desc[idx], status);
        const bool inclusive = (dsc >> 62) == 2 || idx < 0;
        const unsigned ballot = __ballot_sync(kFull, inclusive);
        const int first = ballot ? (__ffs(ballot) - 1) : 32;  // nearest inclusive predecessor
        int val = (lane <= first && idx >= 0) ? (int)(dsc & kValueMask) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          val += __shfl_xor_sync(kFull, val, o);
        exclusive += val;
        if (ballot)
          done = true;
        else
          pred -= 32;
      }
      if (lane == 0)
        publish(&desc[bid], kFlagInclusive | (unsigned)(exclusive + aggregate));
    }
    if (lane == 0) {
      s_prefix = exclusive;
      if (base + kScanTile >= n)
        *total = exclusive + aggregate;
    }
  }
  __syncthreads();
  int run = s_prefix + s_warp[warp] + incl - sum;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    s_data[pad(tid * kScanItems + j)] = run;
    run += v[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const int k = j * kThreads + tid;
    const int64_t g = base + k;
    if (g < n)
      out[g] = s_data[pad(k)];
  }
}

// ---------------------------------------------------------------------------
// Scatter and per-tile ordering
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads) k_scatter(const int32_t* tile_of, int64_t n,
                                                      int32_t* cursor, int32_t* perm) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int t = i < n ? tile_of[i] : -1;
    const bool valid = t >= 0;  // negative keys (outliers) are not placed
    const unsigned mask = __match_any_sync(kFull, t);
    const int leader = __ffs(mask) - 1;
    int pos = 0;
    if (valid && lane == leader)
      pos = atomicAdd(&cursor[t], __popc(mask));
    pos = __shfl_sync(kFull, pos, leader);
    if (valid)
      perm[pos + __popc(mask & lanemask_lt())] = (int32_t)i;
  }
}

// Histogram of non-negative keys (warp-aggregated atomics).
__global__ void __launch_bounds__(kThreads) k_hist(const int32_t* keys, int64_t n, int32_t* count) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int t = i < n ? keys[i] : -1;
    const unsigned mask = __match_any_sync(kFull, t);
    if (t >= 0 && lane == __ffs(mask) - 1)
      atomicAdd(&count[t], __popc(mask));
  }
}

// Bitonic sort of s[0..P) (P a power of two) by the whole block.
__device__ void block_bitonic(int* s, int P) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const int a = s[i], b = s[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Sorts a segment of at most kSortCap ids in place (ascending).
__device__ void sort_segment(int32_t* seg, int m, int* s) {
  // Already ascending? (common when one warp scattered the whole tile)
  int unsorted = 0;
  for (int i = threadIdx.x; i + 1 < m; i += blockDim.x)
    unsorted |= seg[i] > seg[i + 1];
  if (!__syncthreads_or(unsorted))
    return;
  int P = 1;
  while (P < m)
    P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x)
    s[i] = (i < m) ? seg[i] : INT_MAX;
  __syncthreads();
  block_bitonic(s, P);
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    seg[i] = s[i];
  __syncthreads();
}

// Rank sort of one segment of m <= 32 * R distinct ids by one warp: lane L
// holds ids L, L + 32, ... in registers, `ids` holds all of them in shared
// memory, and an id's final position is the number of ids below it.
template <int R>
__device__ __forceinline__ void warp_rank_sort(int32_t* seg, int m, int* ids, int lane) {
  int v[R], r[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int i = k * 32 + lane;
    v[k] = i < m ? ids[i] : INT_MAX;
    r[k] = 0;
  }
  int j = 0;
  for (; j + 4 <= m; j += 4) {
    const int4 x = *reinterpret_cast<const int4*>(ids + j);
#pragma unroll
    for (int k = 0; k < R; ++k)
      r[k] += (x.x < v[k]) + (x.y < v[k]) + (x.z < v[k]) + (x.w < v[k]);
  }
  for (; j < m; ++j) {
    const int x = ids[j];
#pragma unroll
    for (int k = 0; k < R; ++k)
      r[k] += x < v[k];
  }
#pragma unroll
  for (int k = 0; k < R; ++k)
    if (k * 32 + lane < m)
      seg[r[k]] = v[k];
}

// Whether the ids of the segment starting at `begin` may stay in any order:
// with `event_exact` given, the segment is a tile of an event whose density
// sums are exact in any order (common.cuh), the only use of the ascending
// order within a tile on this run.
__device__ __forceinline__ bool order_free(const int32_t* event_exact, const int32_t* point_event,
                                          const EventDesc* events, const int32_t* perm, int begin) {
  if (!event_exact)
    return false;
  const int e = point_event[perm[begin]];
  return event_sums_exact(event_exact, e, events[e].n);
}

// Sets *some_ordered when any event of the run is not order-free (its sums
// are not exact in any order, event_sums_exact): one block, which clears the
// word first.
__global__ void k_events_order_free(const int32_t* event_exact, const EventDesc* events, int n_events,
                                    int32_t* some_ordered) {
  if (threadIdx.x == 0)
    *some_ordered = 0;
  __syncthreads();
  int ordered = 0;
  for (int e = threadIdx.x; e < n_events; e += blockDim.x)
    ordered |= !event_sums_exact(event_exact, e, events[e].n);
  if (__syncthreads_or(ordered) && threadIdx.x == 0)
    *some_ordered = 1;
}

// Orders the ids of every tile ascending. One warp per tile: tiles of up to
// kWarpSortCap ids are rank-sorted by the warp with no block barrier; larger
// tiles are listed for k_tile_sort_large (and for k_cells, which gives each a
// block). Tiles already in order (one warp of the scatter placed all of them)
// and tiles whose order does not matter (order_free) are left as they are.
constexpr int kWarpSortCap = kLargeTilePoints;
__global__ void __launch_bounds__(kThreads) k_tile_sort(const int32_t* tile_offset, int64_t n_tiles,
                                                        int32_t* perm, int32_t* large,
                                                        int32_t* large_count, const int32_t* event_exact,
                                                        const int32_t* point_event,
                                                        const EventDesc* events,
                                                        const int32_t* some_ordered) {
  __shared__ __align__(16) int s_ids[kThreads / 32][kWarpSortCap];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int* ids = s_ids[warp];
  // every event order-free: no tile is sorted, only the large ones listed
  const bool all_free = event_exact && *some_ordered == 0;
  const int64_t stride = (int64_t)gridDim.x * (kThreads / 32);
  for (int64_t t = (int64_t)blockIdx.x * (kThreads / 32) + warp; t < n_tiles; t += stride) {
    const int begin = tile_offset[t], end = tile_offset[t + 1];
    const int m = end - begin;
    if (m <= 1)
      continue;
    if (m > kWarpSortCap) {
      if (lane == 0)
        large[atomicAdd(large_count, 1)] = (int32_t)t;
      continue;
    }
    if (all_free || order_free(event_exact, point_event, events, perm, begin))
      continue;
    int unsorted = 0;
    for (int i = lane; i < m; i += 32) {
      const int v = perm[begin + i];
      ids[i] = v;
      if (i + 1 < m)
        unsorted |= v > perm[begin + i + 1];
    }
    __syncwarp();
    if (__any_sync(kFull, unsorted)) {
      int32_t* seg = perm + begin;
      if (m <= 64)
        warp_rank_sort<2>(seg, m, ids, lane);
      else if (m <= 128)
        warp_rank_sort<4>(seg, m, ids, lane);
      else
        warp_rank_sort<8>(seg, m, ids, lane);
    }
    __syncwarp();
  }
}

// Ascending bitonic sort of one value per lane across the warp.
__device__ __forceinline__ int warp_bitonic(int v, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int o = __shfl_xor_sync(kFull, v, j);
      const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
      v = keep_min ? min(v, o) : max(v, o);
    }
  }
  return v;
}

// Number of entries of the ascending 32-entry run `c` below v.
__device__ __forceinline__ int count_below(const int* c, int v) {
  int p = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    p += (c[p + step - 1] < v) ? step : 0;
  return p + (c[p] < v);
}

// Segments of kWarpSortCap < m <= kChunkRankCap ids: every warp sorts runs of
// 32 ids in registers, then each id's position is its place in its own run
// plus, for every other run, the number of ids below it (ids are distinct).
constexpr int kChunkRankCap = 1024;
__device__ void chunk_rank_sort(int32_t* seg, int m, int* s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int unsorted = 0;
  for (int i = threadIdx.x; i + 1 < m; i += kThreads)
    unsorted |= seg[i] > seg[i + 1];
  if (!__syncthreads_or(unsorted))
    return;
  const int runs = (m + 31) >> 5;
  for (int c = warp; c < runs; c += kThreads / 32) {
    const int i = c * 32 + lane;
    s[i] = warp_bitonic(i < m ? seg[i] : INT_MAX, lane);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < runs * 32; i += kThreads) {
    const int v = s[i];
    if (v == INT_MAX)
      continue;
    const int own = i >> 5;
    int rank = i & 31;
    for (int c = 0; c < runs; ++c)
      if (c != own)
        rank += count_below(s + c * 32, v);
    seg[rank] = v;
  }
  __syncthreads();
}

// Tiles listed by k_tile_sort (more than kWarpSortCap ids): one block each.
// Up to kChunkRankCap ids: chunk_rank_sort; up to kSortCap: a shared-memory
// bitonic sort; larger tiles become sorted chunks of kSortCap ids, listed for
// k_tile_merge.
__global__ void __launch_bounds__(kThreads) k_tile_sort_large(const int32_t* tile_offset,
                                                              const int32_t* large,
                                                              const int32_t* large_count,
                                                              int32_t* perm, int32_t* oversize,
                                                              int32_t* oversize_count,
                                                              const int32_t* event_exact,
                                                              const int32_t* point_event,
                                                              const EventDesc* events,
                                                              const int32_t* some_ordered) {
  __shared__ int s[kSortCap];
  if (event_exact && *some_ordered == 0)
    return;  // every event order-free
  const int count = *large_count;
  for (int e = blockIdx.x; e < count; e += gridDim.x) {
    const int t = large[e];
    const int begin = tile_offset[t], end = tile_offset[t + 1];
    const int m = end - begin;
    if (m <= 1 || order_free(event_exact, point_event, events, perm, begin))
      continue;
    if (m <= kChunkRankCap) {
      chunk_rank_sort(perm + begin, m, s);
    } else if (m <= kSortCap) {
      sort_segment(perm + begin, m, s);
    } else {
      for (int c = begin; c < end; c += kSortCap)
        sort_segment(perm + c, min(kSortCap, end - c), s);
      if (threadIdx.x == 0)
        oversize[atomicAdd(oversize_count, 1)] = (int32_t)t;
    }
  }
}

// Tiles larger than kSortCap hold sorted chunks of kSortCap ids. Each id's
// final rank is its rank in its chunk plus, for every other chunk, the number
// of ids below it (binary search); ids are distinct, so ranks are a permutation.
__global__ void __launch_bounds__(kThreads) k_tile_merge(const int32_t* tile_offset,
                                                         const int32_t* oversize,
                                                         const int32_t* oversize_count,
                                                         const int32_t* perm, int32_t* tmp) {
  const int count = *oversize_count;
  for (int e = blockIdx.x; e < count; e += gridDim.x) {
    const int t = oversize[e];
    const int begin = tile_offset[t], end = tile_offset[t + 1];
    const int m = end - begin;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      const int v = perm[begin + i];
      const int my_chunk = i / kSortCap;
      int rank = i - my_chunk * kSortCap;
      for (int c = 0; c * kSortCap < m; ++c) {
        if (c == my_chunk)
          continue;
        int lo = c * kSortCap, hi = min(m, lo + kSortCap);
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (perm[begin + mid] < v)
            lo = mid + 1;
          else
            hi = mid;
        }
        rank += lo - c * kSortCap;
      }
      tmp[begin + rank] = v;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_tile_merge_copy(const int32_t* tile_offset,
                                                              const int32_t* oversize,
                                                              const int32_t* oversize_count,
                                                              const int32_t* tmp, int32_t* perm) {
  const int count = *oversize_count;
  for (int e = blockIdx.x; e < count; e += gridDim.x) {
    const int t = oversize[e];
    for (int i = tile_offset[t] + threadIdx.x; i < tile_offset[t + 1]; i += blockDim.x)
      perm[i] = tmp[i];
  }
}

// Tile-contiguous copy of everything the sweeps read.
__global__ void __launch_bounds__(kThreads) k_gather(int D, int64_t n, const int32_t* perm,
                                                     CoordPtrs x, const float* w, CoordPtrs sig,
                                                     int32_t has_sigma, const float* unc,
                                                     const uint32_t* tags,
                                                     const int32_t* point_event, float* sx,
                                                     float* sw, float* ssig, float* sunc,
                                                     uint32_t* stag, int32_t* sevt, float4* rec,
                                                     int32_t flat, float flat_p0, int32_t* queue) {
  // The density records of the fast sweeps (rec, D = 2: {x, y, v, w}; D = 3:
  // {x, y, z, v}, v = fl(flat * w) for the flat kernel, ConvolutionalKernel.hpp:
  // 24-27, else w) come from the same loads, and the sweeps' work queues start
  // empty (queue[0], queue[1]).
  if (queue && blockIdx.x == 0 && threadIdx.x < 2)
    queue[threadIdx.x] = 0;
  auto record = [&](int64_t s, float x0, float x1, float x2, float wt) {
    const float v = flat ? __fmul_rn(flat_p0, wt) : wt;
    rec[s] = D == 2 ? make_float4(x0, x1, v, wt) : make_float4(x0, x1, x2, v);
  };
  // Two-dimensional runs with no per-point options (the common case) take
  // four points per thread a grid-stride apart, every gather issued before
  // any store, so more of this memory pass is in flight.
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if (D == 2 && !has_sigma && !unc && !tags) {
    constexpr int U = 4;
    for (int64_t s0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s0 < n; s0 += U * stride) {
      int i[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        i[u] = s0 + u * stride < n ? perm[s0 + u * stride] : 0;
      float vx[U], vy[U], vw[U];
      int ve[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        vx[u] = vy[u] = vw[u] = 0.0f;
        ve[u] = 0;
        if (s0 + u * stride < n) {
          vx[u] = x.p[0][i[u]];
          vy[u] = x.p[1][i[u]];
          vw[u] = w[i[u]];
          ve[u] = point_event[i[u]];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t s = s0 + u * stride;
        if (s >= n)
          break;
        sx[s] = vx[u];
        sx[n + s] = vy[u];
        sw[s] = vw[u];
        sevt[s] = ve[u];
        if (rec)
          record(s, vx[u], vy[u], 0.0f, vw[u]);
      }
    }
    return;
  }
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    const int i = perm[s];
    for (int d = 0; d < D; ++d)
      sx[d * n + s] = x.p[d][i];
    sw[s] = w[i];
    sevt[s] = point_event[i];
    if (rec && (D == 2 || D == 3))
      record(s, x.p[0][i], x.p[1][i], D == 3 ? x.p[2][i] : 0.0f, w[i]);
    if (has_sigma)
      for (int d = 0; d < D; ++d)
        ssig[d * n + s] = ((has_sigma >> d) & 1) ? sig.p[d][i] : 0.0f;
    if (unc)
      sunc[s] = unc[i];
    if (tags)
      stag[s] = tags[i];
  }
}

// ---------------------------------------------------------------------------
// Seeds and labels: core/detail/ClusteringKernels.hpp:293-343, :419-446
// ---------------------------------------------------------------------------

// One round of pointer jumping over the whole follower tree: every point moves
// its parent to its grandparent. Every write stores an ancestor, so rounds may
// overlap reads of updated entries; each round at least halves every path.
__global__ void k_jump(int64_t n, int32_t* parent) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int p = parent[s];
    const int pp = __ldcg(&parent[p]);
    if (pp != p)
      parent[s] = pp;
  }
}

// Root of each point's nearest-higher chain by pointer jumping with path
// halving: every write stores an ancestor, so concurrent updates stay valid
// and every step moves strictly up the tree. The tree is walked in the
// tile-contiguous layout (`parent` holds sorted positions, a root points to
// itself): a chain runs between neighbouring points, so its steps stay within
// a few tiles and mostly hit cache, and the lanes of a warp, which start on
// neighbouring points, share most of their chains.
// A piece of a larger batch (piece_base set) numbers its clusters and seed
// slots from *piece_base and its seed and nearest-higher indices from
// point_base.
__global__ void k_labels(int64_t n, int32_t* parent, const int32_t* perm, const int32_t* seed_flag,
                         const int32_t* seed_rank, const int32_t* point_event,
                         int32_t* cluster_index, int32_t* seeds, int32_t* seed_event,
                         uint32_t* status, const int32_t* piece_base, int32_t point_base,
                         int32_t event_base, int32_t* nh) {
  const int32_t base = piece_base ? *piece_base : 0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)s;
    int64_t steps = 0;
    for (;;) {
      const int px = __ldcg(&parent[x]);
      if (px == x)
        break;
      const int ppx = __ldcg(&parent[px]);
      if (ppx != px)
        parent[x] = ppx;
      x = ppx;
      if (++steps > n) {
        atomicOr(status, kStatusLabelTimeout);
        break;
      }
    }
    const int gi = perm[s];
    const int gr = perm[x];
    cluster_index[gi] = seed_flag[gr] ? seed_rank[gr] + base : -1;
    if (seed_flag[gi]) {
      seeds[seed_rank[gi] + base] = gi + point_base;
      seed_event[seed_rank[gi] + base] = point_event[gi] + event_base;
    }
    if (nh && nh[gi] >= 0)
      nh[gi] += point_base;
  }
}

// Labels of a run whose events each occupy their own range of the layout (one
// grid per event: event e's points are layout positions [begin, begin + n),
// and every nearest-higher chain stays inside its event) and hold at most
// kLocalLabelPoints points. A block takes one event at a time from a queue
// (largest first, so the longest ones do not run as a tail),
// copies the event's part of `parent` into shared memory as 16-bit event-local
// positions, and shortens every chain there by pointer-jumping rounds (every
// write stores an ancestor, so in-place rounds stay valid). The chains
// never touch global memory again: the global form above re-reads `parent`
// from L2 at every step and needs whole-array jumping rounds before it. The
// outputs are those of k_labels.
constexpr int kLocalLabelThreads = 1024;
constexpr int kLabelBatch = 4;
constexpr int kLabelRounds = 20;

__global__ void __launch_bounds__(kLocalLabelThreads, 1)
    k_labels_local(const EventDesc* events, int32_t n_events, int32_t* queue, const int32_t* parent,
                   const int32_t* perm, const int32_t* seed_flag, const int32_t* seed_rank,
                   const int32_t* point_event, int32_t* cluster_index, int32_t* seeds,
                   int32_t* seed_event, uint32_t* status, const int32_t* piece_base,
                   int32_t point_base, int32_t event_base, int32_t* nh) {
  extern __shared__ uint16_t up[];  // event-local parent of each point of the event
  __shared__ int s_event;
  const int32_t base = piece_base ? *piece_base : 0;
  for (;;) {
    if (threadIdx.x == 0)
      s_event = atomicAdd(queue, 1);
    __syncthreads();
    const int e = s_event;
    if (e >= n_events)
      break;
    const EventDesc ev = events[events[e].by_size];
    const int b = ev.begin, m = ev.n;
    bool outside = false;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      const int q = parent[b + i] - b;
      outside |= (unsigned)q >= (unsigned)m;
      up[i] = (uint16_t)((unsigned)q < (unsigned)m ? q : i);
    }
    if (outside)  // a chain leaving its event: never, for one grid per event
      atomicOr(status, kStatusLabelRange);
    __syncthreads();
    // chains: pointer-jumping rounds over the whole event (a round at least
    // halves every path, so 17 rounds reach the root of any chain of at most
    // 65,536 points; more means a cycle, which is reported) until every point
    // sits on its root. Rounds run over all points at once, so their shared-
    // memory loads overlap instead of following one chain at a time.
    for (int round = 0;; ++round) {
      int moved = 0;
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int q = up[i];
        const int qq = up[q];
        if (qq != q) {
          up[i] = (uint16_t)qq;
          moved = 1;
        }
      }
      if (!__syncthreads_or(moved))
        break;
      if (round == kLabelRounds) {
        if (threadIdx.x == 0)
          atomicOr(status, kStatusLabelTimeout);
        break;
      }
    }
    // outputs, kLabelBatch points per thread at a time so that their global
    // loads are in flight together
    for (int i0 = threadIdx.x; i0 < m; i0 += kLabelBatch * blockDim.x) {
      int gi[kLabelBatch], gr[kLabelBatch];
#pragma unroll
      for (int u = 0; u < kLabelBatch; ++u) {
        const int i = i0 + u * blockDim.x;
        gi[u] = gr[u] = -1;
        if (i < m) {
          gi[u] = perm[b + i];
          gr[u] = perm[b + up[i]];
        }
      }
#pragma unroll
      for (int u = 0; u < kLabelBatch; ++u) {
        if (gi[u] < 0)
          continue;
        cluster_index[gi[u]] = seed_flag[gr[u]] ? seed_rank[gr[u]] + base : -1;
        if (seed_flag[gi[u]]) {
          seeds[seed_rank[gi[u]] + base] = gi[u] + point_base;
          seed_event[seed_rank[gi[u]] + base] = point_event[gi[u]] + event_base;
        }
        if (nh && nh[gi[u]] >= 0)
          nh[gi[u]] += point_base;
      }
    }
    __syncthreads();  // up[] and s_event are rewritten for the next event
  }
}

// Moves a piece's base past its seeds, for the next piece of the batch.
__global__ void k_advance_piece(int32_t* piece_base, const int32_t* n_seeds) {
  if (threadIdx.x == 0)
    *piece_base += *n_seeds;
}

// Per-event relabelling after a batched run with one grid per event.
__global__ void k_localize(const EventDesc* events, const int32_t* point_event,
                           const int32_t* seed_rank, int64_t n, int32_t* cluster_index,
                           int32_t* nh) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const EventDesc ev = events[point_event[i]];
    const int c = cluster_index[i];
    if (c >= 0)
      cluster_index[i] = c - seed_rank[ev.begin];
    if (nh && nh[i] >= 0)
      nh[i] -= ev.begin;
  }
}

int grid_for(int64_t n, int per_block = kThreads) {
  const int64_t b = (n + per_block - 1) / per_block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count() * 16));
}

cudaError_t fill32(void* p, int64_t words, uint32_t v, cudaStream_t st) {
  if (words <= 0)
    return cudaSuccess;
  k_fill32<<<grid_for(words), kThreads, 0, st>>>((uint32_t*)p, words, v);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t scan(const int32_t* in, int32_t* out, int64_t n, int32_t* total,
                 const DeviceBuffers& b, cudaStream_t st) {
  if (n == 0)
    return fill32(total, 1, 0, st);
  const int blocks = scan_blocks_for(n);
  k_scan_reset<<<(blocks + kThreads - 1) / kThreads, kThreads, 0, st>>>(b.scan_desc, blocks,
                                                                        b.counters);  // [0]: ticket
  k_scan<<<blocks, kThreads, 0, st>>>(in, out, n, b.scan_desc, b.counters, total, b.status);
  count_launches(2);
  return cudaGetLastError();
}

// Sorts ids[offsets[k] .. offsets[k + 1]) ascending for every segment k.
// With `event_exact`, segments are tiles and those of exact-sum events keep
// their order (order_free).
cudaError_t sort_segments(const int32_t* offsets, int64_t n_segments, int32_t* ids,
                          const DeviceBuffers& b, cudaStream_t st, const int32_t* event_exact = nullptr,
                          int n_events = 0) {
  int32_t* oversize_count = b.counters + 2;
  int32_t* large_count = b.counters + 3;
  int32_t* some_ordered = b.counters + 7;
  cudaError_t e = fill32(oversize_count, 2, 0, st);  // and large_count, the next counter
  if (e != cudaSuccess)
    return e;
  if (event_exact) {
    k_events_order_free<<<1, 1024, 0, st>>>(event_exact, b.events, n_events, some_ordered);
    count_launches(1);
  }
  const int64_t warps_per_block = kThreads / 32;
  const int blocks =
      (int)std::max<int64_t>(1, std::min<int64_t>((n_segments + warps_per_block - 1) / warps_per_block,
                                                  (int64_t)sm_count() * 16));
  k_tile_sort<<<blocks, kThreads, 0, st>>>(offsets, n_segments, ids, b.large_tiles, large_count,
                                           event_exact, b.point_event, b.events, some_ordered);
  k_tile_sort_large<<<sm_count() * 8, kThreads, 0, st>>>(offsets, b.large_tiles, large_count, ids,
                                                  b.oversize, oversize_count, event_exact,
                                                  b.point_event, b.events, some_ordered);
  k_tile_merge<<<sm_count(), kThreads, 0, st>>>(offsets, b.oversize, oversize_count, ids, b.merge_tmp);
  k_tile_merge_copy<<<sm_count(), kThreads, 0, st>>>(offsets, b.oversize, oversize_count, b.merge_tmp,
                                              ids);
  count_launches(4);
  return cudaGetLastError();
}

thread_local int64_t t_launches = 0;

}  // namespace

int sm_count() {
  constexpr int kDevices = 64;
  static std::atomic<int> cache[kDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices)
    return 148;  // no usable device: the launch that follows reports the error
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      return 148;
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

// Lets k_labels_local take the shared memory of an event of `points` points
// on the current device (above the default 48 KB it needs the opt-in, set
// once per device for the largest event size). False when the device refuses.
bool local_labels_ready(int32_t points) {
  const size_t smem = ((size_t)std::max(points, 1) * sizeof(uint16_t) + 15) & ~(size_t)15;
  if (smem <= (48u << 10))
    return true;
  constexpr int kDevices = 64;
  static std::atomic<int> granted[kDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices)
    return false;
  const int need = (int)(((size_t)kLocalLabelPoints * sizeof(uint16_t)));
  if (granted[dev].load(std::memory_order_relaxed) < need) {
    if (cudaFuncSetAttribute(k_labels_local, cudaFuncAttributeMaxDynamicSharedMemorySize, need) != cudaSuccess) {
      cudaGetLastError();  // the refusal is not left pending for the next launch
      return false;
    }
    granted[dev].store(need, std::memory_order_relaxed);
  }
  return true;
}

int scan_blocks_for(int64_t n) { return (int)std::max<int64_t>(1, (n + kScanTile - 1) / kScanTile); }

void reset_launch_count() { t_launches = 0; }
int64_t launch_count() { return t_launches; }
void count_launches(int k) { t_launches += k; }

cudaError_t launch_fill32(void* p, int64_t words, uint32_t value, cudaStream_t st) {
  return fill32(p, words, value, st);
}

cudaError_t launch_wait_probe(unsigned long long* desc, uint32_t* status, cudaStream_t st) {
  k_wait_probe<<<1, 32, 0, st>>>(desc, status);
  return cudaGetLastError();
}

// utils/detail/get_clusters.hpp:24-49 on the device: cluster -> points as CSR,
// point ids ascending within a cluster (the order the reference's serial
// make_associator produces). The same stable counting sort as the tile
// binning, keyed by cluster id; outliers (-1) are left out.
cudaError_t launch_clusters_csr(const DeviceBuffers& b, int64_t n, const int32_t* labels,
                                int32_t n_clusters, int32_t* offsets, int32_t* points,
                                cudaStream_t st) {
  int32_t* count = b.parent;    // free after the run: n >= n_clusters
  int32_t* cursor = b.tile_of;  // idem
  cudaError_t e;
  if (n_clusters == 0)
    return cudaMemsetAsync(offsets, 0, sizeof(int32_t), st);
  if ((e = cudaMemsetAsync(count, 0, sizeof(int32_t) * n_clusters, st)))
    return e;
  k_hist<<<grid_for(n), kThreads, 0, st>>>(labels, n, count);
  count_launches(1);
  if ((e = cudaGetLastError()))
    return e;
  if ((e = scan(count, offsets, n_clusters, offsets + n_clusters, b, st)))
    return e;
  if ((e = cudaMemcpyAsync(cursor, offsets, sizeof(int32_t) * n_clusters, cudaMemcpyDeviceToDevice, st)))
    return e;
  k_scatter<<<grid_for(n), kThreads, 0, st>>>(labels, n, cursor, points);
  count_launches(1);
  if ((e = cudaGetLastError()))
    return e;
  return sort_segments(offsets, n_clusters, points, b, st);
}

cudaError_t launch_localize(const DeviceBuffers& b, int32_t n_events, int64_t n,
                            int32_t* cluster_index, int32_t* nh, cudaStream_t st) {
  (void)n_events;
  if (n == 0)
    return cudaSuccess;
  k_localize<<<grid_for(n), kThreads, 0, st>>>(b.events, b.point_event, b.seed_rank, n,
                                              cluster_index, nh);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_run(const RunShape& sh, const RunParams& prm, const RunIO& io,
                       const DeviceBuffers& b, cudaStream_t st, cudaEvent_t* marks) {
  const int D = sh.D;
  const int64_t n = sh.n;
  CoordPtrs x{}, sig{};
  for (int d = 0; d < D; ++d) {
    x.p[d] = io.coords[d];
    sig.p[d] = io.sigma[d];
  }
#define CLUE_CHECK(expr)          \
  do {                            \
    cudaError_t e_ = (expr);      \
    if (e_ != cudaSuccess)        \
      return e_;                  \
  } while (0)
#define CLUE_LAUNCHED()                 \
  do {                                  \
    count_launches(1);                  \
    CLUE_CHECK(cudaGetLastError());     \
  } while (0)
#define CLUE_MARK(i)                             \
  do {                                           \
    if (marks)                                   \
      CLUE_CHECK(cudaEventRecord(marks[i], st)); \
  } while (0)

  // grid extents
  CLUE_MARK(0);
  if (io.stats)
    CLUE_CHECK(fill32(io.stats, 16, 0, st));
  // exact-sum bounds per event (2-D and 3-D runs: their workspace holds them)
  int32_t* exact = (D == 2 || D == 3) ? b.event_exact : nullptr;
  const int64_t init_items = std::max<int64_t>((int64_t)sh.n_grids * kMaxDim, exact ? 4 * (int64_t)sh.n_events : 0);
  k_grid_init<<<(int)((init_items + 127) / 128), 128, 0, st>>>(b.grid_minmax, sh.n_grids, exact,
                                                               sh.n_events);
  CLUE_LAUNCHED();
  k_minmax<<<sh.n_chunks, kThreads, 0, st>>>(D, x, b.chunks, b.events, b.grid_minmax);
  CLUE_LAUNCHED();
  k_grid_finalize<<<(sh.n_grids + 127) / 128, 128, 0, st>>>(D, b.grids, sh.n_grids, b.grid_minmax);
  CLUE_LAUNCHED();

  // counting sort by tile
  CLUE_MARK(1);
  if (sh.stable && prm.stable_binning) {
    // Stable binning: runs of consecutive points, one warp each; the count
    // matrices (at most 4 n entries) live in the nearest-higher records, which
    // the sweeps write much later.
    int32_t* matrix = reinterpret_cast<int32_t*>(b.rec_nh);
    const int wpb = std::max(1, std::min(kThreads / 32, (48 << 10) / (4 * std::max(1, sh.max_event_tiles))));
    const int blocks = (sh.sort_warps + wpb - 1) / wpb;
    const size_t smem = (size_t)wpb * sh.max_event_tiles * sizeof(int);
    CLUE_CHECK(fill32(b.counters + 3, 1, 0, st));  // large-tile count
    k_bin_stable<<<blocks, wpb * 32, smem, st>>>(prm, x, b.events, sh.n_events, sh.sort_warps, b.grids,
                                                 b.tile_of, b.point_event, matrix,
                                                 sh.max_event_tiles, io.weight, exact, b.tile_cursor);
    CLUE_LAUNCHED();
    k_tile_prefix<<<grid_for(sh.n_tiles), kThreads, 0, st>>>(b.events, b.grids, sh.n_tiles, b.tile_cursor,
                                                             matrix, b.tile_count);
    CLUE_LAUNCHED();
    CLUE_CHECK(scan(b.tile_count, b.tile_offset, sh.n_tiles, b.tile_offset + sh.n_tiles, b, st));
    k_scatter_stable<<<blocks, wpb * 32, smem, st>>>(b.events, sh.n_events, sh.sort_warps, b.grids,
                                                     b.tile_of, matrix, sh.max_event_tiles,
                                                     b.tile_offset, b.tile_count, b.perm,
                                                     b.large_tiles, b.counters + 3);
    CLUE_LAUNCHED();
  } else {
    CLUE_CHECK(fill32(b.tile_count, sh.n_tiles, 0, st));
    k_bin<<<sh.n_chunks, kThreads, 0, st>>>(prm, x, b.chunks, b.events, b.grids, b.tile_of,
                                             b.point_event, b.tile_count, io.weight, exact);
    CLUE_LAUNCHED();
    CLUE_CHECK(scan(b.tile_count, b.tile_offset, sh.n_tiles, b.tile_offset + sh.n_tiles, b, st));
    k_copy32<<<grid_for(sh.n_tiles), kThreads, 0, st>>>((uint32_t*)b.tile_cursor,
                                                       (const uint32_t*)b.tile_offset, sh.n_tiles);
    CLUE_LAUNCHED();
    k_scatter<<<grid_for(n), kThreads, 0, st>>>(b.tile_of, n, b.tile_cursor, b.perm);
    CLUE_LAUNCHED();
    // Exact-sum events need no ascending order within their tiles when nothing
    // else on this run reads it (flat kernel, cell path: no user tags).
    const bool order_free_tiles = sweep_cells_path(prm) && prm.kernel_kind == CLUE_KERNEL_FLAT;
    CLUE_CHECK(sort_segments(b.tile_offset, sh.n_tiles, b.perm, b, st, order_free_tiles ? exact : nullptr,
                             sh.n_events));
  }
  CLUE_MARK(2);
  k_gather<<<grid_for(n), kThreads, 0, st>>>(D, n, b.perm, x, io.weight, sig, prm.has_sigma,
                                             io.unc, io.tags, b.point_event, b.sorted_coords,
                                             b.sorted_weight, b.sorted_sigma, b.sorted_unc,
                                             b.sorted_tag, b.sorted_event,
                                             sweep_fast_path(prm) ? b.rec_dens : nullptr,
                                             prm.kernel_kind == CLUE_KERNEL_FLAT, prm.kernel_p0,
                                             b.counters + 4);
  CLUE_LAUNCHED();

  // the two sweeps
  SweepArgs a{};
  a.n = n;
  a.n_tiles = sh.n_tiles;
  a.work_dens = b.work_dens;
  a.work_nh = b.work_nh;
  a.cls_dens = b.cls_dens;
  a.cls_nh = b.cls_nh;
  a.queue = b.counters + 4;
  a.large_tiles = b.large_tiles;  // listed by sort_segments above
  a.large_count = b.counters + 3;
  a.rec_dens = b.rec_dens;
  a.rec_nh = b.rec_nh;
  a.rec_tag = b.rec_tag;
  a.events = b.events;
  a.grids = b.grids;
  a.tile_offset = b.tile_offset;
  a.sx = b.sorted_coords;
  a.sw = b.sorted_weight;
  a.ssig = b.sorted_sigma;
  a.sunc = b.sorted_unc;
  a.stag = b.sorted_tag;
  a.perm = b.perm;
  a.sevt = b.sorted_event;
  a.srho = b.sorted_rho;
  a.out_rho = io.rho;
  a.out_nh = io.nh ? io.nh : b.nh;
  a.out_seed = io.is_seed;
  a.seed_flag = b.seed_flag;
  a.parent = b.parent;
  a.stats = io.stats;
  a.status = b.status;
  if (sweep_fast_path(prm)) {
    a.nh_cells = sweep_cells_path(prm);
    a.nh_pos = b.nh_pos;
    a.nh_q = b.nh_q;
    a.cell_slot = b.cell_slot;
    a.cell_s = b.cell_s;
    a.cell_geom = b.cell_geom;
    a.cell_info = b.cell_info;
    a.cell_box = b.cell_box;
    a.rec_cell = b.rec_cell;
    a.event_exact = b.event_exact;
    a.n_events = sh.n_events;
    a.walk = b.cls_nh;  // k_work_order's scratch, free once it has run
  }
  CLUE_CHECK(launch_work_order(D, prm, a, st));
  CLUE_MARK(3);
  CLUE_CHECK(launch_density(D, prm, a, st));
  CLUE_MARK(4);
  CLUE_CHECK(launch_nearest_higher(D, prm, a, st));
  CLUE_MARK(5);

  // seeds and labels
  CLUE_CHECK(scan(b.seed_flag, b.seed_rank, n, b.counters + 1, b, st));
  const bool piece = io.piece_base != nullptr;
  int32_t* nh_shift = piece && io.point_base ? io.nh : nullptr;
  // One grid per event keeps every event in its own range of the layout: the
  // chains are walked per event in shared memory.
  const bool local_labels = sh.n_grids == sh.n_events && sh.max_event_points <= kLocalLabelPoints &&
                            local_labels_ready(sh.max_event_points);
  if (local_labels) {
    const size_t smem = ((size_t)std::max(sh.max_event_points, 1) * sizeof(uint16_t) + 15) & ~(size_t)15;
    const int blocks = std::max(1, std::min(sh.n_events, sm_count() * (smem <= (96u << 10) ? 2 : 1)));
    CLUE_CHECK(fill32(b.counters + 6, 1, 0, st));
    k_labels_local<<<blocks, kLocalLabelThreads, smem, st>>>(
        b.events, sh.n_events, b.counters + 6, b.parent, b.perm, b.seed_flag, b.seed_rank,
        b.point_event, io.cluster_index, b.seeds, b.seed_event, b.status, io.piece_base,
        (int32_t)io.point_base, io.event_base, nh_shift);
    CLUE_LAUNCHED();
  } else {
    // Large runs first shorten every chain with whole-array jumping rounds, so
    // the per-point walks below take a few steps; small runs walk directly.
    const int jump_rounds = prm.jump_rounds >= 0                ? prm.jump_rounds
                            : n >= (int64_t)1 << 22 ? 3
                            : n >= (int64_t)1 << 18 ? 2
                                                    : 0;
    for (int r = 0; r < jump_rounds; ++r) {
      k_jump<<<grid_for(n), kThreads, 0, st>>>(n, b.parent);
      CLUE_LAUNCHED();
    }
    k_labels<<<grid_for(n), kThreads, 0, st>>>(n, b.parent, b.perm, b.seed_flag, b.seed_rank,
                                               b.point_event, io.cluster_index, b.seeds,
                                               b.seed_event, b.status, io.piece_base,
                                               (int32_t)io.point_base, io.event_base, nh_shift);
    CLUE_LAUNCHED();
  }
  if (piece) {
    k_advance_piece<<<1, 32, 0, st>>>(io.piece_base, b.counters + 1);
    CLUE_LAUNCHED();
  }
  CLUE_MARK(6);
#undef CLUE_MARK
#undef CLUE_LAUNCHED
#undef CLUE_CHECK
  return cudaSuccess;
}

}  // namespace clue_impl
