// abi.cu — the extern "C" entry points of libclue_sm100.so (include/clue_sm100.h):
// parameter validation, workspace management, host/device clustering calls and
// result accessors. The serving loop lives in server.cu.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "abi_internal.h"

using namespace clue_impl;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------

namespace {
thread_local std::string t_last_error;
}

namespace clue_impl {

clue_status fail(clue_status s, const std::string& msg) {
  t_last_error = msg;
  return s;
}

clue_status fail_cuda(cudaError_t e, const char* where) {
  return fail(e == cudaErrorMemoryAllocation ? CLUE_ERR_OUT_OF_MEMORY : CLUE_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Tables
// ---------------------------------------------------------------------------

int32_t sort_runs(int64_t n, int32_t* len) {
  const int64_t runs = std::max<int64_t>(1, (n + kStableRun - 1) / kStableRun);
  *len = kStableRun;
  return (int32_t)std::min<int64_t>(runs, INT32_MAX);
}

// core/detail/SetupTiles.hpp:30-34.
bool grid_shape(int D, int64_t n, int ppt, int32_t* k_out, int64_t* T_out) {
  const int64_t nt = (n + ppt - 1) / ppt;
  int64_t k = 1;
  auto powk = [D](int64_t k) {
    int64_t p = 1;
    for (int d = 0; d < D; ++d) {
      p *= k;
      if (p > (int64_t)1 << 40)
        return p;
    }
    return p;
  };
  // the smallest k with k^D >= nt, searched upward from just below the root
  if (nt > 1)
    k = std::max<int64_t>(1, (int64_t)std::floor(std::pow((double)nt, 1.0 / D)) - 1);
  while (powk(k) < nt)
    ++k;
  *k_out = (int32_t)k;
  *T_out = powk(k);
  return *T_out < INT32_MAX;
}

void fill_grid(GridDesc* g, int D, int32_t k, int64_t T) {
  std::memset(g, 0, sizeof(GridDesc));
  g->k = k;
  g->T = (int32_t)T;
  int32_t s = 1;
  for (int d = D - 1; d >= 0; --d) {
    g->stride[d] = s;
    s *= k;
  }
}

// EventDesc::by_size of events[0, B): largest first, by a counting sort on
// the size's binary magnitude and next two bits (sizes within 25 % keep index
// order; the order only balances per-event passes).
void order_by_size(EventDesc* events, int32_t B) {
  auto bucket = [](int32_t m) {
    if (m <= 3)
      return m;
    const int lg = 31 - __builtin_clz((uint32_t)m);
    return 4 * (lg - 1) + ((m >> (lg - 2)) & 3);
  };
  constexpr int kBuckets = 4 * 31;
  int32_t first[kBuckets + 1] = {};
  for (int e = 0; e < B; ++e)
    ++first[kBuckets - 1 - bucket(events[e].n)];
  for (int b = 0, acc = 0; b <= kBuckets; ++b) {
    const int c = first[b];
    first[b] = acc;
    acc += c;
  }
  for (int e = 0; e < B; ++e)
    events[first[kBuckets - 1 - bucket(events[e].n)]++].by_size = e;
}

bool build_tables(int32_t D, const uint32_t* sizes, int32_t B, int32_t grid_mode, int32_t ppt,
                  HostTables* t, RunShape* sh, const char** err) {
  ppt = ppt > 0 ? ppt : 128;
  int64_t N = 0;
  for (int e = 0; e < B; ++e)
    N += sizes[e];
  if (N <= 0 || N >= INT32_MAX) {
    *err = N <= 0 ? "the number of points must be positive" : "too many points for int32 indices";
    return false;
  }
  t->grids.clear();
  t->events.clear();
  t->chunks.clear();
  t->events.resize(B);
  int64_t tiles = 0;
  int64_t begin = 0;
  if (grid_mode == CLUE_GRID_SHARED) {
    int32_t k;
    int64_t T;
    if (!grid_shape(D, N, ppt, &k, &T) || T * B >= INT32_MAX) {
      *err = "tile grid too large";
      return false;
    }
    t->grids.resize(1);
    fill_grid(&t->grids[0], D, k, T);
    for (int e = 0; e < B; ++e) {
      t->events[e] = EventDesc{(int32_t)begin, (int32_t)sizes[e], (int32_t)(T * e), 0, 0, 0, 0, 0};
      begin += sizes[e];
    }
    tiles = T * B;
  } else {
    t->grids.resize(B);
    for (int e = 0; e < B; ++e) {
      int32_t k;
      int64_t T;
      if (!grid_shape(D, sizes[e], ppt, &k, &T)) {
        *err = "tile grid too large";
        return false;
      }
      fill_grid(&t->grids[e], D, k, T);
      t->events[e] = EventDesc{(int32_t)begin, (int32_t)sizes[e], (int32_t)tiles, e, 0, 0, 0, 0};
      begin += sizes[e];
      tiles += T;
      if (tiles >= INT32_MAX) {
        *err = "tile grid too large";
        return false;
      }
    }
  }
  int64_t n_chunks = 0;
  for (int e = 0; e < B; ++e)
    n_chunks += (t->events[e].n + kChunkPoints - 1) / kChunkPoints;
  t->chunks.reserve(n_chunks);
  for (int e = 0; e < B; ++e) {
    const EventDesc& ev = t->events[e];
    for (int32_t c = ev.begin; c < ev.begin + ev.n; c += kChunkPoints)
      t->chunks.push_back(Chunk{e, c, std::min(ev.begin + ev.n, c + kChunkPoints)});
  }
  // Stable binning layout: runs of each event, their warps and count matrices.
  int64_t warps = 0, entries = 0;
  int32_t max_tiles = 0, max_points = 0;
  for (int e = 0; e < B; ++e) {
    EventDesc& ev = t->events[e];
    max_points = std::max(max_points, ev.n);
    const int64_t T = t->grids[ev.grid].T;
    ev.sort_chunks = sort_runs(ev.n, &ev.sort_len);
    ev.sort_first = (int32_t)std::min<int64_t>(warps, INT32_MAX);
    ev.sort_base = (int32_t)std::min<int64_t>(entries, INT32_MAX);
    warps += ev.sort_chunks;
    entries += T * ev.sort_chunks;
    max_tiles = (int32_t)std::max<int64_t>(max_tiles, std::min<int64_t>(T, INT32_MAX));
  }
  order_by_size(t->events.data(), B);
  sh->stable = max_tiles <= kStableMaxTiles && entries <= 4 * N && warps < INT32_MAX;
  sh->sort_warps = (int32_t)std::min<int64_t>(warps, INT32_MAX);
  sh->sort_entries = entries;
  sh->max_event_tiles = max_tiles;
  sh->max_event_points = max_points;
  sh->D = D;
  sh->n = N;
  sh->n_tiles = tiles;
  sh->n_events = B;
  sh->n_grids = (int32_t)t->grids.size();
  sh->n_chunks = (int32_t)t->chunks.size();
  return true;
}

// The tables of a batch shape in ws->tables: rebuilt only when the dimension,
// grid mode, points per tile or event sizes differ from the last build's
// (a batch of the same shape has the same tables). False, with *err set, when
// build_tables rejects the shape.
bool shape_tables(clue_workspace* ws, int32_t D, const uint32_t* sizes, int32_t B, int32_t grid_mode,
                  int32_t ppt, const char** err) {
  clue_workspace::TableCache& c = ws->tables;
  if (c.valid && c.D == D && c.grid_mode == grid_mode && c.ppt == ppt &&
      c.sizes.size() == (size_t)std::max(B, 0) && std::equal(sizes, sizes + B, c.sizes.begin()))
    return true;
  c.valid = c.split = false;
  if (!build_tables(D, sizes, B, grid_mode, ppt, &c.tables, &c.shape, err))
    return false;
  c.sizes.assign(sizes, sizes + B);
  c.D = D;
  c.grid_mode = grid_mode;
  c.ppt = ppt;
  c.valid = true;
  return true;
}

// ---------------------------------------------------------------------------
// Workspace memory
// ---------------------------------------------------------------------------

namespace {

struct Layout {
  size_t total = 0;
  template <typename T>
  size_t add(int64_t count) {
    const size_t off = total;
    total += ((size_t)std::max<int64_t>(count, 1) * sizeof(T) + 255) & ~size_t(255);
    return off;
  }
};

// Places every buffer of `cap` in one allocation (or measures it when base is null).
size_t place(DeviceBuffers* b, const Capacity& c, char* base) {
  Layout L;
  const int64_t N = c.points, T = c.tiles, D = c.dims;
  auto at = [&](size_t off) { return base ? base + off : nullptr; };
#define CLUE_PLACE(field, type, count) \
  do {                                 \
    size_t o_ = L.add<type>(count);    \
    b->field = (type*)at(o_);          \
  } while (0)
  CLUE_PLACE(grids, GridDesc, c.grids);
  CLUE_PLACE(events, EventDesc, c.events);
  CLUE_PLACE(chunks, Chunk, c.chunks);
  CLUE_PLACE(grid_minmax, int32_t, c.grids * 2 * kMaxDim);
  CLUE_PLACE(tile_of, int32_t, N);
  CLUE_PLACE(point_event, int32_t, N);
  CLUE_PLACE(nh, int32_t, N);
  CLUE_PLACE(seed_flag, int32_t, N);
  CLUE_PLACE(seed_rank, int32_t, N);
  CLUE_PLACE(parent, int32_t, N);
  CLUE_PLACE(tile_count, int32_t, T);
  CLUE_PLACE(tile_offset, int32_t, T + 1);
  CLUE_PLACE(tile_cursor, int32_t, T);
  CLUE_PLACE(perm, int32_t, N);
  CLUE_PLACE(sorted_event, int32_t, N);
  CLUE_PLACE(sorted_coords, float, D * N);
  CLUE_PLACE(sorted_weight, float, N);
  CLUE_PLACE(sorted_rho, float, N);
  CLUE_PLACE(merge_tmp, int32_t, N);
  CLUE_PLACE(work_dens, int32_t, N);
  CLUE_PLACE(work_nh, int32_t, N);
  CLUE_PLACE(cls_dens, int32_t, N);
  CLUE_PLACE(cls_nh, int32_t, N);
  CLUE_PLACE(rec_dens, float4, N);
  CLUE_PLACE(rec_nh, float4, N);
  CLUE_PLACE(rec_tag, uint32_t, N);
  // cell layout of 2-D and 3-D runs, sized for D = 3
  CLUE_PLACE(nh_pos, int32_t, c.cells ? N : 0);
  CLUE_PLACE(nh_q, int32_t, c.cells ? N : 0);
  CLUE_PLACE(cell_slot, int32_t, c.cells ? N : 0);
  CLUE_PLACE(cell_s, int32_t, c.cells ? T : 0);
  CLUE_PLACE(cell_geom, float4, c.cells ? 2 * T : 0);
  CLUE_PLACE(cell_info, CellInfo, c.cells ? N : 0);
  CLUE_PLACE(cell_box, float4, c.cells ? 2 * N : 0);
  CLUE_PLACE(rec_cell, float4, c.cells ? N : 0);
  CLUE_PLACE(event_exact, int32_t, c.cells ? 4 * c.events : 0);
  CLUE_PLACE(seeds, int32_t, N);
  CLUE_PLACE(seed_event, int32_t, N);
  CLUE_PLACE(scan_desc, unsigned long long, c.scan_blocks);
  CLUE_PLACE(counters, int32_t, 16);
  CLUE_PLACE(large_tiles, int32_t, N / 256 + 1);
  CLUE_PLACE(oversize, int32_t, N / 4096 + 1);
  CLUE_PLACE(status, uint32_t, 1);
  CLUE_PLACE(stats, unsigned long long, 8);
  CLUE_PLACE(sorted_sigma, float, c.sigma ? D * N : 0);
  CLUE_PLACE(sorted_unc, float, c.unc ? N : 0);
  CLUE_PLACE(sorted_tag, uint32_t, c.tags ? N : 0);
  const int64_t S = c.staged_points;
  CLUE_PLACE(in_coords, float, S ? D * S : 0);
  CLUE_PLACE(in_weight, float, S);
  CLUE_PLACE(in_sigma, float, (S && c.sigma) ? D * S : 0);
  CLUE_PLACE(in_unc, float, (S && c.unc) ? S : 0);
  CLUE_PLACE(in_tags, uint32_t, (S && c.tags) ? S : 0);
  CLUE_PLACE(out_cluster, int32_t, S);
  CLUE_PLACE(out_seed, int32_t, S);
  CLUE_PLACE(out_rho, float, S);
  CLUE_PLACE(out_nh, int32_t, S);
#undef CLUE_PLACE
  return L.total;
}

}  // namespace

size_t carve_buffers(DeviceBuffers* b, const Capacity& c, char* base) { return place(b, c, base); }

size_t scratch_bytes(const RunShape& s, bool sigma, bool unc, bool tags) {
  Capacity c;
  c.points = s.n;
  c.tiles = s.n_tiles;
  c.events = s.n_events;
  c.chunks = s.n_chunks;
  c.grids = s.n_grids;
  c.scan_blocks = scan_blocks_for(std::max<int64_t>(s.n, s.n_tiles));
  c.dims = s.D;
  c.sigma = sigma;
  c.unc = unc;
  c.tags = tags;
  c.cells = s.D == 2 || s.D == 3;
  DeviceBuffers b;
  return place(&b, c, nullptr);
}

// Whether the workspace's buffers already hold a run of this shape.
bool capacity_fits(const clue_workspace* ws, const RunShape& s, bool sigma, bool unc, bool tags,
                   int64_t staged) {
  const Capacity& c = ws->cap;
  const int64_t scan_blocks = scan_blocks_for(std::max<int64_t>(s.n, s.n_tiles));
  const bool cells = s.D == 2 || s.D == 3;
  return c.points >= s.n && c.tiles >= s.n_tiles && c.events >= s.n_events &&
         c.chunks >= s.n_chunks && c.grids >= s.n_grids && c.scan_blocks >= scan_blocks &&
         c.dims >= s.D && (!sigma || c.sigma) && (!unc || c.unc) && (!tags || c.tags) &&
         (!cells || c.cells) && c.staged_points >= staged;
}

clue_status ensure_capacity(clue_workspace* ws, const RunShape& s, bool sigma, bool unc, bool tags,
                            int64_t staged) {
  if (capacity_fits(ws, s, sigma, unc, tags, staged))
    return CLUE_OK;
  const Capacity& c = ws->cap;
  const bool cells = s.D == 2 || s.D == 3;
  // Grow every dimension that is short by 25 % headroom; keep what fits.
  auto grow = [](int64_t have, int64_t need) { return have >= need ? have : need + need / 4; };
  Capacity n = c;
  n.points = grow(c.points, s.n);
  n.tiles = grow(c.tiles, s.n_tiles);
  n.events = grow(c.events, s.n_events);
  n.chunks = grow(c.chunks, s.n_chunks);
  n.grids = grow(c.grids, s.n_grids);
  n.scan_blocks = scan_blocks_for(std::max<int64_t>(n.points, n.tiles));
  n.dims = std::max(c.dims, s.D);
  n.sigma = c.sigma || sigma;
  n.unc = c.unc || unc;
  n.tags = c.tags || tags;
  n.cells = c.cells || cells;
  n.staged_points = staged ? grow(c.staged_points, staged) : c.staged_points;
  DeviceBuffers nb;
  const size_t bytes = place(&nb, n, nullptr);
  if (ws->base) {
    // cudaFree waits for the device; earlier runs on any stream are finished.
    cudaFree(ws->base);
    ws->base = nullptr;
    ws->bytes = 0;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    ws->cap = Capacity{};
    ws->b = DeviceBuffers{};
    return fail_cuda(e, "workspace allocation");
  }
  ws->base = (char*)p;
  ws->bytes = bytes;
  place(&ws->b, n, ws->base);
  ws->cap = n;
  cudaMemset(ws->b.status, 0, sizeof(uint32_t));
  return CLUE_OK;
}

clue_status check_params(const clue_params* p) {
  if (!p)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "params is null");
  // core/detail/Clusterer.hpp:42-48
  if (!(p->dc > 0.0f) || !(p->rhoc >= 0.0f) || !(p->dm > 0.0f) || !(p->seed_dc > 0.0f))
    return fail(CLUE_ERR_INVALID_ARGUMENT,
                "Invalid clustering parameters. The parameters must be positive.");
  // core/detail/ConvolutionalKernel.hpp:13-50
  switch (p->kernel_kind) {
    case CLUE_KERNEL_FLAT:
      if (!(p->kernel_params[0] > 0.0f))
        return fail(CLUE_ERR_INVALID_ARGUMENT, "Flat kernel parameter must be positive.");
      break;
    case CLUE_KERNEL_GAUSSIAN:
      if (!(p->kernel_params[0] > 0.0f) || !(p->kernel_params[1] > 0.0f))
        return fail(CLUE_ERR_INVALID_ARGUMENT, "Gaussian kernel parameters must be positive.");
      break;
    case CLUE_KERNEL_EXPONENTIAL:
      if (!(p->kernel_params[0] > 0.0f) || !(p->kernel_params[1] > 0.0f))
        return fail(CLUE_ERR_INVALID_ARGUMENT, "Exponential kernel parameters must be positive.");
      break;
    default:
      return fail(CLUE_ERR_INVALID_ARGUMENT, "unknown convolutional kernel");
  }
  if (p->metric_kind < CLUE_METRIC_EUCLIDEAN || p->metric_kind > CLUE_METRIC_MAHALANOBIS)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "unknown distance metric");
  if (p->points_per_tile < 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "points_per_tile must be >= 0");
  return CLUE_OK;
}

clue_status check_points(const clue_points* pts, bool need_output, int metric_kind) {
  if (!pts)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "points is null");
  if (pts->ndim < 1 || pts->ndim > CLUE_MAX_DIM)
    return fail(CLUE_ERR_OUT_OF_RANGE, "ndim must be in [1, 10]");
  if (pts->n <= 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT,
                "Number of points passed to the points constructor must be positive.");
  for (int d = 0; d < pts->ndim; ++d)
    if (!pts->coords[d])
      return fail(CLUE_ERR_INVALID_ARGUMENT, "missing coordinate array");
  if (!pts->weight)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "missing weight array");
  if (need_output && !pts->cluster_index)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "missing cluster_index output");
  if (metric_kind == CLUE_METRIC_MAHALANOBIS)
    for (int d = 0; d < pts->ndim; ++d)
      if (!pts->sigma[d])
        return fail(CLUE_ERR_INVALID_ARGUMENT,
                    "the Mahalanobis metric needs sigma for every dimension");
  return CLUE_OK;
}

// Largest float x >= 0 with sqrtf(x) <= r (sqrt is correctly rounded on host
// and device, and monotone, so `sqrt(d2) <= r` is exactly `d2 <= x`).
float sqrt_threshold(float r) {
  if (!(r >= 0.0f))
    return -1.0f;
  if (std::isinf(r))
    return INFINITY;
  float x = (float)((double)r * (double)r);
  if (!std::isfinite(x))
    x = FLT_MAX;
  while (x > 0.0f && std::sqrt(x) > r)
    x = std::nextafter(x, 0.0f);
  for (;;) {
    const float up = std::nextafter(x, INFINITY);
    if (std::isinf(up) || std::sqrt(up) > r)
      break;
    x = up;
  }
  return x;
}

clue_tuning default_tuning() {
  clue_tuning t{};
  // Measured on B200: in 2-D a warp with two box shapes reads its own
  // candidates about as fast as it streams a union a quarter larger; in 3-D
  // the per-point reads of mixed warps are far slower than any union.
  t.density_union_x16_2d = 20;
  t.density_union_x16_3d = 1 << 20;
  t.label_jump_rounds = -1;
  t.cell_points = 2;
  t.density_shape = 0;
  t.nh_shape = 0;
  t.tile_binning = 1;
  return t;
}

RunParams make_run_params(const clue_params* p, const clue_points* pts, const clue_tuning& t) {
  RunParams r{};
  r.union_x16 = pts->ndim == 3 ? t.density_union_x16_3d : t.density_union_x16_2d;
  r.jump_rounds = t.label_jump_rounds;
  r.cell_points = t.cell_points;
  r.dens_shape = t.density_shape;
  r.nh_shape = t.nh_shape;
  r.stable_binning = t.tile_binning;
  r.D = pts->ndim;
  r.dc = p->dc;
  r.rhoc = p->rhoc;
  r.dm = p->dm;
  r.seed_dc = p->seed_dc;
  for (int d = 0; d < kMaxDim; ++d) {
    r.wrapped[d] = p->wrapped[d] ? 1 : 0;
    r.mparam[d] = p->metric_params[d];
  }
  r.kernel_kind = p->kernel_kind;
  r.kernel_p0 = p->kernel_params[0];
  r.kernel_p1 = p->kernel_params[1];
  r.metric_kind = p->metric_kind;
  r.dc2 = sqrt_threshold(p->dc);
  // Nearest-higher thresholds stop at FLT_MAX: the reference's search starts
  // from delta = FLT_MAX and only takes dist < delta, so a candidate at an
  // infinite distance (d2 = inf) never becomes the nearest higher, while every
  // finite d2 has sqrt(d2) < FLT_MAX.
  r.dm2 = std::min(sqrt_threshold(p->dm), FLT_MAX);
  r.seed2 = std::min(sqrt_threshold(p->seed_dc), FLT_MAX);
  r.has_sigma = 0;
  for (int d = 0; d < pts->ndim; ++d)
    if (pts->sigma[d])
      r.has_sigma |= 1 << d;
  r.has_unc = pts->density_uncertainty != nullptr;
  r.has_tags = pts->tags != nullptr;
  // Gaussian denominator (2 * std) * std, rounded as the device rounds it.
  r.gauss_inv_den = 0.0f;
  r.exp_in_range = 0;
  if (p->kernel_kind == CLUE_KERNEL_GAUSSIAN) {
    const float den = (2.0f * p->kernel_params[0]) * p->kernel_params[0];
    int e = 0;
    const float m = std::frexp(den, &e);
    if (m == 0.5f && e - 1 >= -125 && e - 1 <= 125)
      r.gauss_inv_den = std::ldexp(1.0f, 1 - e);
    // exponents of in-range pairs lie in [-(dc^2/den)(1 + 2^-22), 0]
    r.exp_in_range = std::isfinite(den) && den > 0.0f &&
                     (double)p->dc * (double)p->dc / (double)den <= 100.0;
  } else if (p->kernel_kind == CLUE_KERNEL_EXPONENTIAL) {
    // exponents lie in [-(avg * dc)(1 + 2^-23), 0]
    r.exp_in_range = (double)p->kernel_params[0] * (double)p->dc <= 100.0;
  }
  return r;
}

// Uploads the host tables through the workspace's pinned staging buffer.
// Copies the run tables into the pinned staging buffer, after the previous
// upload has left it (a host wait: done before any stream capture).
clue_status stage_tables(clue_workspace* ws, const HostTables& t) {
  const size_t g = t.grids.size() * sizeof(GridDesc);
  const size_t e = t.events.size() * sizeof(EventDesc);
  const size_t c = t.chunks.size() * sizeof(Chunk);
  const size_t need = g + e + c;
  if (ws->staging_event) {
    const cudaError_t err = cudaEventSynchronize(ws->staging_event);
    if (err != cudaSuccess)
      return fail_cuda(err, "table staging wait");
  }
  if (ws->staging_bytes < need) {
    if (ws->staging)
      cudaFreeHost(ws->staging);
    ws->staging = nullptr;
    ws->staging_bytes = 0;
    cudaError_t err = cudaMallocHost(&ws->staging, need + need / 4);
    if (err != cudaSuccess)
      return fail_cuda(err, "pinned staging allocation");
    ws->staging_bytes = need + need / 4;
  }
  char* h = (char*)ws->staging;
  std::memcpy(h, t.grids.data(), g);
  std::memcpy(h + g, t.events.data(), e);
  std::memcpy(h + g + e, t.chunks.data(), c);
  return CLUE_OK;
}

// Stream part of the table upload. `record` marks the staging buffer free
// again once the copies are done; a captured run records that mark after its
// graph launch instead (an event recorded inside a capture cannot be waited on
// from the host).
clue_status copy_tables(clue_workspace* ws, const HostTables& t, cudaStream_t st, bool record) {
  const size_t g = t.grids.size() * sizeof(GridDesc);
  const size_t e = t.events.size() * sizeof(EventDesc);
  const size_t c = t.chunks.size() * sizeof(Chunk);
  const char* h = (const char*)ws->staging;
  cudaError_t err;
  if ((err = cudaMemcpyAsync(ws->b.grids, h, g, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (err = cudaMemcpyAsync(ws->b.events, h + g, e, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (err = cudaMemcpyAsync(ws->b.chunks, h + g + e, c, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail_cuda(err, "table upload");
  if (record && (err = cudaEventRecord(ws->staging_event, st)) != cudaSuccess)
    return fail_cuda(err, "table upload event");
  return CLUE_OK;
}

namespace {

bool same_bits(float a, float b) {
  uint32_t x, y;
  std::memcpy(&x, &a, 4);
  std::memcpy(&y, &b, 4);
  return x == y;
}

bool same_params(const clue_params& a, const clue_params& b) {
  bool same = same_bits(a.dc, b.dc) && same_bits(a.rhoc, b.rhoc) && same_bits(a.dm, b.dm) &&
              same_bits(a.seed_dc, b.seed_dc) && a.kernel_kind == b.kernel_kind &&
              same_bits(a.kernel_params[0], b.kernel_params[0]) &&
              same_bits(a.kernel_params[1], b.kernel_params[1]) && a.metric_kind == b.metric_kind &&
              a.points_per_tile == b.points_per_tile;
  for (int d = 0; d < CLUE_MAX_DIM; ++d)
    same = same && a.wrapped[d] == b.wrapped[d] && same_bits(a.metric_params[d], b.metric_params[d]);
  return same;
}

bool same_points(const clue_points& a, const clue_points& b) {
  bool same = a.ndim == b.ndim && a.n == b.n && a.weight == b.weight &&
              a.density_uncertainty == b.density_uncertainty && a.tags == b.tags &&
              a.cluster_index == b.cluster_index && a.is_seed == b.is_seed && a.rho == b.rho &&
              a.nearest_higher == b.nearest_higher;
  for (int d = 0; same && d < a.ndim; ++d)
    same = a.coords[d] == b.coords[d] && a.sigma[d] == b.sigma[d];
  return same;
}

// Whether a run with these arguments is the one the cached graph was captured for.
bool graph_matches(const clue_workspace* ws, const clue_params* params, const clue_points* pts,
                   const uint32_t* sizes, int32_t n_events, int32_t grid_mode, int64_t staged) {
  const auto& k = ws->graph_key;
  if (!ws->graph_exec || k.grid_mode != grid_mode || k.staged != staged || k.base != ws->base ||
      (int64_t)k.sizes.size() != n_events || !same_params(k.params, *params) ||
      !same_points(k.points, *pts) ||
      std::memcmp(&k.tuning, &ws->tuning, sizeof(clue_tuning)) != 0)
    return false;
  return std::memcmp(k.sizes.data(), sizes, sizeof(uint32_t) * (size_t)n_events) == 0;
}

}  // namespace

clue_status upload_tables(clue_workspace* ws, const HostTables& t, cudaStream_t st) {
  clue_status s = stage_tables(ws, t);
  return s != CLUE_OK ? s : copy_tables(ws, t, st, true);
}

// One run on device-resident points. `sizes` is the host event table. With
// graphs on (and a non-default stream, no stage timing), the run is captured
// into a CUDA graph, and a later run with identical arguments replays it: no
// table building, no per-kernel launches, one graph launch.
clue_status run_device(clue_workspace* ws, const clue_params* params, const clue_points* pts,
                       const uint32_t* sizes, int32_t n_events, int32_t grid_mode,
                       cudaStream_t st, int64_t staged, const Piece* piece) {
  clue_status s = check_params(params);
  if (s != CLUE_OK)
    return s;
  if ((s = check_points(pts, true, params->metric_kind)) != CLUE_OK)
    return s;
  cudaError_t e = cudaSetDevice(ws->device);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  const bool use_graph = ws->graphs && !ws->profiling && st != nullptr && piece == nullptr;
  if (use_graph && graph_matches(ws, params, pts, sizes, n_events, grid_mode, staged)) {
    if ((e = cudaGraphLaunch(ws->graph_exec, st)) != cudaSuccess ||
        (e = cudaEventRecord(ws->staging_event, st)) != cudaSuccess)
      return fail_cuda(e, "graph launch");
    cudaEventRecord(ws->run_event, st);
    ws->has_run = true;
    ws->graph_replays_last = true;
    return CLUE_OK;
  }
  ws->graph_replays_last = false;
  // A piece of a pipelined batch comes with its tables built, checked against
  // the buffers and already on the device.
  const HostTables& t = ws->tables.tables;  // unused by a piece, whose tables are up already
  if (!piece) {
    const char* err = nullptr;
    if (!shape_tables(ws, pts->ndim, sizes, n_events, grid_mode, params->points_per_tile, &err))
      return fail(CLUE_ERR_INVALID_ARGUMENT, err);
  }
  const RunShape& sh = piece ? *piece->shape : ws->tables.shape;
  DeviceBuffers b = ws->b;
  if (piece) {
    b.grids = piece->grids;
    b.events = piece->events;
    b.chunks = piece->chunks;
  } else {
    if (sh.n != pts->n)
      return fail(CLUE_ERR_INVALID_ARGUMENT, "the event sizes do not add up to the number of points");
    bool any_sigma = false;
    for (int d = 0; d < pts->ndim; ++d)
      any_sigma |= pts->sigma[d] != nullptr;
    if ((s = ensure_capacity(ws, sh, any_sigma, pts->density_uncertainty != nullptr,
                             pts->tags != nullptr, staged)) != CLUE_OK)
      return s;
    b = ws->b;
    if ((s = stage_tables(ws, t)) != CLUE_OK)
      return s;
    if (ws->graph_exec) {  // the cached graph reads the staging buffer just overwritten
      if ((e = cudaGraphExecDestroy(ws->graph_exec)) != cudaSuccess)
        return fail_cuda(e, "graph release");
      ws->graph_exec = nullptr;
    }
  }
  // a failure of an earlier call whose status was not read would show up as
  // this run's launch error
  if ((e = cudaGetLastError()) != cudaSuccess)
    return fail_cuda(e, "a CUDA error left pending before this run");
  RunIO io;
  for (int d = 0; d < pts->ndim; ++d) {
    io.coords[d] = pts->coords[d];
    io.sigma[d] = pts->sigma[d];
  }
  io.weight = pts->weight;
  io.unc = pts->density_uncertainty;
  io.tags = pts->tags;
  io.cluster_index = pts->cluster_index;
  io.is_seed = pts->is_seed;
  io.rho = pts->rho;
  io.nh = pts->nearest_higher;
  if (piece) {
    io.piece_base = piece->base;
    io.point_base = piece->point_base;
    io.event_base = piece->event_base;
  }
  io.stats = ws->profiling && !piece ? ws->b.stats : nullptr;
  const RunParams prm = make_run_params(params, pts, ws->tuning);
  reset_launch_count();
  if (sh.max_event_points <= kLocalLabelPoints)
    local_labels_ready(sh.max_event_points);  // a device attribute: set before any capture
  if (use_graph && (e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return fail_cuda(e, "stream capture");
  // Everything from here to the end of the capture is stream work.
  if (!piece)
    s = copy_tables(ws, t, st, !use_graph);
  if (s == CLUE_OK && (e = launch_run(sh, prm, io, b, st, ws->profiling ? ws->marks : nullptr)) !=
                          cudaSuccess)
    s = fail_cuda(e, "kernel launch");
  // Seed count and status word come back with the run (read when needed); a
  // pipelined batch reads them once, after its last piece.
  if (s == CLUE_OK && !piece &&
      ((e = cudaMemcpyAsync(&ws->info->n_seeds, ws->b.counters + 1, sizeof(int32_t),
                            cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
       (e = cudaMemcpyAsync(&ws->info->status, ws->b.status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            st)) != cudaSuccess))
    s = fail_cuda(e, "result copy");
  if (use_graph) {
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st, &graph);
    if (s == CLUE_OK && ec != cudaSuccess)
      s = fail_cuda(ec, "stream capture");
    if (s == CLUE_OK && (e = cudaGraphInstantiate(&ws->graph_exec, graph, 0)) != cudaSuccess) {
      ws->graph_exec = nullptr;
      s = fail_cuda(e, "graph instantiation");
    }
    if (graph)
      cudaGraphDestroy(graph);
    if (s == CLUE_OK && ((e = cudaGraphLaunch(ws->graph_exec, st)) != cudaSuccess ||
                         (e = cudaEventRecord(ws->staging_event, st)) != cudaSuccess))
      s = fail_cuda(e, "graph launch");
    if (s == CLUE_OK) {
      auto& k = ws->graph_key;
      k.params = *params;
      k.points = *pts;
      k.tuning = ws->tuning;
      k.grid_mode = grid_mode;
      k.staged = staged;
      k.base = ws->base;
      k.sizes.assign(sizes, sizes + n_events);
    }
  }
  if (s != CLUE_OK)
    return s;
  ws->last_launches = launch_count();
  cudaEventRecord(ws->run_event, st);
  ws->has_run = true;
  ws->last_n = sh.n;
  if (!piece)
    ws->last_events = t.events;
  ws->last_labels = pts->cluster_index;
  return CLUE_OK;
}

clue_status wait_run(clue_workspace* ws) {
  if (!ws->has_run)
    return fail(CLUE_ERR_RUNTIME, "Seeds are not available. Please run make_clusters first.");
  cudaError_t e = cudaEventSynchronize(ws->run_event);
  if (e != cudaSuccess)
    return fail_cuda(e, "run");
  if (ws->info->status != 0)
    return fail(CLUE_ERR_TIMEOUT, "a bounded device-side wait gave up (status " +
                                      std::to_string(ws->info->status) + ")");
  return CLUE_OK;
}

// Copies points [first, first + count) of a host point set into the
// workspace's staging buffers, which are laid out for all h->n points, and
// points `dev` at them (a point set of `count` points).
clue_status stage_inputs(clue_workspace* ws, const clue_points* h, clue_points* dev,
                         cudaStream_t st, int64_t first, int64_t count) {
  const int64_t n = h->n;
  const int64_t o = first, m = count < 0 ? n - first : count;
  const int D = h->ndim;
  *dev = *h;
  dev->n = m;
  cudaError_t e;
  for (int d = 0; d < D; ++d) {
    float* dst = ws->b.in_coords + d * n + o;
    if ((e = cudaMemcpyAsync(dst, h->coords[d] + o, m * sizeof(float), cudaMemcpyHostToDevice, st)))
      return fail_cuda(e, "coordinate upload");
    dev->coords[d] = dst;
    if (h->sigma[d]) {
      float* sd = ws->b.in_sigma + d * n + o;
      if ((e = cudaMemcpyAsync(sd, h->sigma[d] + o, m * sizeof(float), cudaMemcpyHostToDevice, st)))
        return fail_cuda(e, "sigma upload");
      dev->sigma[d] = sd;
    }
  }
  if ((e = cudaMemcpyAsync(ws->b.in_weight + o, h->weight + o, m * sizeof(float),
                           cudaMemcpyHostToDevice, st)))
    return fail_cuda(e, "weight upload");
  dev->weight = ws->b.in_weight + o;
  if (h->density_uncertainty) {
    if ((e = cudaMemcpyAsync(ws->b.in_unc + o, h->density_uncertainty + o, m * sizeof(float),
                             cudaMemcpyHostToDevice, st)))
      return fail_cuda(e, "uncertainty upload");
    dev->density_uncertainty = ws->b.in_unc + o;
  }
  if (h->tags) {
    if ((e = cudaMemcpyAsync(ws->b.in_tags + o, h->tags + o, m * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, st)))
      return fail_cuda(e, "tag upload");
    dev->tags = ws->b.in_tags + o;
  }
  dev->cluster_index = ws->b.out_cluster + o;
  dev->is_seed = h->is_seed ? ws->b.out_seed + o : nullptr;
  dev->rho = h->rho ? ws->b.out_rho + o : nullptr;
  dev->nearest_higher = h->nearest_higher ? ws->b.out_nh + o : nullptr;
  return CLUE_OK;
}

// Copies the results of points [first, first + count) back to the host point set.
clue_status fetch_outputs(clue_workspace* ws, const clue_points* h, cudaStream_t st, int64_t first,
                          int64_t count) {
  const size_t o = (size_t)first, m = (size_t)(count < 0 ? h->n - first : count);
  const auto down = [&](void* dst, const void* src) {
    return cudaMemcpyAsync((char*)dst + 4 * o, (const char*)src + 4 * o, 4 * m,
                           cudaMemcpyDeviceToHost, st);
  };
  cudaError_t e;
  if ((e = down(h->cluster_index, ws->b.out_cluster)) ||
      (h->is_seed && (e = down(h->is_seed, ws->b.out_seed))) ||
      (h->rho && (e = down(h->rho, ws->b.out_rho))) ||
      (h->nearest_higher && (e = down(h->nearest_higher, ws->b.out_nh))))
    return fail_cuda(e, "result download");
  return CLUE_OK;
}

namespace {

// Host batches of at least kPieceMinPoints points with one grid per event run
// as up to kMaxPieces pieces of whole events, so that the upload of a piece
// overlaps the clustering of the one before it and its download the clustering
// of the one after. Events are independent under per-event grids, so a piece's
// results are those of the whole batch; the pieces only renumber (Piece).
constexpr int64_t kPieceMinPoints = int64_t(1) << 22;
constexpr int kMaxPieces = 4;

// Event boundaries of the pieces: cuts[p] .. cuts[p + 1], in shares of the
// points of 1:2 (two pieces), 1:3:2 (three) and 1:3:8:1 (four). Clustering
// starts after the first piece's upload and the call ends after the last
// piece's download, so both are small; the upload of a piece (about 2.9 times
// faster than its clustering, on the benchmark batch) must still finish
// while the piece before it clusters, which bounds each share at about 2.9
// times the one before. Downloads move 4 bytes per point against 12 up, so
// the last piece's download hides a share up to about 8.7 times its own.
std::vector<int32_t> piece_cuts(const uint32_t* sizes, int32_t n_events, int64_t n) {
  const int64_t k = std::min<int64_t>({kMaxPieces, n / kPieceMinPoints, n_events});
  static constexpr int64_t kShares[kMaxPieces + 1][kMaxPieces] = {
      {0, 0, 0, 0}, {1, 0, 0, 0}, {1, 2, 0, 0}, {1, 3, 2, 0}, {1, 3, 8, 1}};
  std::vector<int64_t> ends;  // cumulative shares
  int64_t shares = 0;
  for (int64_t p = 0; p < k; ++p)
    ends.push_back(shares += kShares[k][p]);
  std::vector<int32_t> cuts{0};
  int64_t acc = 0, at_cut = 0;
  for (int32_t e = 0; e < n_events; ++e) {
    acc += sizes[e];
    const size_t p = cuts.size() - 1;  // the piece this event ends up in
    // every piece holds points: events of size 0 never make a piece alone
    if ((int64_t)p + 1 < k && e + 1 < n_events && acc * shares >= ends[p] * n && acc > at_cut &&
        acc < n) {
      cuts.push_back(e + 1);
      at_cut = acc;
    }
  }
  cuts.push_back(n_events);
  return cuts;
}

}  // namespace

clue_status pipeline_pieces(clue_workspace* ws, const clue_params* params, const clue_points* h,
                            const uint32_t* sizes, cudaStream_t st, const HostTables& whole,
                            const HostTables& all, const std::vector<int32_t>& cuts,
                            const std::vector<Piece>& pieces);

// The pipelined form of run_host (see kPieceMinPoints). Returns false, having
// enqueued nothing, when the batch does not split; else the call's status is
// in *out.
bool run_host_pieces(clue_workspace* ws, const clue_params* params, const clue_points* h,
                     const uint32_t* sizes, int32_t n_events, cudaStream_t st,
                     const HostTables& whole, bool any_sigma, clue_status* out) {
  // The split depends on the tables alone: it is made once per table build
  // (ws->tables, whose tables `whole` are) and reused by calls of the same shape.
  clue_workspace::TableCache& c = ws->tables;
  if (!c.split) {
    c.cuts = piece_cuts(sizes, n_events, h->n);
    const int P = (int)c.cuts.size() - 1;
    if (P >= 2) {
      // Each piece's tables, and all of them end to end: piece p runs on its
      // slice of the table buffers, so one upload ahead of the points serves
      // every piece. With one grid per event a piece's tables are its events'
      // part of the whole batch's, counted from the piece's first point, tile,
      // event, chunk and stable-binning run.
      HostTables& all = c.all;
      all = whole;
      c.shapes.assign(P, RunShape{});
      c.first.assign(P + 1, 0);
      c.chunk_at.assign(P + 1, all.chunks.size());  // chunks are in event order
      for (size_t k = 0, p = 0; p < (size_t)P; ++p) {
        while (k < all.chunks.size() && all.chunks[k].event < c.cuts[p])
          ++k;
        c.chunk_at[p] = k;
      }
      for (int p = 0; p < P; ++p) {
        const int32_t c0 = c.cuts[p], c1 = c.cuts[p + 1];
        const EventDesc e0 = all.events[c0];
        RunShape& sh = c.shapes[p];
        sh.D = h->ndim;
        sh.n_events = sh.n_grids = c1 - c0;
        sh.n_chunks = (int32_t)(c.chunk_at[p + 1] - c.chunk_at[p]);
        int64_t warps = 0, entries = 0;
        for (int32_t e = c0; e < c1; ++e) {
          EventDesc& ev = all.events[e];
          const int64_t T = all.grids[e].T;
          sh.n += ev.n;
          sh.n_tiles += T;
          warps += ev.sort_chunks;
          entries += T * ev.sort_chunks;
          sh.max_event_tiles = (int32_t)std::max<int64_t>(sh.max_event_tiles, T);
          sh.max_event_points = std::max(sh.max_event_points, ev.n);
          ev.begin -= e0.begin;
          ev.tile_base -= e0.tile_base;
          ev.grid -= c0;
          ev.sort_first -= e0.sort_first;
          ev.sort_base -= e0.sort_base;
        }
        order_by_size(all.events.data() + c0, c1 - c0);
        for (size_t k = c.chunk_at[p]; k < c.chunk_at[p + 1]; ++k) {
          Chunk& ch = all.chunks[k];
          ch.event -= c0;
          ch.begin -= e0.begin;
          ch.end -= e0.begin;
        }
        sh.stable = sh.max_event_tiles <= kStableMaxTiles && entries <= 4 * sh.n && warps < INT32_MAX;
        sh.sort_warps = (int32_t)std::min<int64_t>(warps, INT32_MAX);
        sh.sort_entries = entries;
        c.first[p + 1] = c.first[p] + sh.n;
      }
    }
    c.split = true;
  }
  const int P = (int)c.cuts.size() - 1;
  if (P < 2)
    return false;
  // every piece must fit the buffers sized for the whole batch: nothing may
  // be reallocated under the uploads in flight
  for (int p = 0; p < P; ++p)
    if (!capacity_fits(ws, c.shapes[p], any_sigma, h->density_uncertainty != nullptr, h->tags != nullptr,
                       h->n))
      return false;
  if ((int64_t)c.all.grids.size() > ws->cap.grids || (int64_t)c.all.events.size() > ws->cap.events ||
      (int64_t)c.all.chunks.size() > ws->cap.chunks)
    return false;
  std::vector<Piece> pieces(P);
  for (int p = 0; p < P; ++p) {
    Piece& q = pieces[p];
    q.base = ws->b.counters + 8;
    q.point_base = c.first[p];
    q.event_base = c.cuts[p];
    q.shape = &c.shapes[p];
    q.grids = ws->b.grids + c.cuts[p];
    q.events = ws->b.events + c.cuts[p];
    q.chunks = ws->b.chunks + c.chunk_at[p];
  }
  *out = pipeline_pieces(ws, params, h, sizes, st, whole, c.all, c.cuts, pieces);
  return true;
}

// Stream order: [tables] on st, then the point uploads of every piece on `up`;
// piece p clusters on st once its upload is in, and its results go back on
// `down` once it is clustered, while the next piece clusters.
clue_status pipeline_pieces(clue_workspace* ws, const clue_params* params, const clue_points* h,
                            const uint32_t* sizes, cudaStream_t st, const HostTables& whole,
                            const HostTables& all, const std::vector<int32_t>& cuts,
                            const std::vector<Piece>& pieces) {
  const int P = (int)pieces.size();
  cudaError_t e;
  if (!ws->up && (e = cudaStreamCreateWithFlags(&ws->up, cudaStreamNonBlocking)))
    return fail_cuda(e, "upload stream");
  if (!ws->down && (e = cudaStreamCreateWithFlags(&ws->down, cudaStreamNonBlocking)))
    return fail_cuda(e, "download stream");
  // events: [0] tables up, [1] downloads done, then per piece uploaded and clustered
  const size_t n_ev = 2 + 2 * (size_t)kMaxPieces;
  while (ws->piece_events.size() < n_ev) {
    cudaEvent_t ev;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)))
      return fail_cuda(e, "piece event");
    ws->piece_events.push_back(ev);
  }
  cudaEvent_t* ev = ws->piece_events.data();
  cudaEvent_t *uploaded = ev + 2, *clustered = ev + 2 + kMaxPieces;
  clue_status s = stage_tables(ws, all);
  if (s != CLUE_OK)
    return s;
  if (ws->graph_exec) {  // the cached graph reads the staging buffer just overwritten
    if ((e = cudaGraphExecDestroy(ws->graph_exec)) != cudaSuccess)
      return fail_cuda(e, "graph release");
    ws->graph_exec = nullptr;
  }
  if ((e = cudaGetLastError()) != cudaSuccess)
    return fail_cuda(e, "a CUDA error left pending before this run");
  if ((s = copy_tables(ws, all, st, true)) != CLUE_OK)
    return s;
  if ((e = cudaEventRecord(ev[0], st)) || (e = cudaStreamWaitEvent(ws->up, ev[0], 0)))
    return fail_cuda(e, "piece ordering");
  // From here on work is in flight on `up`: every return first waits for it.
  const auto settle = [&](clue_status r) {
    cudaStreamSynchronize(ws->up);
    cudaStreamSynchronize(ws->down);
    return r;
  };
  std::vector<clue_points> dev(P);
  for (int p = 0; p < P && s == CLUE_OK; ++p) {
    s = stage_inputs(ws, h, &dev[p], ws->up, pieces[p].point_base, pieces[p].shape->n);
    if (s == CLUE_OK && (e = cudaEventRecord(uploaded[p], ws->up)))
      s = fail_cuda(e, "piece ordering");
  }
  int32_t* base = pieces[0].base;
  if (s == CLUE_OK && (e = launch_fill32(base, 1, 0, st)))
    s = fail_cuda(e, "piece base");
  int64_t launches = 1;
  for (int p = 0; p < P && s == CLUE_OK; ++p) {
    if ((e = cudaStreamWaitEvent(st, uploaded[p], 0))) {
      s = fail_cuda(e, "piece ordering");
      break;
    }
    s = run_device(ws, params, &dev[p], sizes + cuts[p], cuts[p + 1] - cuts[p], CLUE_GRID_PER_EVENT,
                   st, h->n, &pieces[p]);
    launches += ws->last_launches;
    if (s == CLUE_OK && (e = cudaEventRecord(clustered[p], st)))
      s = fail_cuda(e, "piece ordering");
  }
  for (int p = 0; p < P && s == CLUE_OK; ++p) {
    if ((e = cudaStreamWaitEvent(ws->down, clustered[p], 0)))
      s = fail_cuda(e, "piece ordering");
    else
      s = fetch_outputs(ws, h, ws->down, pieces[p].point_base, pieces[p].shape->n);
  }
  if (s == CLUE_OK && ((e = cudaEventRecord(ev[1], ws->down)) || (e = cudaStreamWaitEvent(st, ev[1], 0))))
    s = fail_cuda(e, "piece ordering");
  // the batch's cluster count is where the last piece left the base
  if (s == CLUE_OK &&
      ((e = cudaMemcpyAsync(&ws->info->n_seeds, base, sizeof(int32_t), cudaMemcpyDeviceToHost, st)) ||
       (e = cudaMemcpyAsync(&ws->info->status, ws->b.status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            st))))
    s = fail_cuda(e, "result copy");
  if (s != CLUE_OK)
    return settle(s);
  cudaEventRecord(ws->run_event, st);
  ws->last_n = h->n;
  ws->last_events = whole.events;
  ws->last_labels = ws->b.out_cluster;
  ws->last_launches = launches;
  ws->last_pieces = P;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
    return settle(fail_cuda(e, "stream synchronize"));
  return wait_run(ws);
}

clue_status run_host(clue_workspace* ws, const clue_params* params, const clue_points* h,
                     const uint32_t* sizes, int32_t n_events, int32_t grid_mode, cudaStream_t st) {
  clue_status s = check_params(params);
  if (s != CLUE_OK)
    return s;
  if ((s = check_points(h, true, params->metric_kind)) != CLUE_OK)
    return s;
  // Make sure the staging buffers exist before copying into them.
  const char* err = nullptr;
  if (!shape_tables(ws, h->ndim, sizes, n_events, grid_mode, params->points_per_tile, &err))
    return fail(CLUE_ERR_INVALID_ARGUMENT, err);
  const HostTables& t = ws->tables.tables;
  const RunShape& sh = ws->tables.shape;
  if (sh.n != h->n)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "the event sizes do not add up to the number of points");
  bool any_sigma = false;
  for (int d = 0; d < h->ndim; ++d)
    any_sigma |= h->sigma[d] != nullptr;
  cudaError_t e = cudaSetDevice(ws->device);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  if ((s = ensure_capacity(ws, sh, any_sigma, h->density_uncertainty != nullptr, h->tags != nullptr,
                           h->n)) != CLUE_OK)
    return s;
  if (grid_mode == CLUE_GRID_PER_EVENT && n_events > 1 && h->n >= 2 * kPieceMinPoints &&
      !ws->profiling) {
    if (run_host_pieces(ws, params, h, sizes, n_events, st, t, any_sigma, &s))
      return s;
  }
  ws->last_pieces = 1;
  clue_points dev;
  if ((s = stage_inputs(ws, h, &dev, st)) != CLUE_OK)
    return s;
  if ((s = run_device(ws, params, &dev, sizes, n_events, grid_mode, st, h->n)) != CLUE_OK)
    return s;
  if ((s = fetch_outputs(ws, h, st)) != CLUE_OK)
    return s;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
    return fail_cuda(e, "stream synchronize");
  return wait_run(ws);
}

}  // namespace clue_impl

// ---------------------------------------------------------------------------
// extern "C"
// ---------------------------------------------------------------------------

extern "C" {

int32_t clue_abi_version(void) { return CLUE_ABI_VERSION; }

const char* clue_status_string(clue_status s) {
  switch (s) {
    case CLUE_OK: return "ok";
    case CLUE_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CLUE_ERR_OUT_OF_RANGE: return "out of range";
    case CLUE_ERR_RUNTIME: return "runtime error";
    case CLUE_ERR_CUDA: return "CUDA error";
    case CLUE_ERR_OUT_OF_MEMORY: return "out of memory";
    case CLUE_ERR_TIMEOUT: return "timeout";
    case CLUE_ERR_NOT_READY: return "not ready";
  }
  return "unknown status";
}

const char* clue_last_error(void) { return t_last_error.c_str(); }

clue_status clue_validate_params(const clue_params* params) { return check_params(params); }

clue_status clue_workspace_create(clue_workspace** out, int32_t device) {
  if (!out)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null output pointer");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaGetDeviceCount");
  if (device < 0 || device >= count)
    return fail(CLUE_ERR_OUT_OF_RANGE, "device index out of range");
  if ((e = cudaSetDevice(device)) != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  auto* ws = new clue_workspace();
  ws->device = device;
  ws->tuning = default_tuning();
  if ((e = cudaEventCreateWithFlags(&ws->run_event, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&ws->staging_event, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaMallocHost((void**)&ws->info, sizeof(RunInfo))) != cudaSuccess) {
    delete ws;
    return fail_cuda(e, "workspace creation");
  }
  std::memset(ws->info, 0, sizeof(RunInfo));
  *out = ws;
  return CLUE_OK;
}

clue_status clue_workspace_destroy(clue_workspace* ws) {
  if (!ws)
    return CLUE_OK;
  cudaSetDevice(ws->device);
  if (ws->has_run)
    cudaEventSynchronize(ws->run_event);
  if (ws->base)
    cudaFree(ws->base);
  if (ws->staging)
    cudaFreeHost(ws->staging);
  if (ws->info)
    cudaFreeHost(ws->info);
  if (ws->run_event)
    cudaEventDestroy(ws->run_event);
  if (ws->staging_event)
    cudaEventDestroy(ws->staging_event);
  for (auto& m : ws->marks)
    if (m)
      cudaEventDestroy(m);
  if (ws->graph_exec)
    cudaGraphExecDestroy(ws->graph_exec);
  for (cudaStream_t s : {ws->up, ws->down})
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  for (cudaEvent_t ev : ws->piece_events)
    cudaEventDestroy(ev);
  delete ws;
  return CLUE_OK;
}

clue_status clue_tuning_defaults(clue_tuning* out) {
  if (!out)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = default_tuning();
  return CLUE_OK;
}

clue_status clue_workspace_get_tuning(const clue_workspace* ws, clue_tuning* out) {
  if (!ws || !out)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  *out = ws->tuning;
  return CLUE_OK;
}

clue_status clue_workspace_set_tuning(clue_workspace* ws, const clue_tuning* tuning) {
  if (!ws || !tuning)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  if (tuning->density_union_x16_2d < 0 || tuning->density_union_x16_3d < 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "union thresholds must be >= 0");
  if (tuning->label_jump_rounds < -1 || tuning->label_jump_rounds > 4)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "label_jump_rounds must be in [-1, 4]");
  if (tuning->cell_points < 1 || tuning->cell_points > 8)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "cell_points must be in [1, 8]");
  if (tuning->density_shape < 0 || tuning->density_shape > 2 || tuning->nh_shape < 0 ||
      tuning->nh_shape > 2)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "density_shape and nh_shape must be in [0, 2]");
  if (tuning->tile_binning < 0 || tuning->tile_binning > 1)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "tile_binning must be 0 or 1");
  ws->tuning = *tuning;
  return CLUE_OK;
}

clue_status clue_selftest_bounded_wait(int32_t device, void* stream) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  // a zeroed descriptor (nothing ever publishes it) and a status word
  void* buf = nullptr;
  if ((e = cudaMalloc(&buf, 16)) != cudaSuccess)
    return fail_cuda(e, "self-test allocation");
  auto* desc = static_cast<unsigned long long*>(buf);
  auto* status = reinterpret_cast<uint32_t*>(desc + 1);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t host_status = 0;
  if ((e = cudaMemsetAsync(buf, 0, 16, st)) == cudaSuccess &&
      (e = launch_wait_probe(desc, status, st)) == cudaSuccess &&
      (e = cudaMemcpyAsync(&host_status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) ==
          cudaSuccess)
    e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (e != cudaSuccess)
    return fail_cuda(e, "bounded-wait self-test");
  if (host_status & kStatusScanTimeout)
    return fail(CLUE_ERR_TIMEOUT, "the bounded wait gave up and reported it (expected)");
  return fail(CLUE_ERR_RUNTIME, "the bounded wait did not report giving up");
}

clue_status clue_workspace_set_graphs(clue_workspace* ws, int32_t enable) {
  if (!ws)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace is null");
  ws->graphs = enable != 0;
  if (!ws->graphs && ws->graph_exec) {
    cudaSetDevice(ws->device);
    if (ws->has_run)
      cudaEventSynchronize(ws->run_event);
    cudaGraphExecDestroy(ws->graph_exec);
    ws->graph_exec = nullptr;
  }
  return CLUE_OK;
}

clue_status clue_workspace_graph_replayed(const clue_workspace* ws, int32_t* replayed) {
  if (!ws || !replayed)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  *replayed = ws->graph_replays_last ? 1 : 0;
  return CLUE_OK;
}

clue_status clue_workspace_host_pieces(const clue_workspace* ws, int32_t* pieces) {
  if (!ws || !pieces)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  *pieces = ws->last_pieces;
  return CLUE_OK;
}

clue_status clue_workspace_set_profiling(clue_workspace* ws, int32_t enable) {
  if (!ws)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace is null");
  if (enable && !ws->marks[0]) {
    cudaSetDevice(ws->device);
    for (auto& m : ws->marks) {
      cudaError_t e = cudaEventCreate(&m);
      if (e != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    }
  }
  ws->profiling = enable != 0;
  return CLUE_OK;
}

clue_status clue_workspace_stage_ms(clue_workspace* ws, float* stage_ms, int32_t capacity) {
  if (!ws || !stage_ms)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  if (!ws->profiling)
    return fail(CLUE_ERR_RUNTIME, "profiling is not enabled on this workspace");
  clue_status s = wait_run(ws);
  if (s != CLUE_OK)
    return s;
  for (int i = 0; i < kStages && i < capacity; ++i) {
    cudaError_t e = cudaEventElapsedTime(&stage_ms[i], ws->marks[i], ws->marks[i + 1]);
    if (e != cudaSuccess)
      return fail_cuda(e, "cudaEventElapsedTime");
  }
  return CLUE_OK;
}

clue_status clue_workspace_sweep_stats(clue_workspace* ws, int64_t* stats, int32_t capacity) {
  if (!ws || !stats)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  if (!ws->profiling)
    return fail(CLUE_ERR_RUNTIME, "profiling is not enabled on this workspace");
  if (!ws->has_run)
    return fail(CLUE_ERR_RUNTIME, "no run on this workspace yet");
  clue_status s = wait_run(ws);
  if (s != CLUE_OK)
    return s;
  unsigned long long v[8] = {};
  cudaError_t e = cudaMemcpy(v, ws->b.stats, sizeof v, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess)
    return fail_cuda(e, "statistics copy");
  for (int i = 0; i < CLUE_N_SWEEP_STATS && i < capacity; ++i)
    stats[i] = (int64_t)v[i];
  return CLUE_OK;
}

clue_status clue_workspace_kernel_launches(const clue_workspace* ws, int64_t* launches) {
  if (!ws || !launches)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  *launches = ws->has_run ? ws->last_launches : 0;
  return CLUE_OK;
}

clue_status clue_workspace_bytes(const clue_workspace* ws, size_t* bytes) {
  if (!ws || !bytes)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = ws->bytes;
  return CLUE_OK;
}

size_t clue_workspace_bytes_for(int32_t ndim, int64_t n_points, int64_t n_tiles, int32_t n_events) {
  RunShape s;
  s.D = ndim;
  s.n = n_points;
  s.n_tiles = n_tiles;
  s.n_events = n_events;
  s.n_grids = n_events;
  s.n_chunks = (int32_t)(n_events + n_points / kChunkPoints + 1);
  return scratch_bytes(s, false, false, false);
}

clue_status clue_make_clusters_device(clue_workspace* ws, const clue_params* params,
                                      const clue_points* points, void* stream) {
  if (!ws)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace is null");
  if (!points || points->n <= 0)
    return check_points(points, true, params ? params->metric_kind : 0);
  const uint32_t size = (uint32_t)points->n;
  return run_device(ws, params, points, &size, 1, CLUE_GRID_PER_EVENT, (cudaStream_t)stream, 0);
}

clue_status clue_workspace_autotune(clue_workspace* ws, const clue_params* params,
                                    const clue_points* points, const uint32_t* event_sizes,
                                    int32_t n_events, int32_t grid_mode, void* stream,
                                    int32_t reps, clue_tuning* chosen) {
  if (!ws || !params || !points)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace, parameters and points are required");
  if (event_sizes && n_events <= 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "n_events must be positive");
  if (event_sizes && grid_mode != CLUE_GRID_SHARED && grid_mode != CLUE_GRID_PER_EVENT)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "unknown grid mode");
  if (reps < 1 || reps > 100)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "reps must be in [1, 100]");
  if (points->n <= 0)
    return check_points(points, true, params->metric_kind);
  const uint32_t one = (uint32_t)points->n;
  const uint32_t* sizes = event_sizes ? event_sizes : &one;
  const int32_t ne = event_sizes ? n_events : 1;
  const int32_t gm = event_sizes ? grid_mode : CLUE_GRID_PER_EVENT;
  const cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaSetDevice(ws->device);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  cudaEvent_t ev[2] = {};
  for (auto& x : ev)
    if ((e = cudaEventCreate(&x)) != cudaSuccess)
      return fail_cuda(e, "cudaEventCreate");
  const clue_tuning start = ws->tuning;
  // candidates run uncaptured: every one has its own tuning
  const bool graphs = ws->graphs;
  ws->graphs = false;
  // Median device time of `reps` runs under t, after one warm-up run.
  auto time_runs = [&](const clue_tuning& t, float* ms) -> clue_status {
    ws->tuning = t;
    clue_status s = run_device(ws, params, points, sizes, ne, gm, st, 0);
    std::vector<float> v;
    for (int r = 0; r < reps && s == CLUE_OK; ++r) {
      cudaEventRecord(ev[0], st);
      s = run_device(ws, params, points, sizes, ne, gm, st, 0);
      cudaEventRecord(ev[1], st);
      if (s == CLUE_OK && (s = wait_run(ws)) == CLUE_OK) {
        float x = 0.0f;
        // the run's own completion event precedes ev[1] on the stream
        if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess ||
            (e = cudaEventElapsedTime(&x, ev[0], ev[1])) != cudaSuccess)
          s = fail_cuda(e, "cudaEventElapsedTime");
        v.push_back(x);
      }
    }
    if (s == CLUE_OK) {
      std::sort(v.begin(), v.end());
      *ms = v[v.size() / 2];
    }
    return s;
  };
  clue_tuning best = start;
  float best_ms = 0.0f;
  clue_status s = time_runs(best, &best_ms);
  // One field at a time, each candidate against the best so far.
  auto try_field = [&](int32_t clue_tuning::*field, std::initializer_list<int32_t> values) {
    const clue_tuning base = best;
    for (int32_t v : values) {
      if (s != CLUE_OK || v == base.*field)
        continue;
      clue_tuning t = base;
      t.*field = v;
      float ms = 0.0f;
      s = time_runs(t, &ms);
      if (s == CLUE_OK && ms < best_ms) {
        best = t;
        best_ms = ms;
      }
    }
  };
  // The union threshold, the cell size and the sweeps' block shapes matter on
  // the packed 2-D/3-D path only.
  if (points->ndim == 2)
    try_field(&clue_tuning::density_union_x16_2d, {0, 12, 16, 20, 24, 32, 48, 1 << 20});
  else if (points->ndim == 3)
    try_field(&clue_tuning::density_union_x16_3d, {0, 16, 24, 32, 48, 64, 1 << 20});
  if (points->ndim == 2 || points->ndim == 3) {
    try_field(&clue_tuning::cell_points, {1, 2, 3, 4});
    try_field(&clue_tuning::density_shape, {0, 1, 2});
    try_field(&clue_tuning::nh_shape, {0, 1, 2});
  }
  try_field(&clue_tuning::tile_binning, {0, 1});
  try_field(&clue_tuning::label_jump_rounds, {0, 1, 2, 3, 4});
  for (auto& x : ev)
    cudaEventDestroy(x);
  ws->tuning = s == CLUE_OK ? best : start;
  ws->graphs = graphs;
  if (s == CLUE_OK && chosen)
    *chosen = best;
  return s;
}

clue_status clue_make_clusters_host(clue_workspace* ws, const clue_params* params,
                                    const clue_points* points, void* stream) {
  if (!ws)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace is null");
  if (!points || points->n <= 0)
    return check_points(points, true, params ? params->metric_kind : 0);
  const uint32_t size = (uint32_t)points->n;
  return run_host(ws, params, points, &size, 1, CLUE_GRID_PER_EVENT, (cudaStream_t)stream);
}

clue_status clue_make_clusters_batched_device(clue_workspace* ws, const clue_params* params,
                                              const clue_points* points, const uint32_t* sizes,
                                              int32_t n_events, int32_t grid_mode, void* stream) {
  if (!ws || !sizes || n_events <= 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace, event sizes and n_events are required");
  if (grid_mode != CLUE_GRID_SHARED && grid_mode != CLUE_GRID_PER_EVENT)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "unknown grid mode");
  return run_device(ws, params, points, sizes, n_events, grid_mode, (cudaStream_t)stream, 0);
}

clue_status clue_make_clusters_batched_host(clue_workspace* ws, const clue_params* params,
                                            const clue_points* points, const uint32_t* sizes,
                                            int32_t n_events, int32_t grid_mode, void* stream) {
  if (!ws || !sizes || n_events <= 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace, event sizes and n_events are required");
  if (grid_mode != CLUE_GRID_SHARED && grid_mode != CLUE_GRID_PER_EVENT)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "unknown grid mode");
  return run_host(ws, params, points, sizes, n_events, grid_mode, (cudaStream_t)stream);
}

clue_status clue_n_clusters(clue_workspace* ws, int32_t* n_clusters) {
  if (!ws || !n_clusters)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  clue_status s = wait_run(ws);
  if (s != CLUE_OK)
    return s;
  *n_clusters = ws->info->n_seeds;
  return CLUE_OK;
}

clue_status clue_get_seeds(clue_workspace* ws, int32_t* seeds, int32_t capacity, int32_t* n_seeds) {
  if (!ws)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace is null");
  clue_status s = wait_run(ws);
  if (s != CLUE_OK)
    return s;
  const int32_t n = ws->info->n_seeds;
  if (n_seeds)
    *n_seeds = n;
  const int32_t m = std::min(n, std::max(capacity, 0));
  if (m > 0 && seeds) {
    cudaError_t e = cudaMemcpy(seeds, ws->b.seeds, sizeof(int32_t) * m, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
      return fail_cuda(e, "seed download");
  }
  return CLUE_OK;
}

clue_status clue_sample_associations(clue_workspace* ws, int32_t* offsets, int32_t capacity,
                                     int32_t* n_keys) {
  if (!ws)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "workspace is null");
  clue_status s = wait_run(ws);
  if (s != CLUE_OK)
    return s;
  const int32_t n = ws->info->n_seeds;
  std::vector<int32_t> ev(std::max(n, 1));
  if (n > 0) {
    cudaError_t e = cudaMemcpy(ev.data(), ws->b.seed_event, sizeof(int32_t) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
      return fail_cuda(e, "association download");
  }
  const int32_t B = (int32_t)ws->last_events.size();
  std::vector<int32_t> off(B + 1, 0);
  for (int32_t k = 0; k < n; ++k)
    off[ev[k] + 1] += 1;
  for (int32_t e = 0; e < B; ++e)
    off[e + 1] += off[e];
  if (offsets)
    for (int32_t e = 0; e <= B && e < capacity; ++e)
      offsets[e] = off[e];
  // make_associator sizes the map by the largest key + 1
  // (data_structures/internal/MakeAssociator.hpp:32-43).
  if (n_keys)
    *n_keys = n > 0 ? ev[n - 1] + 1 : 0;
  return CLUE_OK;
}

clue_status clue_get_clusters_device(clue_workspace* ws, int32_t* offsets, int32_t* points,
                                     void* stream) {
  if (!ws || !offsets || !points)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  clue_status s = wait_run(ws);
  if (s != CLUE_OK)
    return s;
  cudaError_t e = cudaSetDevice(ws->device);
  if (e == cudaSuccess)
    e = launch_clusters_csr(ws->b, ws->last_n, ws->last_labels, ws->info->n_seeds, offsets, points,
                            (cudaStream_t)stream);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cluster map");
}

clue_status clue_stream_create(void** stream, int32_t device) {
  if (!stream)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  cudaStream_t s;
  if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
    return fail_cuda(e, "cudaStreamCreate");
  *stream = s;
  return CLUE_OK;
}

clue_status clue_stream_destroy(void* stream) {
  cudaError_t e = cudaStreamDestroy((cudaStream_t)stream);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaStreamDestroy");
}

clue_status clue_stream_synchronize(void* stream) {
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaStreamSynchronize");
}

clue_status clue_device_malloc(void** ptr, size_t bytes, int32_t device) {
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess)
    e = cudaMalloc(ptr, bytes);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaMalloc");
}

clue_status clue_device_free(void* ptr) {
  cudaError_t e = cudaFree(ptr);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaFree");
}

clue_status clue_host_malloc_pinned(void** ptr, size_t bytes) {
  cudaError_t e = cudaMallocHost(ptr, bytes);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaMallocHost");
}

clue_status clue_host_free_pinned(void* ptr) {
  cudaError_t e = cudaFreeHost(ptr);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaFreeHost");
}

clue_status clue_memcpy_async(void* dst, const void* src, size_t bytes, int32_t kind, void* stream) {
  const cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                           : kind == 1 ? cudaMemcpyDeviceToHost
                                       : cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream);
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "cudaMemcpyAsync");
}

}  // extern "C"
