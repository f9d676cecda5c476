// noalloc.cu — clue_make_clusters_device_noalloc: the single-event run with
// every scratch buffer carved from one file-scope device array instead of a
// workspace allocation. The launch sequence is the library's usual one.

#include "abi_internal.h"

using namespace clue_impl;

namespace {

// The scratch of every no-allocation call on this device. It lives as long as
// the library stays loaded and keeps the last call's contents; the launch
// sequence clears everything that has to start at zero.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CLUE_NOALLOC_SCRATCH_BYTES];

// Device address of the current device's copy of g_noalloc_scratch. In host
// code the array's name is only a host-side stand-in, so the address is looked
// up with the device current. The lookup allocates nothing and runs on every
// call, so the address stays right after cudaDeviceReset or a new primary
// context loads the module elsewhere; the first call on a device may load the
// library's device code.
clue_status scratch_for_current_device(char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaGetSymbolAddress of the no-allocation scratch");
  *out = static_cast<char*>(p);
  return CLUE_OK;
}

// Writes the one-event tables into the scratch: grid, event and the chunks of
// kChunkPoints points (the same split the allocating path builds on the host).
__global__ void k_noalloc_tables(GridDesc g, EventDesc ev, int32_t chunk_points, GridDesc* grids,
                                 EventDesc* events, Chunk* chunks, int32_t n_chunks) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t n = ev.n;
  if (i == 0) {
    grids[0] = g;
    events[0] = ev;
  }
  if (i < n_chunks)
    chunks[i] = Chunk{0, i * chunk_points, min(n, (i + 1) * chunk_points)};
}

}  // namespace

extern "C" clue_status clue_make_clusters_device_noalloc(const clue_params* params,
                                                         const clue_points* pts,
                                                         uint32_t* device_status, void* stream) {
  clue_status s = check_params(params);
  if (s != CLUE_OK)
    return s;
  if ((s = check_points(pts, true, params->metric_kind)) != CLUE_OK)
    return s;
  if (pts->n > CLUE_NOALLOC_MAX_POINTS)
    return fail(CLUE_ERR_INVALID_ARGUMENT,
                "clue_make_clusters_device_noalloc accepts at most " +
                    std::to_string(CLUE_NOALLOC_MAX_POINTS) + " points per call (got " +
                    std::to_string(pts->n) + ")");
  const int D = pts->ndim;
  const int64_t n = pts->n;
  // Tile grid of the event (core/detail/SetupTiles.hpp:30-34), by the same
  // helpers the workspace path builds its tables with.
  const int ppt = params->points_per_tile > 0 ? params->points_per_tile : 128;
  int32_t k = 0;
  int64_t T = 0;
  if (!grid_shape(D, n, ppt, &k, &T))
    return fail(CLUE_ERR_INVALID_ARGUMENT, "tile grid too large");
  GridDesc g;
  fill_grid(&g, D, k, T);
  RunShape sh;
  sh.D = D;
  sh.n = n;
  sh.n_tiles = T;
  sh.n_events = 1;
  sh.n_grids = 1;
  sh.n_chunks = (int32_t)((n + kChunkPoints - 1) / kChunkPoints);
  // the one event and its stable-binning layout (as build_tables lays it out)
  EventDesc ev{0, (int32_t)n, 0, 0, 0, 0, 0, 0};
  ev.sort_chunks = sort_runs(n, &ev.sort_len);
  sh.sort_warps = ev.sort_chunks;
  sh.sort_entries = T * (int64_t)ev.sort_chunks;
  sh.max_event_tiles = (int32_t)T;
  sh.max_event_points = (int32_t)n;
  sh.stable = T <= kStableMaxTiles && sh.sort_entries <= 4 * n;

  bool any_sigma = false;
  for (int d = 0; d < D; ++d)
    any_sigma |= pts->sigma[d] != nullptr;
  Capacity cap;
  cap.points = n;
  cap.tiles = T;
  cap.events = 1;
  cap.chunks = sh.n_chunks;
  cap.grids = 1;
  cap.scan_blocks = scan_blocks_for(std::max<int64_t>(n, T));
  cap.dims = D;
  cap.sigma = any_sigma;
  cap.unc = pts->density_uncertainty != nullptr;
  cap.tags = pts->tags != nullptr;
  cap.cells = D == 2 || D == 3;
  DeviceBuffers b;
  if (carve_buffers(&b, cap, nullptr) > CLUE_NOALLOC_SCRATCH_BYTES)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "event does not fit the no-allocation scratch");

  char* base = nullptr;
  if ((s = scratch_for_current_device(&base)) != CLUE_OK)
    return s;
  carve_buffers(&b, cap, base);

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // a failure of an earlier call whose status was not read would otherwise
  // show up as this call's error
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail_cuda(e, "a CUDA error left pending before this run");
  e = cudaMemsetAsync(b.status, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess)
    return fail_cuda(e, "status reset");
  k_noalloc_tables<<<(sh.n_chunks + 31) / 32, 32, 0, st>>>(g, ev, kChunkPoints, b.grids, b.events,
                                                           b.chunks, sh.n_chunks);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return fail_cuda(e, "table setup");

  RunIO io;
  for (int d = 0; d < D; ++d) {
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
  if ((e = launch_run(sh, make_run_params(params, pts, default_tuning()), io, b, st)) != cudaSuccess)
    return fail_cuda(e, "kernel launch");
  if (device_status &&
      (e = cudaMemcpyAsync(device_status, b.status, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                           st)) != cudaSuccess)
    return fail_cuda(e, "status copy");
  return CLUE_OK;
}
