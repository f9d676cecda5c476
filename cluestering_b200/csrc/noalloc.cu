// noalloc.cu — clue_make_clusters_device_noalloc: the single-event run with
// every scratch buffer carved from one file-scope device array instead of a
// workspace allocation. The launch sequence is the library's usual one.
#include <cstring>
#include <mutex>

#include "abi_internal.h"

using namespace clue_impl;

namespace {

// The scratch of every no-allocation call on this device. It lives as long as
// the library stays loaded and keeps the last call's contents; the launch
// sequence clears everything that has to start at zero.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CLUE_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
char* g_scratch_addr[kMaxDevices] = {};

// Device address of this device's copy of g_noalloc_scratch. In host code the
// array's name is only a host-side stand-in, so the address has to be looked up
// once per device, with that device current.
clue_status scratch_for_current_device(char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return fail(CLUE_ERR_OUT_OF_RANGE, "device index out of range for the no-allocation path");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail_cuda(e, "cudaGetSymbolAddress");
    g_scratch_addr[dev] = static_cast<char*>(p);
  }
  *out = g_scratch_addr[dev];
  return CLUE_OK;
}

// Writes the one-event tables into the scratch: grid, event and the chunks of
// kChunkPoints points (the same split the allocating path builds on the host).
__global__ void k_noalloc_tables(GridDesc g, int32_t n, int32_t chunk_points, GridDesc* grids,
                                 EventDesc* events, Chunk* chunks, int32_t n_chunks) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    grids[0] = g;
    events[0] = EventDesc{0, n, 0, 0};
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
  // Tile grid of the event (core/detail/SetupTiles.hpp:30-34).
  const int ppt = params->points_per_tile > 0 ? params->points_per_tile : 128;
  const int64_t nt = (n + ppt - 1) / ppt;
  int64_t k = 1, T = 1;
  for (;; ++k) {
    T = 1;
    for (int d = 0; d < D; ++d)
      T *= k;
    if (T >= nt)
      break;
  }
  GridDesc g;
  std::memset(&g, 0, sizeof g);
  g.k = (int32_t)k;
  g.T = (int32_t)T;
  for (int d = D - 1, stride = 1; d >= 0; --d, stride *= (int)k)
    g.stride[d] = stride;
  constexpr int kChunkPoints = 4096;
  RunShape sh;
  sh.D = D;
  sh.n = n;
  sh.n_tiles = T;
  sh.n_events = 1;
  sh.n_grids = 1;
  sh.n_chunks = (int32_t)((n + kChunkPoints - 1) / kChunkPoints);

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
  cudaError_t e = cudaMemsetAsync(b.status, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess)
    return fail_cuda(e, "status reset");
  k_noalloc_tables<<<(sh.n_chunks + 31) / 32, 32, 0, st>>>(g, (int32_t)n, kChunkPoints, b.grids,
                                                           b.events, b.chunks, sh.n_chunks);
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
