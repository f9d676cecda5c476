// engine.h — host-side interface between the C ABI / serving layer and the
// CUDA kernels of one clustering run.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"

namespace clue_impl {

// Device buffers of one workspace. Sizes grow on demand and never shrink.
struct DeviceBuffers {
  // tables
  GridDesc* grids = nullptr;
  EventDesc* events = nullptr;
  Chunk* chunks = nullptr;
  int32_t* grid_minmax = nullptr;  // 2*D ordered ints per grid (min, max)
  // per point (original order)
  int32_t* tile_of = nullptr;
  int32_t* point_event = nullptr;
  int32_t* nh = nullptr;           // nearest higher when the caller does not want it
  int32_t* seed_flag = nullptr;
  int32_t* seed_rank = nullptr;
  int32_t* parent = nullptr;
  // per tile
  int32_t* tile_count = nullptr;
  int32_t* tile_offset = nullptr;  // T + 1
  int32_t* tile_cursor = nullptr;
  // per sorted position
  int32_t* perm = nullptr;         // sorted position -> original index
  int32_t* sorted_event = nullptr;
  float* sorted_coords = nullptr;  // D planes of n
  float* sorted_weight = nullptr;
  float* sorted_sigma = nullptr;   // D planes when sigma is set
  float* sorted_unc = nullptr;
  uint32_t* sorted_tag = nullptr;
  float* sorted_rho = nullptr;
  int32_t* merge_tmp = nullptr;
  // sweep processing order and packed candidate records
  int32_t* work_dens = nullptr;
  int32_t* work_nh = nullptr;
  int32_t* cls_dens = nullptr;
  int32_t* cls_nh = nullptr;
  float4* rec_dens = nullptr;
  float4* rec_nh = nullptr;
  float4* rec_cell = nullptr;      // density records in cell-layout order
  int32_t* event_exact = nullptr;  // 4 per event: bounds for exact-sum density
  uint32_t* rec_tag = nullptr;
  // cell layout of the nearest-higher search (D = 2 or 3)
  int32_t* nh_pos = nullptr;
  int32_t* nh_q = nullptr;
  int32_t* cell_slot = nullptr;
  int32_t* cell_s = nullptr;       // per tile
  float4* cell_geom = nullptr;     // 2 per tile
  CellInfo* cell_info = nullptr;   // per sorted position (slot)
  float4* cell_box = nullptr;      // 2 per slot
  // seeds
  int32_t* seeds = nullptr;
  int32_t* seed_event = nullptr;
  // scan state
  unsigned long long* scan_desc = nullptr;
  int32_t* counters = nullptr;     // [0] scan ticket, [1] n_seeds, [2] oversize count, [3] large count,
                                   // [4..5] sweep work queues, [6] label queue, [7] some event not
                                   // order-free (tile sorts), [8] cluster-id base of a pipelined piece
  int32_t* large_tiles = nullptr;  // tiles too large for the per-warp sort
  int32_t* oversize = nullptr;     // tiles needing a chunk merge
  uint32_t* status = nullptr;
  unsigned long long* stats = nullptr;  // sweep statistics of a profiled run (8 counters)
  // staged inputs/outputs for the host entry points
  float* in_coords = nullptr;
  float* in_weight = nullptr;
  float* in_sigma = nullptr;
  float* in_unc = nullptr;
  uint32_t* in_tags = nullptr;
  int32_t* out_cluster = nullptr;
  int32_t* out_seed = nullptr;
  float* out_rho = nullptr;
  int32_t* out_nh = nullptr;
};

struct Capacity {
  int64_t points = 0, tiles = 0, events = 0, chunks = 0, grids = 0, scan_blocks = 0;
  int32_t dims = 0;
  bool sigma = false, unc = false, tags = false;
  bool cells = false;  // cell layout of the nearest-higher search (2-D and 3-D runs)
  int64_t staged_points = 0;
};

struct RunShape {
  int32_t D = 0;
  int64_t n = 0;
  int64_t n_tiles = 0;
  int32_t n_events = 0;
  int32_t n_grids = 0;
  int32_t n_chunks = 0;
  // Stable tile binning (one warp per run of consecutive points of an event):
  // usable when every event has at most kStableMaxTiles tiles and the count
  // matrices of all events hold at most 4 n entries (they live in the
  // nearest-higher records, 16 bytes per point, free until the sweeps).
  bool stable = false;
  int32_t sort_warps = 0;
  int64_t sort_entries = 0;
  int32_t max_event_tiles = 0;
  int32_t max_event_points = 0;  // points of the largest event
};

// Runs of the stable binning for an event of n points: one per kStableRun
// points, at least one. Returns the run count; *len = points per run.
int32_t sort_runs(int64_t n, int32_t* len);

// Largest event whose labels launch_run walks in shared memory (one grid per
// event); local_labels_ready(points) grants that kernel the shared memory of
// an event of `points` points on the current device (outside stream capture,
// once per device). False when the device refuses: the run then labels in
// global memory.
constexpr int32_t kLocalLabelPoints = 1 << 16;
bool local_labels_ready(int32_t points);

// Pointers of one run's inputs and outputs (device memory).
struct RunIO {
  const float* coords[kMaxDim] = {};
  const float* weight = nullptr;
  const float* sigma[kMaxDim] = {};
  const float* unc = nullptr;
  const uint32_t* tags = nullptr;
  int32_t* cluster_index = nullptr;
  int32_t* is_seed = nullptr;
  float* rho = nullptr;
  int32_t* nh = nullptr;
  // A run over one piece of a larger batch (events [event_base, ...), points
  // [point_base, ...)): its cluster ids and seed slots start at *piece_base,
  // which the run then advances by its seed count; seed indices and
  // nearest-higher indices count from point_base, seed events from
  // event_base. Null for a run that is the whole batch.
  int32_t* piece_base = nullptr;
  int64_t point_base = 0;
  int32_t event_base = 0;
  // Sweep statistics: when set, the run zeroes these 8 counters and the sweeps
  // add to them (see SweepArgs::stats).
  unsigned long long* stats = nullptr;
};

// Host tables built for a run.
struct HostTables {
  std::vector<GridDesc> grids;
  std::vector<EventDesc> events;
  std::vector<Chunk> chunks;
};

// Builds the grid/event/chunk tables from host-side event sizes. Returns false
// and sets *err when the configuration is out of range.
bool build_tables(int32_t D, const uint32_t* sizes, int32_t n_events, int32_t grid_mode,
                  int32_t points_per_tile, HostTables* t, RunShape* shape, const char** err);

// Bytes of device scratch a run of this shape needs.
size_t scratch_bytes(const RunShape& s, bool sigma, bool unc, bool tags);

// Enqueues the whole run on `stream`. Tables must already be on the device.
// When `marks` is not null it holds kStages + 1 events recorded at the stage
// boundaries (extents | tiles | gather | density | nearest higher | labels).
constexpr int kStages = 6;
cudaError_t launch_run(const RunShape& shape, const RunParams& prm, const RunIO& io,
                       const DeviceBuffers& b, cudaStream_t stream,
                       cudaEvent_t* marks = nullptr);

// Runs the tile scan's bounded wait on `desc` (zeroed: nothing publishes it);
// the kernel sets a bit in `status` when the wait gives up.
cudaError_t launch_wait_probe(unsigned long long* desc, uint32_t* status, cudaStream_t stream);
// Sets `words` 32-bit words at p to `value` with a kernel (no copy engine).
cudaError_t launch_fill32(void* p, int64_t words, uint32_t value, cudaStream_t stream);
// Turns the batch-wide results of a run into per-event results: cluster ids
// restart at 0 in every event and nearest-higher ids become event-local, which
// is exactly what each event gets when clustered alone.
cudaError_t launch_localize(const DeviceBuffers& b, int32_t n_events, int64_t n,
                            int32_t* cluster_index, int32_t* nh, cudaStream_t stream);

// Device -> host helpers used after a run.
cudaError_t launch_clusters_csr(const DeviceBuffers& b, int64_t n, const int32_t* labels,
                                int32_t n_clusters, int32_t* offsets, int32_t* points,
                                cudaStream_t stream);

int scan_blocks_for(int64_t n);

// Streaming multiprocessors of the current device, queried once per device;
// grids of the grid-stride kernels are capped at a multiple of it.
int sm_count();

// Kernel launches enqueued by the calling thread since its last reset: every
// launch site counts itself, and a run resets the count before it starts.
void reset_launch_count();
int64_t launch_count();
void count_launches(int k);

}  // namespace clue_impl
