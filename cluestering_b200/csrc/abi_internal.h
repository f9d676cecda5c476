// abi_internal.h — state behind the opaque handles of the C ABI, shared by
// abi.cu and server.cu.
#pragma once

#include <string>
#include <vector>

#include "clue_sm100.h"
#include "engine.h"

// Values a run sends back to pinned host memory when it finishes.
struct RunInfo {
  int32_t n_seeds;
  uint32_t status;
};

struct clue_workspace {
  int32_t device = 0;
  char* base = nullptr;  // one device allocation holding every buffer
  size_t bytes = 0;
  clue_impl::DeviceBuffers b;
  clue_impl::Capacity cap;
  void* staging = nullptr;  // pinned host buffer for the run tables
  size_t staging_bytes = 0;
  cudaEvent_t staging_event = nullptr;
  cudaEvent_t run_event = nullptr;
  RunInfo* info = nullptr;  // pinned
  bool profiling = false;
  cudaEvent_t marks[clue_impl::kStages + 1] = {};
  bool has_run = false;
  int64_t last_n = 0;
  std::vector<clue_impl::EventDesc> last_events;
  const int32_t* last_labels = nullptr;  // device cluster ids of the last run
  int64_t last_launches = 0;             // kernels the last run enqueued
  clue_tuning tuning{};                  // launch choices (set at creation to the defaults)
  // CUDA-graph replay (clue_workspace_set_graphs): the last run captured as a
  // graph, and what it was captured for. A run with the same key replays it.
  bool graphs = false;
  cudaGraphExec_t graph_exec = nullptr;
  struct GraphKey {
    clue_params params;
    clue_points points;
    clue_tuning tuning;
    int32_t grid_mode = 0;
    int64_t staged = 0;
    char* base = nullptr;
    std::vector<uint32_t> sizes;
  } graph_key{};
  bool graph_replays_last = false;  // whether the last run was a replay
  // Pipelined host batches: uploads run on `up`, downloads on `down`, both
  // ordered against the caller's stream by these events (created on first use).
  cudaStream_t up = nullptr, down = nullptr;
  std::vector<cudaEvent_t> piece_events;
  int32_t last_pieces = 0;  // pieces of the last host run (1: not pipelined)
  // Tables of the last batch shape (dimension, grid mode, points per tile,
  // event sizes), reused by a call with the same shape, and the pipelined
  // split of those tables once a host call has made it.
  struct TableCache {
    bool valid = false;
    int32_t D = 0, grid_mode = 0, ppt = 0;
    std::vector<uint32_t> sizes;
    clue_impl::HostTables tables;
    clue_impl::RunShape shape;
    bool split = false;             // the fields below belong to these tables
    std::vector<int32_t> cuts;      // event boundaries of the pieces
    clue_impl::HostTables all;      // the tables counted from each piece's start
    std::vector<clue_impl::RunShape> shapes;
    std::vector<int64_t> first;     // first point of each piece
    std::vector<size_t> chunk_at;   // first chunk of each piece
  } tables;
};

namespace clue_impl {

// Points per block of the extents and binning kernels (one chunk each).
constexpr int kChunkPoints = 4096;
// Tile grid of an event of n points in D dimensions with ppt points per tile
// (core/detail/SetupTiles.hpp:30-34): the smallest k with k^D tiles >= n / ppt.
// False when the grid does not fit int32 tile ids.
bool grid_shape(int D, int64_t n, int ppt, int32_t* k_out, int64_t* T_out);
// A grid descriptor of k per dimension and T = k^D tiles, last dimension fastest.
void fill_grid(GridDesc* g, int D, int32_t k, int64_t T);

clue_status fail(clue_status s, const std::string& msg);
clue_status fail_cuda(cudaError_t e, const char* where);
clue_status check_params(const clue_params* p);
clue_status check_points(const clue_points* pts, bool need_output, int metric_kind);
clue_status ensure_capacity(clue_workspace* ws, const RunShape& s, bool sigma, bool unc, bool tags,
                            int64_t staged);
// One piece of a pipelined batch: where its cluster ids start (a device
// counter the piece advances), its first point and event in the batch, and
// its tables, built on the host and already copied to the device.
struct Piece {
  int32_t* base = nullptr;
  int64_t point_base = 0;
  int32_t event_base = 0;
  const RunShape* shape = nullptr;
  GridDesc* grids = nullptr;
  EventDesc* events = nullptr;
  Chunk* chunks = nullptr;
};
clue_status run_device(clue_workspace* ws, const clue_params* params, const clue_points* pts,
                       const uint32_t* sizes, int32_t n_events, int32_t grid_mode,
                       cudaStream_t st, int64_t staged, const Piece* piece = nullptr);
clue_status run_host(clue_workspace* ws, const clue_params* params, const clue_points* h,
                     const uint32_t* sizes, int32_t n_events, int32_t grid_mode, cudaStream_t st);
// Stage points [first, first + count) of `h` (count < 0: all of them) in the
// workspace's input buffers, which are laid out for all h->n points.
clue_status stage_inputs(clue_workspace* ws, const clue_points* h, clue_points* dev,
                         cudaStream_t st, int64_t first = 0, int64_t count = -1);
clue_status fetch_outputs(clue_workspace* ws, const clue_points* h, cudaStream_t st,
                          int64_t first = 0, int64_t count = -1);
clue_status wait_run(clue_workspace* ws);
float sqrt_threshold(float r);
clue_tuning default_tuning();
RunParams make_run_params(const clue_params* p, const clue_points* pts, const clue_tuning& t);
// Lays the buffers of capacity `c` out from `base` (or only measures them when
// base is null) and returns the bytes they span.
size_t carve_buffers(DeviceBuffers* b, const Capacity& c, char* base);

}  // namespace clue_impl
