// sweep.cuh — the local-density and nearest-higher sweeps.
#pragma once

#include "common.cuh"

namespace clue_impl {

// Inputs and outputs of the two sweeps. Arrays prefixed with `s` are in
// tile-contiguous (sorted) order; plane d of sx/ssig starts at d * n.
struct SweepArgs {
  int64_t n;
  int64_t n_tiles;
  const EventDesc* events;
  const GridDesc* grids;
  const int32_t* tile_offset;
  const float* sx;
  const float* sw;
  const float* ssig;
  const float* sunc;
  const uint32_t* stag;
  const int32_t* perm;  // sorted position -> original index
  const int32_t* sevt;
  float* srho;
  // Processing order of each sweep: sorted positions grouped so that the
  // lanes of a warp share one search box (see launch_work_order).
  int32_t* work_dens;
  int32_t* work_nh;
  int32_t* cls_dens;  // scratch: box class per sorted position
  int32_t* cls_nh;
  // Work queues of the fast-path sweeps: [0] density, [1] nearest higher;
  // each counts the 32-point work items taken so far (k_gather resets
  // both), so warps that finish early take the next item.
  int32_t* queue;
  // Tiles of more than 256 points (listed by the tile sort) and their count:
  // k_cells gives each of them a whole block.
  const int32_t* large_tiles;
  const int32_t* large_count;
  // Exact-sum density (flat kernel): the density records again, in cell-layout
  // order, and per event four bounds on its contributions (smallest lowest-set-
  // bit exponent, largest neighbour contribution and largest weight as float
  // bits, and a flag for a negative or non-finite one) that decide whether the
  // event's sums are exact in any order. Null when the cell layout is off.
  float4* rec_cell;
  int32_t* event_exact;
  int32_t n_events;
  // Walk order of the cell layout (k_cells): walk[k] is the layout position
  // visited k-th, tile by tile, cells in strips of 4 rows so that consecutive
  // points are spatial neighbours. Orders the density work and the
  // nearest-higher threads.
  int32_t* walk;
  // Packed candidate records of the fast path (D = 2 or 3).
  float4* rec_dens;  // {x, y, [z], v}: v = flat * w for the flat kernel, else w
  float4* rec_nh;    // D = 2: {x, y, rho, tag bits}; D = 3: {x, y, z, rho}
  uint32_t* rec_tag; // D = 3: tag of each record
  // outputs in original order
  float* out_rho;      // may be null
  int32_t* out_nh;     // required
  int32_t* out_seed;   // may be null
  int32_t* seed_flag;  // required
  // Nearest higher as a sorted position (the point itself when it has none):
  // the follower tree in the tile-contiguous layout, where chains stay local.
  int32_t* parent;
  // Cell layout of the nearest-higher search (null unless sweep_cells_path):
  // every tile is split into s^D cells (s per tile in cell_s, origin and
  // inverse cell width per dimension in cell_geom); the points of a tile are
  // reordered cell by cell inside the tile's range. A tile starting at sorted
  // position b keeps its cells in slots b .. b + s^D - 1 (s^D never exceeds
  // the tile's point count).
  // The cells are built for every fast-path run (the density sweep uses them to
  // skip out-of-reach candidates); the nearest-higher search runs over them
  // when nh_cells is set (no user tags), and then its records are in cell order.
  bool nh_cells;
  int32_t* nh_pos;        // sorted position -> layout position
  int32_t* nh_q;          // layout position -> sorted position
  int32_t* cell_slot;     // sorted position -> slot of its cell
  int32_t* cell_s;        // per tile
  float4* cell_geom;      // per tile: D = 2 {lo0, lo1, inv0, inv1}; D = 3 two entries
  CellInfo* cell_info;    // per slot
  float4* cell_box;       // per slot: bounding box of the members (D = 3: two entries)
  // Sweep statistics (null unless the run counts them): [0] density candidate
  // tests (a lane testing one record), [1] density work items, [2] nearest-
  // higher members tested, [3] cells checked, [4] cells whose members were tested.
  unsigned long long* stats;
  // Status word of the run: kernels with bounded waits set bits here.
  uint32_t* status;
};

// True when the packed fast path applies: D = 2 or 3, Euclidean metric, no
// per-point sigma and no wrapped coordinate.
bool sweep_fast_path(const RunParams& p);

// True when the nearest-higher sweep runs over the cell layout: the fast path
// without user tags. Keys (density, tag) are then unique, so the nearest
// higher is the candidate of least distance, ties to the larger key, whatever
// order the candidates are visited in.
bool sweep_cells_path(const RunParams& p);

cudaError_t launch_work_order(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);
cudaError_t launch_density(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);
cudaError_t launch_nearest_higher(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);

}  // namespace clue_impl
