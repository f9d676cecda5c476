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
};

// True when the packed fast path applies: D = 2 or 3, Euclidean metric, no
// per-point sigma and no wrapped coordinate.
bool sweep_fast_path(const RunParams& p);

cudaError_t launch_work_order(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);
cudaError_t launch_density(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);
cudaError_t launch_nearest_higher(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);

}  // namespace clue_impl
