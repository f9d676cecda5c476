// sweep.cuh — the local-density and nearest-higher sweeps.
#pragma once

#include "common.cuh"

namespace clue_impl {

// Inputs and outputs of the two sweeps. Arrays prefixed with `s` are in
// tile-contiguous (sorted) order; plane d of sx/ssig starts at d * n.
struct SweepArgs {
  int64_t n;
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
  // outputs in original order
  float* out_rho;      // may be null
  int32_t* out_nh;     // required
  int32_t* out_seed;   // may be null
  int32_t* seed_flag;  // required
};

cudaError_t launch_density(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);
cudaError_t launch_nearest_higher(int D, const RunParams& p, const SweepArgs& a, cudaStream_t st);

}  // namespace clue_impl
