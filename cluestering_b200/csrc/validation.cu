// validation.cu — cluster centroids and silhouette scores on the device
// (utils/detail/cluster_centroid.hpp:86-140, utils/detail/scores.hpp:24-100).
//
// Both take the cluster -> points map of clue_get_clusters_device (points of
// each cluster in ascending index order, the order the reference's host
// association map holds them) and add in that order with round-to-nearest
// intrinsics, so every centroid and every per-point silhouette is the
// reference's float value bit for bit. Neither allocates.
#include <cfloat>

#include "abi_internal.h"

using namespace clue_impl;

namespace {

constexpr int kThreads = 256;

struct CoordTable {
  const float* p[kMaxDim];
};

// Thread t: cluster t / D, dimension t % D. Sum of coordinates (or of
// coordinate * weight) over the cluster's points in order, divided by the size
// (or by the sum of the weights in the same order).
__global__ void __launch_bounds__(kThreads) k_centroids(int D, CoordTable x, const float* w,
                                                        const int32_t* offsets, const int32_t* members,
                                                        int32_t n_clusters, int weighted, float* out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n_clusters * D)
    return;
  const int c = (int)(t / D), d = (int)(t % D);
  const int b = offsets[c], e = offsets[c + 1];
  float sum = 0.0f, total = 0.0f;
  for (int k = b; k < e; ++k) {
    const int i = members[k];
    const float v = x.p[d][i];
    if (weighted) {
      sum = __fadd_rn(sum, __fmul_rn(v, w[i]));
      total = __fadd_rn(total, w[i]);
    } else {
      sum = __fadd_rn(sum, v);
    }
  }
  out[t] = weighted ? __fdiv_rn(sum, total) : __fdiv_rn(sum, (float)(e - b));
}

// One thread per point. Every thread of a block walks all clusters' points in
// the map's order through shared-memory tiles (cluster boundaries are the same
// for all threads), summing the distances from its point to each cluster's
// points; a cluster's mean is taken when its last point has passed.
__global__ void __launch_bounds__(kThreads) k_silhouette(int D, CoordTable x, const int32_t* labels,
                                                         const int32_t* offsets, const int32_t* members,
                                                         int32_t n_clusters, int64_t n, float* scores) {
  __shared__ float s_x[kMaxDim][kThreads];
  __shared__ int32_t s_m[kThreads];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int own = valid ? labels[i] : -1;
  float xi[kMaxDim];
#pragma unroll
  for (int d = 0; d < kMaxDim; ++d)
    xi[d] = (valid && d < D) ? x.p[d][i] : 0.0f;
  const bool take = own >= 0 && own < n_clusters && offsets[own + 1] - offsets[own] >= 2;
  float a = 0.0f, b = FLT_MAX, sum = 0.0f;
  int c = 0;
  // a cluster's mean: its own, or a candidate for the smallest other one
  auto finish = [&](int cl) {
    const int count = offsets[cl + 1] - offsets[cl];
    if (cl == own) {
      a = __fdiv_rn(sum, (float)(count - 1));
    } else {
      const float mean = __fdiv_rn(sum, (float)count);
      b = mean < b ? mean : b;  // std::min(acc, val)
    }
    sum = 0.0f;
  };
  const int M = n_clusters > 0 ? offsets[n_clusters] : 0;
  int cend = n_clusters > 0 ? offsets[1] : 0;
  for (int base = 0; base < M; base += kThreads) {
    const int cnt = min(kThreads, M - base);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const int m = members[base + threadIdx.x];
      s_m[threadIdx.x] = m;
      for (int d = 0; d < D; ++d)
        s_x[d][threadIdx.x] = x.p[d][m];
    }
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      const int pos = base + j;
      while (pos >= cend) {  // the same for every thread
        finish(c);
        ++c;
        cend = offsets[c + 1];
      }
      float dist = 0.0f;
#pragma unroll
      for (int d = 0; d < kMaxDim; ++d)
        if (d < D) {
          const float diff = __fsub_rn(xi[d], s_x[d][j]);
          dist = __fadd_rn(dist, __fmul_rn(diff, diff));
        }
      if (s_m[j] != (int)i)
        sum = __fadd_rn(sum, __fsqrt_rn(dist));
    }
  }
  for (; c < n_clusters; ++c)
    finish(c);
  if (valid) {
    const float hi = a < b ? b : a;  // std::max(a, b)
    scores[i] = take ? __fdiv_rn(__fsub_rn(b, a), hi) : __int_as_float(0x7fc00000);
  }
}

clue_status check_map(const clue_points* pts, const int32_t* offsets, const int32_t* members,
                      int32_t n_clusters) {
  if (!pts || pts->ndim < 1 || pts->ndim > kMaxDim || pts->n <= 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "points with 1..10 dimensions and n > 0 are required");
  for (int d = 0; d < pts->ndim; ++d)
    if (!pts->coords[d])
      return fail(CLUE_ERR_INVALID_ARGUMENT, "a coordinate plane is null");
  if (n_clusters < 0 || (n_clusters > 0 && (!offsets || !members)))
    return fail(CLUE_ERR_INVALID_ARGUMENT, "the cluster map is required");
  return CLUE_OK;
}

}  // namespace

extern "C" {

clue_status clue_cluster_centroids_device(const clue_points* points, const int32_t* cluster_offsets,
                                          const int32_t* cluster_points, int32_t n_clusters,
                                          int32_t weighted, float* centroids, void* stream) {
  clue_status s = check_map(points, cluster_offsets, cluster_points, n_clusters);
  if (s != CLUE_OK)
    return s;
  if (weighted && !points->weight)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "weighted centroids need the weights");
  if (n_clusters == 0)
    return CLUE_OK;
  if (!centroids)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "the centroid output is required");
  CoordTable x{};
  for (int d = 0; d < points->ndim; ++d)
    x.p[d] = points->coords[d];
  const int64_t threads = (int64_t)n_clusters * points->ndim;
  k_centroids<<<(int)((threads + kThreads - 1) / kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      points->ndim, x, points->weight, cluster_offsets, cluster_points, n_clusters, weighted ? 1 : 0,
      centroids);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "centroid kernel launch");
}

clue_status clue_silhouette_device(const clue_points* points, const int32_t* cluster_offsets,
                                   const int32_t* cluster_points, int32_t n_clusters, float* scores,
                                   void* stream) {
  clue_status s = check_map(points, cluster_offsets, cluster_points, n_clusters);
  if (s != CLUE_OK)
    return s;
  if (!points->cluster_index || !scores)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "labels (cluster_index) and the score output are required");
  CoordTable x{};
  for (int d = 0; d < points->ndim; ++d)
    x.p[d] = points->coords[d];
  k_silhouette<<<(points->n + kThreads - 1) / kThreads, kThreads, 0, (cudaStream_t)stream>>>(
      points->ndim, x, points->cluster_index, cluster_offsets, cluster_points, n_clusters, points->n,
      scores);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CLUE_OK : fail_cuda(e, "silhouette kernel launch");
}

}  // extern "C"
