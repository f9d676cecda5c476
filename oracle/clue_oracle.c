/*
 * clue_oracle.c — TEST INFRASTRUCTURE ONLY (see clue_oracle.h).
 *
 * Serial CPU restatement of CLUEstering v2.11.0's clustering path. Each
 * function cites the reference lines it restates; paths are relative to the
 * CLUEstering repository root.
 */
#include "clue_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/clue_expf.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Scalar helpers                                                            */
/* ------------------------------------------------------------------------ */

/* static_cast<int>(float) as the reference's x86 serial backend executes it
 * (cvttss2si): truncation toward zero, and INT_MIN for NaN or any value outside
 * the int range (undefined behaviour in C++, fixed here so both the checker and
 * the GPU path agree). */
static int f2i_x86(float v) {
  if (v >= -2147483648.0f && v < 2147483648.0f)
    return (int)v;
  return INT_MIN;
}

/* std::max / std::min on floats: max(a,b) = (a < b) ? b : a; min(a,b) = (b < a) ? b : a. */
static float std_max(float a, float b) { return (a < b) ? b : a; }
static float std_min(float a, float b) { return (b < a) ? b : a; }

float clue_oracle_expf(float x) { return clue_expf(x); }

static float call_exp(int mode, float x) { return mode == ORACLE_EXP_CLUE ? clue_expf(x) : expf(x); }

/* ------------------------------------------------------------------------ */
/* Tile grid                                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
  int D;
  int k;       /* tiles per dimension (n_per_dim) */
  int T;       /* tiles per event = k^D */
  float minv[ORACLE_MAX_DIM], maxv[ORACLE_MAX_DIM], tile[ORACLE_MAX_DIM];
  uint8_t wrapped[ORACLE_MAX_DIM];
  int stride[ORACLE_MAX_DIM]; /* k^(D-1-d) */
} grid_t;

/* core/detail/SetupTiles.hpp:30-34: ntiles = ceil(n / points_per_tile); the
 * smallest k with k^D >= ntiles; ntiles = k^D. */
static void grid_shape(grid_t* g, int D, int64_t n, int points_per_tile) {
  int64_t nt = (n + points_per_tile - 1) / points_per_tile;
  int k = 1;
  for (;;) {
    int64_t p = 1;
    for (int d = 0; d < D; ++d)
      p *= k;
    if (p >= nt)
      break;
    ++k;
  }
  int64_t T = 1;
  for (int d = 0; d < D; ++d)
    T *= k;
  g->D = D;
  g->k = k;
  g->T = (int)T;
  int s = 1;
  for (int d = D - 1; d >= 0; --d) {
    g->stride[d] = s;
    s *= k;
  }
}

/* core/detail/ComputeTiles.hpp:16-38: per-dimension max and min by std::reduce
 * with std::max/std::min from lowest()/max(), then tile size = (max - min) / k. */
static void grid_extent(grid_t* g, const oracle_points* p, int begin, int end) {
  for (int d = 0; d < g->D; ++d) {
    float mx = -FLT_MAX, mn = FLT_MAX;
    for (int i = begin; i < end; ++i) {
      mx = std_max(mx, p->coords[d][i]);
      mn = std_min(mn, p->coords[d][i]);
    }
    g->minv[d] = mn;
    g->maxv[d] = mx;
    g->tile[d] = (mx - mn) / (float)g->k;
  }
}

/* data_structures/internal/TilesView.hpp:96-104 */
static float normalize_coordinate(const grid_t* g, float coord, int dim) {
  const float range = g->maxv[dim] - g->minv[dim];
  float remainder = coord - (float)f2i_x86(coord / range) * range;
  if (remainder >= g->maxv[dim])
    remainder -= range;
  else if (remainder < g->minv[dim])
    remainder += range;
  return remainder;
}

/* data_structures/internal/TilesView.hpp:38-52 */
static int get_bin(const grid_t* g, float coord, int dim) {
  int b;
  if (g->wrapped[dim])
    b = f2i_x86((normalize_coordinate(g, coord, dim) - g->minv[dim]) / g->tile[dim]);
  else
    b = f2i_x86((coord - g->minv[dim]) / g->tile[dim]);
  if (b > g->k - 1)
    b = g->k - 1;
  if (b < 0)
    b = 0;
  return b;
}

/* data_structures/internal/TilesView.hpp:54-64. The reference accumulates in
 * float (pow(float k, e) * bin); every partial value is an integer below 2^24
 * for any grid this restatement accepts, so integer arithmetic is identical. */
static int64_t global_bin(const grid_t* g, const oracle_points* p, int i, int64_t event) {
  int64_t b = 0;
  for (int d = 0; d < g->D; ++d)
    b += (int64_t)g->stride[d] * get_bin(g, p->coords[d][i], d);
  return b + event * g->T;
}

/* data_structures/internal/TilesView.hpp:66-75 */
static int64_t global_bin_by_bin(const grid_t* g, const int* bins, int64_t event) {
  int64_t b = 0;
  for (int d = 0; d < g->D; ++d) {
    const int bi = g->wrapped[d] ? (bins[d] % g->k) : bins[d];
    b += (int64_t)g->stride[d] * bi;
  }
  return b + event * g->T;
}

/* data_structures/internal/TilesView.hpp:77-87 */
static void search_box(const grid_t* g, const float* lo, const float* hi, int* inf, int* sup) {
  for (int d = 0; d < g->D; ++d) {
    int a = get_bin(g, lo[d], d);
    int b = get_bin(g, hi[d], d);
    if (g->wrapped[d] && a > b)
      b += g->k;
    inf[d] = a;
    sup[d] = b;
  }
}

/* Association map filled serially: data_structures/detail/AssociationMap.hpp:
 * 20-81 (bin -> histogram -> scan -> scatter) executed by the serial backend,
 * where the scatter visits points in ascending index, so each tile lists its
 * points in ascending index order. */
typedef struct {
  int64_t nkeys;
  int32_t* offsets; /* nkeys + 1 */
  int32_t* indexes; /* n */
} assoc_t;

static int assoc_fill(assoc_t* a, const int64_t* keys, int n, int64_t nkeys, int index_base) {
  a->nkeys = nkeys;
  a->offsets = (int32_t*)calloc((size_t)nkeys + 1, sizeof(int32_t));
  a->indexes = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  if (!a->offsets || !a->indexes)
    return 1;
  for (int i = 0; i < n; ++i)
    a->offsets[keys[i] + 1] += 1;
  for (int64_t t = 0; t < nkeys; ++t)
    a->offsets[t + 1] += a->offsets[t];
  int32_t* cursor = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nkeys > 0 ? nkeys : 1));
  if (!cursor)
    return 1;
  memcpy(cursor, a->offsets, sizeof(int32_t) * (size_t)nkeys);
  for (int i = 0; i < n; ++i)
    a->indexes[cursor[keys[i]]++] = index_base + i;
  free(cursor);
  return 0;
}

static void assoc_free(assoc_t* a) {
  free(a->offsets);
  free(a->indexes);
}

/* ------------------------------------------------------------------------ */
/* Distance metrics: core/DistanceMetrics.hpp                                */
/* ------------------------------------------------------------------------ */

/* meta::accumulate (internal/meta/accumulate.hpp:17) is the right fold
 * f0 + (f1 + (... + (f_{D-1} + 0))), evaluated here innermost first. */
static float metric_distance(const oracle_params* prm, const oracle_points* p, int i, int j) {
  const int D = p->ndim;
  float acc = 0.0f;
  switch (prm->metric_kind) {
    case ORACLE_METRIC_EUCLIDEAN: /* :108-113 */
      for (int d = D - 1; d >= 0; --d) {
        const float l = p->coords[d][i], r = p->coords[d][j];
        acc = (l - r) * (l - r) + acc;
      }
      return sqrtf(acc);
    case ORACLE_METRIC_WEIGHTED_EUCLIDEAN: /* :156-162 */
      for (int d = D - 1; d >= 0; --d) {
        const float l = p->coords[d][i], r = p->coords[d][j];
        acc = prm->metric_params[d] * (l - r) * (l - r) + acc;
      }
      return sqrtf(acc);
    case ORACLE_METRIC_PERIODIC_EUCLIDEAN: /* :212-220 */
      for (int d = D - 1; d >= 0; --d) {
        const float diff = fabsf(p->coords[d][i] - p->coords[d][j]);
        const float pd = std_min(diff, prm->metric_params[d] - diff);
        acc = pd * pd + acc;
      }
      return sqrtf(acc);
    case ORACLE_METRIC_MANHATTAN: /* :241-245 */
      for (int d = D - 1; d >= 0; --d)
        acc = fabsf(p->coords[d][i] - p->coords[d][j]) + acc;
      return acc;
    case ORACLE_METRIC_CHEBYSHEV: /* :266-270, meta::maximum from 0 in dimension order */
      for (int d = 0; d < D; ++d)
        acc = std_max(acc, fabsf(p->coords[d][i] - p->coords[d][j]));
      return acc;
    case ORACLE_METRIC_WEIGHTED_CHEBYSHEV: /* :313-317 */
      for (int d = 0; d < D; ++d)
        acc = std_max(acc, prm->metric_params[d] * fabsf(p->coords[d][i] - p->coords[d][j]));
      return acc;
    case ORACLE_METRIC_MAHALANOBIS: /* :76-86 */
      for (int d = D - 1; d >= 0; --d) {
        const float diff = p->coords[d][i] - p->coords[d][j];
        const float si = p->sigma[d][i], sj = p->sigma[d][j];
        acc = diff * diff / (si * si + sj * sj) + acc;
      }
      return sqrtf(acc);
    default:
      return NAN;
  }
}

/* core/detail/ConvolutionalKernel.hpp:13-57 */
static float kernel_value(const oracle_params* prm, float dist, int i, int j) {
  if (i == j)
    return 1.0f;
  switch (prm->kernel_kind) {
    case ORACLE_KERNEL_FLAT:
      return prm->kernel_params[0];
    case ORACLE_KERNEL_GAUSSIAN: {
      const float sd = prm->kernel_params[0], amp = prm->kernel_params[1];
      return amp * call_exp(prm->exp_mode, -dist * dist / (2 * sd * sd));
    }
    case ORACLE_KERNEL_EXPONENTIAL: {
      const float avg = prm->kernel_params[0], amp = prm->kernel_params[1];
      return amp * call_exp(prm->exp_mode, -avg * dist);
    }
    default:
      return NAN;
  }
}

/* ------------------------------------------------------------------------ */
/* The two sweeps                                                            */
/* ------------------------------------------------------------------------ */

/* Search-box half width per dimension: core/detail/ClusteringKernels.hpp:112-118
 * (density) and :257-263 (nearest higher): max(r, r * sigma_i * sqrt(2)). */
static void box_extremes(const oracle_points* p, int i, float radius, float* lo, float* hi) {
  const float sqrt2 = sqrtf(2.0f);
  for (int d = 0; d < p->ndim; ++d) {
    const float s = p->sigma[d] ? p->sigma[d][i] : 0.0f;
    const float r = std_max(radius, radius * s * sqrt2);
    lo[d] = p->coords[d][i] - r;
    hi[d] = p->coords[d][i] + r;
  }
}

/* Visits the tiles of the search box in the order of for_recursion
 * (ClusteringKernels.hpp:72-88): dimension 0 outermost, last dimension fastest. */
#define FOR_EACH_TILE(g, inf, sup, event, TILE_VAR, BODY)              \
  do {                                                                 \
    int base_[ORACLE_MAX_DIM];                                         \
    for (int d_ = 0; d_ < (g)->D; ++d_)                                \
      base_[d_] = (inf)[d_];                                           \
    for (;;) {                                                         \
      const int64_t TILE_VAR = global_bin_by_bin((g), base_, (event)); \
      BODY;                                                            \
      int d_ = (g)->D - 1;                                             \
      while (d_ >= 0) {                                                \
        if (base_[d_] < (sup)[d_]) {                                   \
          ++base_[d_];                                                 \
          break;                                                       \
        }                                                              \
        base_[d_] = (inf)[d_];                                         \
        --d_;                                                          \
      }                                                                \
      if (d_ < 0)                                                      \
        break;                                                         \
    }                                                                  \
  } while (0)

/* core/detail/ClusteringKernels.hpp:92-140 with for_recursion :29-90 (and the
 * batched form BatchedClusteringKernels.hpp:28-86). */
static float local_density(const oracle_params* prm, const oracle_points* p, const grid_t* g,
                           const assoc_t* tiles, int i, int64_t event) {
  float lo[ORACLE_MAX_DIM], hi[ORACLE_MAX_DIM];
  int inf[ORACLE_MAX_DIM], sup[ORACLE_MAX_DIM];
  box_extremes(p, i, prm->dc, lo, hi);
  search_box(g, lo, hi, inf, sup);
  float rho = 0.0f;
  FOR_EACH_TILE(g, inf, sup, event, t, {
    for (int32_t s = tiles->offsets[t]; s < tiles->offsets[t + 1]; ++s) {
      const int j = tiles->indexes[s];
      const float dist = metric_distance(prm, p, i, j);
      const float k = kernel_value(prm, dist, i, j);
      rho += (float)(int)(dist <= prm->dc) * k * p->weight[j];
    }
  });
  return rho;
}

static uint64_t tag_of(const oracle_points* p, int idx) {
  return p->tags ? (uint64_t)p->tags[idx] : (uint64_t)idx;
}

/* core/detail/ClusteringKernels.hpp:231-291 with for_recursion_nearest_higher
 * :142-229 (batched form BatchedClusteringKernels.hpp:88-159). */
static int nearest_higher(const oracle_params* prm, const oracle_points* p, const grid_t* g,
                          const assoc_t* tiles, const float* rho, int i, int64_t event) {
  float delta = FLT_MAX;
  int nh = -1;
  const float rho_i = rho[i];
  const float unc = p->density_uncertainty ? p->density_uncertainty[i] : 1.0f;
  const float min_density = prm->rhoc * unc;
  float lo[ORACLE_MAX_DIM], hi[ORACLE_MAX_DIM];
  int inf[ORACLE_MAX_DIM], sup[ORACLE_MAX_DIM];
  box_extremes(p, i, prm->dm, lo, hi);
  search_box(g, lo, hi, inf, sup);
  const float eff = (rho_i >= min_density) ? prm->seed_dc : prm->dm;
  const uint64_t tag_i = tag_of(p, i);
  FOR_EACH_TILE(g, inf, sup, event, t, {
    for (int32_t s = tiles->offsets[t]; s < tiles->offsets[t + 1]; ++s) {
      const int j = tiles->indexes[s];
      const uint64_t tag_j = tag_of(p, j);
      const float rho_j = rho[j];
      int higher = rho_j > rho_i;
      higher = higher || ((rho_j == rho_i) && (rho_j > 0.0f) && (tag_j > tag_i));
      if (higher) {
        const float dist = metric_distance(prm, p, i, j);
        if (dist <= eff &&
            ((dist < delta) ||
             ((dist == delta) && (nh >= 0) &&
              ((rho_j > rho[nh]) || ((rho_j == rho[nh]) && (tag_j > tag_of(p, nh))))))) {
          delta = dist;
          nh = j;
        }
      }
    }
  });
  return nh;
}

/* ------------------------------------------------------------------------ */
/* Driver                                                                    */
/* ------------------------------------------------------------------------ */

static int check_params(const oracle_params* prm, const oracle_points* p) {
  /* core/detail/Clusterer.hpp:42-48 */
  if (!(prm->dc > 0.0f) || !(prm->rhoc >= 0.0f) || !(prm->dm > 0.0f) || !(prm->seed_dc > 0.0f))
    return 1;
  if (p->ndim < 1 || p->ndim > ORACLE_MAX_DIM || p->n <= 0)
    return 1;
  if (prm->metric_kind == ORACLE_METRIC_MAHALANOBIS)
    for (int d = 0; d < p->ndim; ++d)
      if (!p->sigma[d])
        return 1;
  return 0;
}

/* Seeds, labels and followers: ClusteringKernels.hpp:293-343 and
 * assignPointsToClusters :419-446. The serial backend pushes seeds in
 * ascending point order, so seed k (k-th smallest index) gets cluster id k. */
static void assign_clusters(const oracle_params* prm, const oracle_points* p, oracle_out* out) {
  const int n = p->n;
  out->n_seeds = 0;
  for (int i = 0; i < n; ++i) {
    out->cluster_index[i] = -1;
    const float unc = p->density_uncertainty ? p->density_uncertainty[i] : 1.0f;
    const int seed = (out->nearest_higher[i] == -1) && (out->rho[i] >= prm->rhoc * unc);
    out->is_seed[i] = seed ? 1 : 0;
    if (seed)
      out->seeds[out->n_seeds++] = i;
  }
  if (out->n_seeds == 0)
    return; /* every point stays at -1 */
  for (int k = 0; k < out->n_seeds; ++k)
    out->cluster_index[out->seeds[k]] = k;
  for (int i = 0; i < n; ++i) {
    if (out->is_seed[i] || out->nearest_higher[i] == -1)
      continue;
    int cur = i;
    while (!out->is_seed[cur] && out->nearest_higher[cur] != -1)
      cur = out->nearest_higher[cur];
    out->cluster_index[i] = out->cluster_index[cur];
  }
}

/* Runs both sweeps over the points [begin, end) of one event, with the given
 * grid and tiles (event id selects the event's block of tiles). */
static void sweeps(const oracle_params* prm, const oracle_points* p, const grid_t* g,
                   const assoc_t* tiles, int begin, int end, int64_t event, oracle_out* out) {
  int nthreads = prm->n_threads > 1 ? prm->n_threads : 1;
  (void)nthreads;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
  for (int i = begin; i < end; ++i)
    out->rho[i] = local_density(prm, p, g, tiles, i, event);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
  for (int i = begin; i < end; ++i)
    out->nearest_higher[i] = nearest_higher(prm, p, g, tiles, out->rho, i, event);
}

static void record_grid(const grid_t* g, oracle_out* out) {
  out->n_per_dim = g->k;
  out->n_tiles = g->T;
  for (int d = 0; d < g->D; ++d) {
    out->min_coord[d] = g->minv[d];
    out->max_coord[d] = g->maxv[d];
    out->tile_size[d] = g->tile[d];
  }
}

static int one_event(const oracle_params* prm, const oracle_points* p, int begin, int end,
                     int record, oracle_out* out) {
  const int ppt = prm->points_per_tile > 0 ? prm->points_per_tile : 128;
  grid_t g;
  grid_shape(&g, p->ndim, end - begin, ppt);
  for (int d = 0; d < p->ndim; ++d)
    g.wrapped[d] = prm->wrapped[d];
  grid_extent(&g, p, begin, end);
  if (record)
    record_grid(&g, out);
  /* Tile keys of the points [begin, end); the map stores global indices. */
  int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * (size_t)(end - begin));
  if (!keys)
    return 1;
  for (int i = begin; i < end; ++i)
    keys[i - begin] = global_bin(&g, p, i, 0);
  assoc_t tiles;
  if (assoc_fill(&tiles, keys, end - begin, g.T, begin)) {
    free(keys);
    assoc_free(&tiles);
    return 1;
  }
  free(keys);
  sweeps(prm, p, &g, &tiles, begin, end, 0, out);
  assoc_free(&tiles);
  return 0;
}

int clue_oracle_make_clusters(const oracle_params* prm, const oracle_points* p, oracle_out* out) {
  if (check_params(prm, p))
    return 1;
  if (one_event(prm, p, 0, p->n, 1, out))
    return 2;
  assign_clusters(prm, p, out);
  return 0;
}

/* core/detail/Clusterer.hpp:286-349. With shared_grid the grid comes from all
 * points of the batch (Clusterer.hpp:62-68, SetupTiles.hpp:19-57 with
 * batch_size) and is replicated per event (Tiles.hpp:146-147); points only see
 * their own event's tiles. Seeds are pushed in (event, index) order, which is
 * ascending global index, so labels follow the single-event rule; the event of
 * each cluster is recorded (BatchedClusteringKernels.hpp:183-187). */
int clue_oracle_make_clusters_batched(const oracle_params* prm, const oracle_points* p,
                                      const uint32_t* sizes, int32_t n_events,
                                      int32_t shared_grid, oracle_out* out,
                                      int32_t* event_assoc) {
  if (check_params(prm, p) || n_events <= 0)
    return 1;
  int64_t total = 0;
  for (int e = 0; e < n_events; ++e)
    total += sizes[e];
  if (total != p->n)
    return 1;
  if (shared_grid) {
    const int ppt = prm->points_per_tile > 0 ? prm->points_per_tile : 128;
    grid_t g;
    grid_shape(&g, p->ndim, p->n, ppt);
    for (int d = 0; d < p->ndim; ++d)
      g.wrapped[d] = prm->wrapped[d];
    grid_extent(&g, p, 0, p->n);
    record_grid(&g, out);
    int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * (size_t)p->n);
    if (!keys)
      return 2;
    int begin = 0;
    for (int e = 0; e < n_events; ++e) {
      for (uint32_t q = 0; q < sizes[e]; ++q)
        keys[begin + (int)q] = global_bin(&g, p, begin + (int)q, e);
      begin += (int)sizes[e];
    }
    assoc_t tiles;
    if (assoc_fill(&tiles, keys, p->n, (int64_t)g.T * n_events, 0)) {
      free(keys);
      assoc_free(&tiles);
      return 2;
    }
    free(keys);
    begin = 0;
    for (int e = 0; e < n_events; ++e) {
      sweeps(prm, p, &g, &tiles, begin, begin + (int)sizes[e], e, out);
      begin += (int)sizes[e];
    }
    assoc_free(&tiles);
  } else {
    int begin = 0;
    for (int e = 0; e < n_events; ++e) {
      if (sizes[e] > 0 && one_event(prm, p, begin, begin + (int)sizes[e], e == 0, out))
        return 2;
      begin += (int)sizes[e];
    }
  }
  assign_clusters(prm, p, out);
  if (event_assoc) {
    int begin = 0, k = 0;
    for (int e = 0; e < n_events; ++e) {
      for (; k < out->n_seeds && out->seeds[k] < begin + (int)sizes[e]; ++k)
        event_assoc[k] = e;
      begin += (int)sizes[e];
    }
  }
  return 0;
}

/* ---- validation utilities (utils/detail/cluster_centroid.hpp, scores.hpp) ---- */

/* Cluster -> points in ascending index order (utils/detail/get_clusters.hpp:24-49):
 * offsets[n_clusters + 1], members[offsets[n_clusters]]. */
static void cluster_map(int32_t n, const int32_t* labels, int32_t n_clusters, int32_t* offsets,
                        int32_t* members) {
  memset(offsets, 0, sizeof(int32_t) * (size_t)(n_clusters + 1));
  for (int32_t i = 0; i < n; ++i)
    if (labels[i] >= 0 && labels[i] < n_clusters)
      ++offsets[labels[i] + 1];
  for (int32_t c = 0; c < n_clusters; ++c)
    offsets[c + 1] += offsets[c];
  int32_t* cursor = malloc(sizeof(int32_t) * (size_t)(n_clusters + 1));
  memcpy(cursor, offsets, sizeof(int32_t) * (size_t)(n_clusters + 1));
  for (int32_t i = 0; i < n; ++i)
    if (labels[i] >= 0 && labels[i] < n_clusters)
      members[cursor[labels[i]]++] = i;
  free(cursor);
}

void clue_oracle_centroids(int32_t ndim, int32_t n, const float* const* coords, const float* weights,
                           const int32_t* labels, int32_t n_clusters, int32_t weighted, float* out) {
  int32_t* offsets = malloc(sizeof(int32_t) * (size_t)(n_clusters + 1));
  int32_t* members = malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  cluster_map(n, labels, n_clusters, offsets, members);
  for (int32_t c = 0; c < n_clusters; ++c) {
    for (int32_t d = 0; d < ndim; ++d) {
      float sum = 0.0f, total = 0.0f;
      for (int32_t k = offsets[c]; k < offsets[c + 1]; ++k) {
        const int32_t i = members[k];
        sum += weighted ? coords[d][i] * weights[i] : coords[d][i];
        total += weights ? weights[i] : 0.0f;
      }
      const int32_t size = offsets[c + 1] - offsets[c];
      out[(size_t)c * ndim + d] = weighted ? sum / total : sum / (float)size;
    }
  }
  free(offsets);
  free(members);
}

/* utils/detail/scores.hpp:24-31: sqrt of the left fold of squared differences. */
static float silhouette_distance(int32_t ndim, const float* const* x, int32_t i, int32_t j) {
  float dist = 0.0f;
  for (int32_t d = 0; d < ndim; ++d) {
    const float diff = x[d][i] - x[d][j];
    dist += diff * diff;
  }
  return sqrtf(dist);
}

void clue_oracle_silhouette(int32_t ndim, int32_t n, const float* const* coords, const int32_t* labels,
                            int32_t n_clusters, float* scores) {
  int32_t* offsets = malloc(sizeof(int32_t) * (size_t)(n_clusters + 1));
  int32_t* members = malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  cluster_map(n, labels, n_clusters, offsets, members);
#pragma omp parallel for schedule(dynamic, 64)
  for (int32_t i = 0; i < n; ++i) {
    const int32_t own = labels[i];
    if (own < 0 || own >= n_clusters || offsets[own + 1] - offsets[own] < 2) {
      scores[i] = NAN;
      continue;
    }
    float a = 0.0f, b = FLT_MAX;
    for (int32_t c = 0; c < n_clusters; ++c) {
      float sum = 0.0f;
      for (int32_t k = offsets[c]; k < offsets[c + 1]; ++k)
        if (members[k] != i)
          sum += silhouette_distance(ndim, coords, i, members[k]);
      const int32_t count = offsets[c + 1] - offsets[c];
      if (c == own) {
        a = sum / (float)(count - 1);
      } else {
        const float mean = sum / (float)count;
        b = mean < b ? mean : b;  /* std::min(acc, val) */
      }
    }
    const float hi = a < b ? b : a;  /* std::max(a, b) */
    scores[i] = (b - a) / hi;
  }
  free(offsets);
  free(members);
}
