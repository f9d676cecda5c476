/*
 * clue_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * A serial CPU restatement of CLUEstering's `Clusterer::make_clusters` (single
 * event and batched) that the test suite, `__graft_entry__.smoke()` and the CPU
 * baseline of `bench.py` use as the checker. The product path never links,
 * loads or calls it.
 *
 * Parity status: pinned. tests/test_reference_build.py checks it bit for bit
 * against the reference's own make_clusters, compiled from its unmodified
 * headers on its serial CPU backend (oracle/_ref, built by `make ref` against
 * the alpaka stand-in in alpaka_shim/), and tests/test_oracle.py against the
 * reference's own known-answer tests and its committed truth files
 * (tests/golden/).
 *
 * Floating-point semantics are the reference's source-level IEEE-754 single
 * precision semantics: every operation rounds once, in the order the reference
 * writes it (no contraction into FMA, no reassociation). Build with
 * -ffp-contract=off and without -ffast-math/-funsafe-math-optimizations.
 */
#ifndef CLUE_ORACLE_H
#define CLUE_ORACLE_H

#include <stdint.h>

#define ORACLE_MAX_DIM 10

enum { ORACLE_KERNEL_FLAT = 0, ORACLE_KERNEL_EXPONENTIAL = 1, ORACLE_KERNEL_GAUSSIAN = 2 };
enum {
  ORACLE_METRIC_EUCLIDEAN = 0,
  ORACLE_METRIC_WEIGHTED_EUCLIDEAN = 1,
  ORACLE_METRIC_PERIODIC_EUCLIDEAN = 2,
  ORACLE_METRIC_MANHATTAN = 3,
  ORACLE_METRIC_CHEBYSHEV = 4,
  ORACLE_METRIC_WEIGHTED_CHEBYSHEV = 5,
  ORACLE_METRIC_MAHALANOBIS = 6
};
/* Which exponential the Gaussian/exponential kernels call: the C library's
 * expf (what the reference's serial backend calls through std::exp) or the
 * library-owned clue_expf that the GPU path also uses. */
enum { ORACLE_EXP_LIBM = 0, ORACLE_EXP_CLUE = 1 };

typedef struct {
  float dc, rhoc, dm, seed_dc;
  uint8_t wrapped[ORACLE_MAX_DIM];
  int32_t kernel_kind;
  float kernel_params[2];
  int32_t metric_kind;
  float metric_params[ORACLE_MAX_DIM];
  int32_t exp_mode;
  int32_t points_per_tile; /* the reference hard-codes 128 */
  int32_t n_threads;       /* 0 or 1: serial; >1: OpenMP over points in the two sweeps */
} oracle_params;

typedef struct {
  int32_t ndim;
  int32_t n;
  const float* coords[ORACLE_MAX_DIM];
  const float* weight;
  const float* sigma[ORACLE_MAX_DIM]; /* NULL where unset */
  const float* density_uncertainty;   /* NULL if unset */
  const uint32_t* tags;               /* NULL if unset */
} oracle_points;

typedef struct {
  float* rho;
  int32_t* nearest_higher;
  int32_t* is_seed;
  int32_t* cluster_index;
  int32_t* seeds; /* capacity n; filled in push order */
  int32_t n_seeds;
  /* Tile grid actually used (single event, or the shared batch grid). */
  int32_t n_per_dim;
  int32_t n_tiles;
  float min_coord[ORACLE_MAX_DIM];
  float max_coord[ORACLE_MAX_DIM];
  float tile_size[ORACLE_MAX_DIM];
} oracle_out;

#ifdef __cplusplus
extern "C" {
#endif

/* Single event. Returns 0 on success, nonzero on invalid arguments. */
int clue_oracle_make_clusters(const oracle_params* params, const oracle_points* points,
                              oracle_out* out);

/* Batched form with the reference's batch-wide tile grid (shared_grid = 1),
 * or with one grid per event computed from that event's points alone
 * (shared_grid = 0, identical to running each event on its own).
 * event_associations (capacity n) receives the event of each cluster. */
int clue_oracle_make_clusters_batched(const oracle_params* params, const oracle_points* points,
                                      const uint32_t* event_sizes, int32_t n_events,
                                      int32_t shared_grid, oracle_out* out,
                                      int32_t* event_associations);

/* The library-owned exponential, exposed so tests can check its error. */
float clue_oracle_expf(float x);

/* Cluster centroids (utils/detail/cluster_centroid.hpp:86-140): for every
 * cluster c < n_clusters and dimension d, the float sum of coords[d][i] (or of
 * coords[d][i] * weights[i] when weighted) over the points with label c in
 * ascending index order, divided by the cluster's size (or by the float sum of
 * its weights, accumulated in the same order). out is n_clusters x ndim. */
void clue_oracle_centroids(int32_t ndim, int32_t n, const float* const* coords, const float* weights,
                           const int32_t* labels, int32_t n_clusters, int32_t weighted, float* out);

/* Silhouette of every point (utils/detail/scores.hpp:33-73): the points of
 * every cluster in ascending index order, distance sqrt of the left fold of
 * squared differences, a = own-cluster mean without the point itself, b = the
 * smallest other-cluster mean (FLT_MAX when there is none), (b - a) / max(a, b).
 * Points with label -1 or in a cluster of one point get NaN. */
void clue_oracle_silhouette(int32_t ndim, int32_t n, const float* const* coords, const int32_t* labels,
                            int32_t n_clusters, float* scores);

#ifdef __cplusplus
}
#endif

#endif
