/*
 * clue_sm100.h — C ABI of libclue_sm100.so, a B200 (sm_100a) implementation of
 * CLUEstering's `clue::Clusterer<Ndim>::make_clusters` (single event and
 * batched) and of the result accessors around it.
 *
 * The reference has no C ABI: its boundary is the header-only C++20 template
 * API in include/CLUEstering/core/Clusterer.hpp. Each entry point below names
 * the reference member it replaces. The C++20 header clue_sm100.hpp rebuilds
 * that template API (clue::Clusterer, clue::PointsHost, clue::PointsDevice,
 * the convolutional kernels and the distance metrics) on top of these calls.
 *
 * Conventions
 *   - Plain pointers and sizes only. Streams are passed as `void*` holding a
 *     cudaStream_t (NULL = the legacy default stream).
 *   - Every call returns a clue_status. CLUE_ERR_INVALID_ARGUMENT,
 *     CLUE_ERR_OUT_OF_RANGE and CLUE_ERR_RUNTIME correspond to the reference's
 *     std::invalid_argument, std::out_of_range and std::runtime_error.
 *     clue_last_error() returns a message for the calling thread's last error.
 *   - "_device" entry points take device pointers and are asynchronous on the
 *     given stream. "_host" entry points take host pointers, copy through
 *     pinned staging and return with the results in host memory, as the
 *     reference's PointsHost overloads do.
 *   - Coordinates, weights and every FP quantity are float32. The index type
 *     is int32 (the reference's is uint32 for sizes and int32 for ids).
 *   - A workspace is not thread-safe (like the reference's Clusterer, whose
 *     tiles and seed buffers are reused between calls). Use one per thread or
 *     per stream. Different workspaces may run concurrently.
 */
#ifndef CLUE_SM100_H
#define CLUE_SM100_H

#include <stddef.h>
#include <stdint.h>

/* Exported with default visibility even when the library is built with
 * -fvisibility=hidden. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CLUE_MAX_DIM 10
#define CLUE_ABI_VERSION 1

typedef enum {
  CLUE_OK = 0,
  CLUE_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  CLUE_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range */
  CLUE_ERR_RUNTIME = 3,          /* std::runtime_error */
  CLUE_ERR_CUDA = 4,             /* a CUDA runtime call failed */
  CLUE_ERR_OUT_OF_MEMORY = 5,    /* device allocation or admission budget */
  CLUE_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up */
  CLUE_ERR_NOT_READY = 7         /* serving: the event has not completed yet */
} clue_status;

/* Convolutional kernels: core/ConvolutionalKernel.hpp:18-109. */
typedef enum {
  CLUE_KERNEL_FLAT = 0,        /* params[0] = flat value (reference default 0.5) */
  CLUE_KERNEL_EXPONENTIAL = 1, /* params = {exp_avg, exp_amplitude} */
  CLUE_KERNEL_GAUSSIAN = 2     /* params = {gaus_std, gaus_amplitude} */
} clue_kernel_kind;

/* Distance metrics: core/DistanceMetrics.hpp:63-318. */
typedef enum {
  CLUE_METRIC_EUCLIDEAN = 0,
  CLUE_METRIC_WEIGHTED_EUCLIDEAN = 1, /* metric_params = per-dimension weights */
  CLUE_METRIC_PERIODIC_EUCLIDEAN = 2, /* metric_params = per-dimension periods (0 = not periodic) */
  CLUE_METRIC_MANHATTAN = 3,
  CLUE_METRIC_CHEBYSHEV = 4,
  CLUE_METRIC_WEIGHTED_CHEBYSHEV = 5, /* metric_params = per-dimension weights */
  CLUE_METRIC_MAHALANOBIS = 6         /* needs sigma for every dimension */
} clue_metric_kind;

/* Tile grid of the batched call. */
typedef enum {
  /* One grid from all points of the batch, replicated per event: the
   * reference's batched semantics (core/Clusterer.hpp:62-68). */
  CLUE_GRID_SHARED = 0,
  /* One grid per event from that event's points: every event gets exactly the
   * result the single-event call would give it, independent of the batch. */
  CLUE_GRID_PER_EVENT = 1
} clue_grid_mode;

/* Clustering parameters: the Clusterer constructor arguments
 * (core/Clusterer.hpp:102-105; dm and seed_dc default to dc there — pass dc),
 * setWrappedCoordinates (:259-267) and the kernel/metric objects. */
typedef struct {
  float dc;      /* density_radius */
  float rhoc;    /* min_density */
  float dm;      /* outlier_distance */
  float seed_dc; /* seeding_distance */
  uint8_t wrapped[CLUE_MAX_DIM];
  int32_t kernel_kind;
  float kernel_params[2];
  int32_t metric_kind;
  float metric_params[CLUE_MAX_DIM];
  int32_t points_per_tile; /* 0 = the reference's 128 (core/Clusterer.hpp:57) */
} clue_params;

/* One SoA point set (data_structures/internal/PointsCommon.hpp:96-110).
 * Inputs: coords[d] for d < ndim, weight; optional sigma[d], density_uncertainty
 * and tags (NULL when unset: PointsHost::set_sigma/set_density_uncertainty/
 * set_tags). Outputs: cluster_index is required; is_seed, rho and
 * nearest_higher are optional (NULL = not returned). */
typedef struct {
  int32_t ndim;
  int32_t n;
  const float* coords[CLUE_MAX_DIM];
  const float* weight;
  const float* sigma[CLUE_MAX_DIM];
  const float* density_uncertainty;
  const uint32_t* tags;
  int32_t* cluster_index;
  int32_t* is_seed;
  float* rho;
  int32_t* nearest_higher;
} clue_points;

typedef struct clue_workspace clue_workspace;

/* ---- library -------------------------------------------------------------- */
int32_t clue_abi_version(void);
const char* clue_status_string(clue_status status);
/* Message of the calling thread's last failed call ("" if none). */
const char* clue_last_error(void);

/* Parameter validation of the Clusterer constructor and setParameters
 * (core/detail/Clusterer.hpp:42-48, :81-87) and of the kernel constructors
 * (core/detail/ConvolutionalKernel.hpp:13-50). */
clue_status clue_validate_params(const clue_params* params);

/* ---- workspace ------------------------------------------------------------ */
/* The reusable device state a Clusterer owns (core/Clusterer.hpp:49-51: tiles,
 * seeds, event associations). Buffers grow on demand and are never shrunk. */
clue_status clue_workspace_create(clue_workspace** ws, int32_t device);
clue_status clue_workspace_destroy(clue_workspace* ws);
/* Bytes of device memory the workspace holds. */
clue_status clue_workspace_bytes(const clue_workspace* ws, size_t* bytes);
/* Device bytes a run over n points / n_tiles tiles would need (admission). */
size_t clue_workspace_bytes_for(int32_t ndim, int64_t n_points, int64_t n_tiles, int32_t n_events);

/* Stage timing (off by default): when enabled, every run records CUDA events at
 * its stage boundaries on the run's stream. clue_workspace_stage_ms waits for
 * the last run and returns the device time of each stage in this order:
 * extents, tiles (bin + scan + scatter + order), gather, density,
 * nearest_higher, labels. Profiling tools are not needed for these numbers. */
#define CLUE_N_STAGES 6
clue_status clue_workspace_set_profiling(clue_workspace* ws, int32_t enable);
clue_status clue_workspace_stage_ms(clue_workspace* ws, float* stage_ms, int32_t capacity);
/* Sweep statistics of the last profiled run (device counters the sweeps add to
 * while profiling is on; no reference counterpart): [0] density candidate
 * tests (one point tested against one candidate record), [1] density work
 * items of 32 points, [2] nearest-higher candidate members tested, [3] cells
 * checked by the nearest-higher search, [4] cells whose members it tested.
 * The nearest-higher counters cover the cell search (2-D and 3-D Euclidean runs
 * without user tags); other paths leave them at 0. Waits for the run. */
#define CLUE_N_SWEEP_STATS 5
clue_status clue_workspace_sweep_stats(clue_workspace* ws, int64_t* stats, int32_t capacity);
/* CUDA-graph replay (off by default; no reference counterpart). When on, a
 * device run on a non-default stream (without stage timing) is captured into a
 * CUDA graph, and a later run with identical arguments — the same pointers,
 * event sizes, parameters, grid mode and tuning — replays it: no host-side
 * table building and one graph launch instead of ~20 kernel launches. The
 * inputs' contents may change between replays. Any other run replaces the
 * graph. Turning it off releases the graph. */
clue_status clue_workspace_set_graphs(clue_workspace* ws, int32_t enable);
/* Failure-detection self-test (no reference counterpart). Runs, on `device`,
 * the bounded wait of the tile scan's decoupled look-back on a flag that
 * nothing sets: the wait gives up after its limit (about 2^21 polls), the
 * kernel records that in a status word and returns, and the call returns
 * CLUE_ERR_TIMEOUT — the status every run reports when one of its waits gives
 * up. The GPU stays usable afterwards. CLUE_ERR_RUNTIME means the wait did not
 * report. Blocks until done. */
clue_status clue_selftest_bounded_wait(int32_t device, void* stream);
/* 1 when the workspace's last run was a graph replay, else 0. */
clue_status clue_workspace_graph_replayed(const clue_workspace* ws, int32_t* replayed);
/* Pieces the last host-buffer run on this workspace was split into: a batch of
 * at least 2^23 points with one grid per event runs as up to 4 pieces of whole
 * events, so that host<->device copies overlap the clustering; 1 otherwise.
 * Results are the same either way. */
clue_status clue_workspace_host_pieces(const clue_workspace* ws, int32_t* pieces);
/* Number of CUDA kernels the last run on this workspace enqueued (no reference
 * counterpart; a check that the run executed on the GPU). */
clue_status clue_workspace_kernel_launches(const clue_workspace* ws, int64_t* launches);

/* ---- launch tuning (no counterpart in the reference, whose alpaka work
 * division is fixed at compile time). None of these choices changes a result:
 * they decide only how the work is spread over the GPU. ------------------- */
typedef struct {
  /* Density sweep, 2-D and 3-D Euclidean runs: a warp whose 32 points have
   * different search boxes streams the union of their boxes through shared
   * memory when the union holds at most (threshold / 16) times the
   * candidates of the warp's largest own box; otherwise each point reads its
   * own candidates from global memory. 0 never streams such warps; a large
   * value (>= 1 << 20) always does. One value for 2-D runs, one for 3-D. */
  int32_t density_union_x16_2d;
  int32_t density_union_x16_3d;
  /* Labels: whole-array pointer-jumping rounds over the follower tree before
   * each point walks to its seed (0..4); -1 picks by size (none below 2^18
   * points, 2 below 2^22, else 3). */
  int32_t label_jump_rounds;
  /* Sweeps of 2-D and 3-D Euclidean runs: average points per cell of the cell
   * layout that orders and prunes the candidates inside each tile (1..8;
   * default 2). The tile grid itself stays the reference's (128 points per
   * tile): it decides the search boxes and the order of the density sums. */
  int32_t cell_points;
  /* Block shape of the density sweep: 0 = 256 threads with 4 blocks per SM,
   * 1 = 128 threads with 8, 2 = 256 threads with 3. */
  int32_t density_shape;
  /* Block shape of the nearest-higher cell search: 0 = 256 threads with 8
   * blocks per SM in 2-D (4 in 3-D), 1 = 256 threads with 6, 2 = 128 threads
   * with 16 in 2-D (8 in 3-D). */
  int32_t nh_shape;
  /* Tile binning: 0 = counting sort by atomics, then each tile's points put
   * in ascending index; 1 = stable runs (one warp per run of consecutive
   * points, per-event count matrices), used when every event of the run has at
   * most 4,096 tiles (else 0). Both give every tile its points in ascending
   * index. */
  int32_t tile_binning;
} clue_tuning;

/* Defaults: the values the library ships with. */
clue_status clue_tuning_defaults(clue_tuning* out);
/* The workspace's current choices (defaults until set or autotuned). */
clue_status clue_workspace_get_tuning(const clue_workspace* ws, clue_tuning* out);
/* CLUE_ERR_INVALID_ARGUMENT if a field is out of range (a negative threshold,
 * jump rounds outside -1..4, cell_points outside 1..8, a shape outside 0..2,
 * tile_binning outside 0..1). */
clue_status clue_workspace_set_tuning(clue_workspace* ws, const clue_tuning* tuning);
/* Autotuner: runs make_clusters on these device points (the single-event form
 * when event_sizes is NULL, else the batched form with grid_mode) under
 * candidate tunings, one field at a time, times each candidate with CUDA events
 * on `stream` (median of `reps` runs after one warm-up run), keeps the fastest
 * in the workspace and returns it in *chosen (may be NULL). The points' outputs
 * are written by every run and hold the (unchanged) result at the end. Blocks
 * until done. */
clue_status clue_workspace_autotune(clue_workspace* ws, const clue_params* params,
                                    const clue_points* points, const uint32_t* event_sizes,
                                    int32_t n_events, int32_t grid_mode, void* stream,
                                    int32_t reps, clue_tuning* chosen);

/* ---- clustering ----------------------------------------------------------- */
/* Clusterer::make_clusters(Queue&, PointsDevice&, metric, kernel)
 * (core/detail/Clusterer.hpp:139-151). Device pointers; asynchronous. */
clue_status clue_make_clusters_device(clue_workspace* ws, const clue_params* params,
                                      const clue_points* points, void* stream);

/* Clusterer::make_clusters(Queue&, PointsHost&, [PointsDevice&,] metric, kernel)
 * (core/detail/Clusterer.hpp:90-138). Host pointers; returns synchronised. */
clue_status clue_make_clusters_host(clue_workspace* ws, const clue_params* params,
                                    const clue_points* points, void* stream);

/* Clusterer::make_clusters(Queue&, PointsDevice&, span<const uint32_t> batch_item_sizes,
 * metric, kernel) (core/detail/Clusterer.hpp:170-183). event_sizes is a host
 * array of n_events sizes summing to points->n. Device pointers; asynchronous. */
clue_status clue_make_clusters_batched_device(clue_workspace* ws, const clue_params* params,
                                              const clue_points* points,
                                              const uint32_t* event_sizes, int32_t n_events,
                                              int32_t grid_mode, void* stream);

/* Clusterer::make_clusters(Queue&, PointsHost&, PointsDevice&, span<const uint32_t>,
 * metric, kernel) (core/detail/Clusterer.hpp:153-168). Host pointers. */
clue_status clue_make_clusters_batched_host(clue_workspace* ws, const clue_params* params,
                                            const clue_points* points,
                                            const uint32_t* event_sizes, int32_t n_events,
                                            int32_t grid_mode, void* stream);

/* Single-event clustering that allocates nothing. No counterpart in the
 * reference: it exists for callers that must not allocate device memory when
 * they cluster, such as a framework that hands all device memory to its own
 * caching allocator, or a real-time trigger loop with a fixed memory
 * reservation where an allocation could fail or stall. Inputs and outputs are
 * the caller's device buffers (as in clue_make_clusters_device); all scratch
 * comes from one array of CLUE_NOALLOC_SCRATCH_BYTES that the library reserves
 * in device memory on every GPU that loads it, for the life of the process.
 *   - At most CLUE_NOALLOC_MAX_POINTS points per call; larger events are
 *     rejected with CLUE_ERR_INVALID_ARGUMENT before any GPU work.
 *   - Every call looks up the current device's copy of the array (a lookup
 *     that allocates nothing), so the address stays valid after
 *     cudaDeviceReset. The first call on a device may load the library's
 *     device code; make it before capturing any stream.
 *   - All calls share the array: calls whose GPU work overlaps (different
 *     streams, or different host threads, on one device) race and corrupt each
 *     other. Serialise them, e.g. on one stream.
 *   - Asynchronous on `stream`. `device_status` (device pointer, may be NULL)
 *     receives the run's status word: 0, or nonzero when a bounded wait
 *     inside a kernel gave up. */
#define CLUE_NOALLOC_MAX_POINTS 16384
#define CLUE_NOALLOC_SCRATCH_BYTES (4u << 20)
clue_status clue_make_clusters_device_noalloc(const clue_params* params, const clue_points* points,
                                              uint32_t* device_status, void* stream);

/* ---- results of the last run ---------------------------------------------- */
/* Number of clusters (= seeds) of the last run; waits for it to finish.
 * PointsHost::n_clusters / PointsDevice::n_clusters
 * (data_structures/detail/PointsHost.hpp:106-116, detail/PointsDevice.hpp:109-123). */
clue_status clue_n_clusters(clue_workspace* ws, int32_t* n_clusters);

/* Clusterer::getSeeds (core/detail/Clusterer.hpp:197-203): seed indices of the
 * last run in ascending order (cluster id k is seeds[k]). Copies up to
 * capacity entries to host memory; CLUE_ERR_RUNTIME before the first run. */
clue_status clue_get_seeds(clue_workspace* ws, int32_t* seeds, int32_t capacity,
                           int32_t* n_seeds);

/* Clusterer::getClusters / clue::get_clusters (utils/detail/get_clusters.hpp:24-49):
 * cluster -> points map of the last run as CSR on the device. offsets has
 * n_clusters + 1 entries, points has room for every clustered point; point
 * ids within a cluster are ascending. Asynchronous on stream. */
clue_status clue_get_clusters_device(clue_workspace* ws, int32_t* offsets, int32_t* points,
                                     void* stream);

/* ---- validation utilities -------------------------------------------------- */
/* Both take a cluster map as clue_get_clusters_device writes it (offsets with
 * n_clusters + 1 entries, point ids ascending within a cluster), the points'
 * device buffers, and allocate nothing; asynchronous on stream.
 *
 * clue::cluster_centroids / weighted_cluster_centroids
 * (utils/detail/cluster_centroid.hpp:86-140): centroids[c * ndim + d] is the
 * float sum of coordinate d (weighted: of coordinate * weight) over cluster c's
 * points in ascending index order, divided by the cluster's size (weighted: by
 * the sum of its weights in the same order) — the reference's values bit for
 * bit. points->weight is needed when weighted. */
clue_status clue_cluster_centroids_device(const clue_points* points, const int32_t* cluster_offsets,
                                          const int32_t* cluster_points, int32_t n_clusters,
                                          int32_t weighted, float* centroids, void* stream);
/* clue::silhouette(points, point) for every point (utils/detail/scores.hpp:33-73):
 * scores[i] = (b - a) / max(a, b) with a the mean distance from i to the other
 * points of its cluster and b the smallest mean distance to another cluster
 * (FLT_MAX when there is none), Euclidean distances, sums in cluster order —
 * the reference's per-point values bit for bit; NaN for points the reference's
 * mean skips (label -1 or a cluster of one point). Reads
 * points->cluster_index as the labels. Work grows as n times the clustered
 * points, like the reference's. clue::silhouette(points) is the mean of the
 * non-NaN scores. */
clue_status clue_silhouette_device(const clue_points* points, const int32_t* cluster_offsets,
                                   const int32_t* cluster_points, int32_t n_clusters, float* scores,
                                   void* stream);

/* Clusterer::getSampleAssociations (core/detail/Clusterer.hpp:219-242): event
 * -> cluster ids of the last batched run, as CSR in host memory. offsets has
 * n_events + 1 entries; cluster ids of event e are offsets[e]..offsets[e+1]-1
 * (ids are grouped by event). n_keys receives the number of keys the reference's
 * associator reports (1 + the last event that has a cluster). */
clue_status clue_sample_associations(clue_workspace* ws, int32_t* offsets, int32_t capacity,
                                     int32_t* n_keys);

/* ---- streams and memory (used by the C++ header; no CUDA headers needed) -- */
clue_status clue_stream_create(void** stream, int32_t device);
clue_status clue_stream_destroy(void* stream);
clue_status clue_stream_synchronize(void* stream);
clue_status clue_device_malloc(void** ptr, size_t bytes, int32_t device);
clue_status clue_device_free(void* ptr);
clue_status clue_host_malloc_pinned(void** ptr, size_t bytes);
clue_status clue_host_free_pinned(void* ptr);
/* kind: 0 host->device, 1 device->host, 2 device->device. Asynchronous. */
clue_status clue_memcpy_async(void* dst, const void* src, size_t bytes, int32_t kind, void* stream);

/* ---- serving -------------------------------------------------------------- */
/* A request loop with continuous batching (no counterpart in the reference,
 * whose callers run one make_clusters per event and thread, as in
 * benchmark/throughput/worker.cpp:17-39). Events are submitted from host memory
 * as they arrive. A scheduler thread admits them in arrival order by device
 * memory: an event is admitted when its input planes fit the resident pool
 * (the budget left after the stream slots), and its points are uploaded at
 * once and stay on the device until the event completes. Admitted events of
 * one profile and one set of per-point options are grouped by size into
 * batches; a batch starts when a stream slot is free and runs while earlier
 * batches are still on the GPU; each event completes on its own. Every event
 * gets the single-event result (CLUE_GRID_PER_EVENT semantics), so a result
 * does not depend on what it was batched with. */
typedef struct clue_server clue_server;

/* Events of one profile share ndim and clustering parameters. */
typedef struct {
  int32_t ndim;
  clue_params params;
} clue_server_profile;

typedef struct {
  int32_t device;
  /* Device memory the server may hold: the stream slots (each a workspace and
   * the planes of one batch) and the resident pool of admitted events (the
   * rest, at least one batch of event planes). When max_batch_points is 0 the
   * batch size is chosen so that the slots take at most half of it. */
  size_t budget_bytes;
  int32_t max_inflight;     /* batches on the GPU at once (one stream slot each) */
  int32_t max_batch_events; /* events per batch */
  int64_t max_batch_points; /* points per batch (0: derived from the budget) */
  int32_t linger_us;        /* how long a small batch may wait for company */
  /* Target device time of one batch in ms (0: no time cap). The scheduler
   * learns each profile's device time per point from finished batches (CUDA
   * events) and stops adding events to a batch when its estimate reaches this;
   * the first event always goes in. */
  float max_batch_ms;
  /* Batches whose estimated device time is at least this many ms (0: never)
   * run on a high-priority stream, so the GPU schedules their blocks before
   * those of concurrent batches and a large event does not stretch by sharing
   * the GPU. */
  float priority_ms;
} clue_server_config;

typedef struct {
  int64_t submitted, completed, batches;
  int64_t points_completed;
  int64_t inflight_bytes_peak;  /* peak device bytes of busy slots plus resident events */
  double latency_p50_ms, latency_p99_ms, latency_max_ms;
  int64_t resident_bytes_peak;  /* peak bytes of the resident pool in use */
  int64_t resident_pool_bytes;  /* size of the resident pool */
  int64_t slot_bytes;           /* device bytes of all stream slots */
  int64_t admission_waits;      /* times the oldest waiting event did not fit yet */
  int64_t max_batch_points;     /* points one batch can hold */
} clue_server_stats;

clue_status clue_server_create(clue_server** server, const clue_server_config* config,
                               const clue_server_profile* profiles, int32_t n_profiles);
/* Queues one event of the given profile, with the per-point options the
 * reference's points take (sigma per dimension, density uncertainty, tags:
 * PointsHost.hpp:217-244). The host buffers must stay valid (and unmodified)
 * until the event completes; pinned buffers are copied by DMA, pageable ones
 * through the server's pinned staging. Outputs land in points->cluster_index
 * (and the optional outputs). An event larger than a batch or the resident
 * pool can hold is rejected with CLUE_ERR_OUT_OF_MEMORY. */
clue_status clue_server_submit(clue_server* server, int32_t profile, const clue_points* points,
                               uint64_t* ticket);
/* CLUE_OK when the event completed, CLUE_ERR_NOT_READY otherwise. */
clue_status clue_server_poll(clue_server* server, uint64_t ticket);
/* Waits until every submitted event has completed. */
clue_status clue_server_drain(clue_server* server);
clue_status clue_server_stats_get(clue_server* server, clue_server_stats* stats);
/* Per-event latencies (completion - submission, ms) in ticket order. */
clue_status clue_server_latencies(clue_server* server, double* latencies_ms, int64_t capacity,
                                  int64_t* count);
clue_status clue_server_destroy(clue_server* server);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* CLUE_SM100_H */
