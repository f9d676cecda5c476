// server.cu — the serving loop: continuous batching of independent events.
//
// Threads: any number of submitters, and one scheduler thread that forms
// batches, starts them on free stream slots and retires finished ones.
// Completion is signalled from the stream by a host function, so the scheduler
// sleeps on a condition variable instead of spinning on the GPU.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "abi_internal.h"

using namespace clue_impl;

namespace {

using Clock = std::chrono::steady_clock;

double now_s() {
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

bool is_pinned(const void* p) {
  if (!p)
    return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

enum : uint8_t { kPending = 0, kRunning = 1, kDone = 2, kFailed = 3 };

struct Request {
  uint64_t ticket;
  int32_t profile;
  clue_points pts;  // host pointers
  bool pinned;
  double t_submit;
};

// Tiles a batch of P points in E events can need with one grid per event: an
// event of n points gets k^D tiles with k = ceil((n/128)^(1/D)), which for
// D <= 3 stays below n/16 + 8 (the rounding of k up costs at most a factor 8).
// Larger dimensions are reserved more loosely; a batch that still needs more
// grows the workspace.
int64_t tiles_bound(int32_t D, int64_t P, int64_t E) {
  return D <= 3 ? P / 16 + 8 * E + 1024 : P / 4 + 64 * E + 1024;
}

// Size bucket of an event: batches are formed from one bucket (and smaller
// ones), so a small event does not wait behind a batch of large ones.
int bucket_of(int32_t n) {
  int b = 0;
  while ((1 << (b + 1)) <= n)
    ++b;
  return b;
}

}  // namespace

struct Slot {
  cudaStream_t stream = nullptr;     // default priority
  cudaStream_t stream_hi = nullptr;  // highest priority: batches holding a long event
  cudaStream_t active = nullptr;     // the stream of the batch in flight
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;  // device time of the batch
  int32_t profile = 0;
  clue_workspace* ws = nullptr;
  // device inputs and outputs of one batch (planes of max_points)
  float* d_coords = nullptr;
  float* d_weight = nullptr;
  int32_t* d_cluster = nullptr;
  int32_t* d_seed = nullptr;
  float* d_rho = nullptr;
  int32_t* d_nh = nullptr;
  // pinned staging for requests whose buffers are pageable
  float* h_coords = nullptr;
  float* h_weight = nullptr;
  int32_t* h_cluster = nullptr;
  int32_t* h_seed = nullptr;
  float* h_rho = nullptr;
  int32_t* h_nh = nullptr;
  std::vector<Request> batch;
  std::vector<int64_t> offsets;
  int64_t bytes = 0;
  bool busy = false;
  std::atomic<bool> done{false};
  clue_server* server = nullptr;
};

struct clue_server {
  clue_server_config cfg;
  std::vector<clue_server_profile> profiles;
  // Device time per point of each profile (ns), learned from finished batches
  // of at least kCostSamplePoints points; 0 until the first such batch.
  std::vector<double> ns_per_point;
  int32_t max_dim = 1;
  int64_t max_points = 0;
  std::vector<Slot*> slots;
  // queues: profile -> bucket -> FIFO of requests
  std::vector<std::map<int, std::deque<Request>>> queues;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  std::thread scheduler;
  // per ticket
  std::vector<uint8_t> state;
  std::vector<double> t_submit, t_done;
  std::vector<int32_t> sizes;
  int64_t submitted = 0, completed = 0, batches = 0, points_completed = 0;
  int64_t inflight_bytes = 0, inflight_peak = 0;
  std::string error;
};

namespace {

void CUDART_CB on_batch_done(void* arg) {
  Slot* s = static_cast<Slot*>(arg);
  s->done.store(true);
  clue_server* srv = s->server;
  std::lock_guard<std::mutex> lock(srv->mu);
  srv->cv.notify_all();
}

// Oldest pending request over all profiles and buckets, or false.
bool oldest_bucket(clue_server* srv, int* profile, int* bucket, double* t) {
  bool found = false;
  for (int p = 0; p < (int)srv->queues.size(); ++p)
    for (auto& [b, q] : srv->queues[p])
      if (!q.empty() && (!found || q.front().t_submit < *t)) {
        found = true;
        *profile = p;
        *bucket = b;
        *t = q.front().t_submit;
      }
  return found;
}

int64_t pending_points(clue_server* srv, int profile) {
  int64_t n = 0;
  for (auto& [b, q] : srv->queues[profile])
    for (auto& r : q)
      n += r.pts.n;
  return n;
}

// Batches of fewer points have their time dominated by per-launch latency and
// are not used to learn the per-point cost.
constexpr int64_t kCostSamplePoints = 1 << 16;

int64_t pending_points(clue_server* srv, int profile);

// Points a batch of `profile` may hold: the memory cap, and the time cap once
// the profile's cost per point is known (at least one event always goes in).
// The time cap grows with the backlog: when the pending work of the profile
// exceeds what the slots clear in batches of max_batch_ms, queueing dominates
// the latency and larger batches (fewer per-batch overheads) clear it sooner.
int64_t batch_point_cap(clue_server* srv, int profile) {
  const double ns = srv->ns_per_point[profile];
  if (srv->cfg.max_batch_ms <= 0.0f || ns <= 0.0)
    return srv->max_points;
  const double backlog_ms = (double)pending_points(srv, profile) * ns * 1e-6;
  const double cap_ms = std::max<double>(srv->cfg.max_batch_ms, backlog_ms / srv->cfg.max_inflight);
  return std::min<int64_t>(srv->max_points, (int64_t)(cap_ms * 1e6 / ns));
}

// Takes a batch for `profile` starting from `bucket`, then smaller buckets.
std::vector<Request> take_batch(clue_server* srv, int profile, int bucket) {
  std::vector<Request> out;
  int64_t pts = 0;
  const int64_t cap = batch_point_cap(srv, profile);
  auto& qs = srv->queues[profile];
  for (auto it = qs.find(bucket);; --it) {
    auto& q = it->second;
    while (!q.empty() && (int)out.size() < srv->cfg.max_batch_events &&
           pts + q.front().pts.n <= srv->max_points && (out.empty() || pts + q.front().pts.n <= cap)) {
      pts += q.front().pts.n;
      out.push_back(q.front());
      q.pop_front();
    }
    if (it == qs.begin() || (int)out.size() >= srv->cfg.max_batch_events)
      break;
  }
  return out;
}

clue_status launch_batch(clue_server* srv, Slot* s, std::vector<Request>&& reqs) {
  const clue_server_profile& prof = srv->profiles[reqs[0].profile];
  const int D = prof.ndim;
  s->batch = std::move(reqs);
  const int B = (int)s->batch.size();
  std::vector<uint32_t> sizes(B);
  s->offsets.assign(B + 1, 0);
  for (int e = 0; e < B; ++e) {
    sizes[e] = (uint32_t)s->batch[e].pts.n;
    s->offsets[e + 1] = s->offsets[e] + sizes[e];
  }
  const int64_t P = s->offsets[B];
  bool want_seed = false, want_rho = false, want_nh = false;
  cudaError_t e;
  // A batch holding an event that is expected to run long goes first on the GPU.
  int32_t n_max = 0;
  for (uint32_t z : sizes)
    n_max = std::max<int32_t>(n_max, (int32_t)z);
  const double ns = srv->ns_per_point[s->batch[0].profile];
  const bool urgent = srv->cfg.priority_ms > 0.0f && ns > 0.0 &&
                      (double)n_max * ns * 1e-6 >= srv->cfg.priority_ms;
  s->active = urgent ? s->stream_hi : s->stream;
  s->profile = s->batch[0].profile;
  if ((e = cudaEventRecord(s->ev_start, s->active)))
    return fail_cuda(e, "batch start event");
  for (int k = 0; k < B; ++k) {
    const Request& r = s->batch[k];
    const int64_t off = s->offsets[k];
    const size_t nb = (size_t)r.pts.n * sizeof(float);
    want_seed |= r.pts.is_seed != nullptr;
    want_rho |= r.pts.rho != nullptr;
    want_nh |= r.pts.nearest_higher != nullptr;
    for (int d = 0; d <= D; ++d) {
      const float* src = d < D ? r.pts.coords[d] : r.pts.weight;
      float* dst_dev = d < D ? s->d_coords + d * P + off : s->d_weight + off;
      if (r.pinned) {
        if ((e = cudaMemcpyAsync(dst_dev, src, nb, cudaMemcpyHostToDevice, s->active)))
          return fail_cuda(e, "event upload");
      } else {
        float* dst_host = d < D ? s->h_coords + d * P + off : s->h_weight + off;
        std::memcpy(dst_host, src, nb);
      }
    }
  }
  // pageable requests: one copy per plane from the staging buffer
  bool any_pageable = false;
  for (auto& r : s->batch)
    any_pageable |= !r.pinned;
  if (any_pageable)
    for (int k = 0; k < B; ++k) {
      const Request& r = s->batch[k];
      if (r.pinned)
        continue;
      const int64_t off = s->offsets[k];
      const size_t nb = (size_t)r.pts.n * sizeof(float);
      for (int d = 0; d <= D; ++d) {
        float* dst_dev = d < D ? s->d_coords + d * P + off : s->d_weight + off;
        const float* src = d < D ? s->h_coords + d * P + off : s->h_weight + off;
        if ((e = cudaMemcpyAsync(dst_dev, src, nb, cudaMemcpyHostToDevice, s->active)))
          return fail_cuda(e, "event upload");
      }
    }
  clue_points dev{};
  dev.ndim = D;
  dev.n = (int32_t)P;
  for (int d = 0; d < D; ++d)
    dev.coords[d] = s->d_coords + d * P;
  dev.weight = s->d_weight;
  dev.cluster_index = s->d_cluster;
  dev.is_seed = want_seed ? s->d_seed : nullptr;
  dev.rho = want_rho ? s->d_rho : nullptr;
  dev.nearest_higher = want_nh ? s->d_nh : nullptr;
  clue_status st = run_device(s->ws, &prof.params, &dev, sizes.data(), B, CLUE_GRID_PER_EVENT,
                              s->active, 0);
  if (st != CLUE_OK)
    return st;
  if ((e = launch_localize(s->ws->b, B, P, s->d_cluster, want_nh ? s->d_nh : nullptr, s->active)))
    return fail_cuda(e, "relabel");
  for (int k = 0; k < B; ++k) {
    const Request& r = s->batch[k];
    const int64_t off = s->offsets[k];
    const size_t nb = (size_t)r.pts.n * 4;
    struct {
      void* user;
      void* staging;
      const void* dev;
    } outs[4] = {{r.pts.cluster_index, s->h_cluster + off, s->d_cluster + off},
                 {r.pts.is_seed, s->h_seed + off, s->d_seed + off},
                 {r.pts.rho, s->h_rho + off, s->d_rho + off},
                 {r.pts.nearest_higher, s->h_nh + off, s->d_nh + off}};
    for (auto& o : outs) {
      if (!o.user)
        continue;
      void* dst = r.pinned ? o.user : o.staging;
      if ((e = cudaMemcpyAsync(dst, o.dev, nb, cudaMemcpyDeviceToHost, s->active)))
        return fail_cuda(e, "result download");
    }
  }
  if ((e = cudaEventRecord(s->ev_end, s->active)))
    return fail_cuda(e, "batch end event");
  s->done.store(false);
  if ((e = cudaLaunchHostFunc(s->active, on_batch_done, s)))
    return fail_cuda(e, "completion callback");
  return CLUE_OK;
}

// Copies staged outputs of pageable requests back and completes the tickets.
void retire_batch(clue_server* srv, Slot* s, bool ok) {
  const double t = now_s();
  int64_t P = 0;
  for (auto& r : s->batch)
    P += r.pts.n;
  float ms = 0.0f;
  const bool timed = ok && P >= kCostSamplePoints &&
                     cudaEventElapsedTime(&ms, s->ev_start, s->ev_end) == cudaSuccess;
  for (size_t k = 0; k < s->batch.size(); ++k) {
    const Request& r = s->batch[k];
    if (ok && !r.pinned) {
      const int64_t off = s->offsets[k];
      const size_t nb = (size_t)r.pts.n * 4;
      std::memcpy(r.pts.cluster_index, s->h_cluster + off, nb);
      if (r.pts.is_seed)
        std::memcpy(r.pts.is_seed, s->h_seed + off, nb);
      if (r.pts.rho)
        std::memcpy(r.pts.rho, s->h_rho + off, nb);
      if (r.pts.nearest_higher)
        std::memcpy(r.pts.nearest_higher, s->h_nh + off, nb);
    }
  }
  std::lock_guard<std::mutex> lock(srv->mu);
  if (timed) {
    double& ns = srv->ns_per_point[s->profile];
    const double sample = (double)ms * 1e6 / (double)P;
    ns = ns > 0.0 ? 0.8 * ns + 0.2 * sample : sample;
  }
  for (auto& r : s->batch) {
    srv->state[r.ticket] = ok ? kDone : kFailed;
    srv->t_done[r.ticket] = t;
    srv->completed += 1;
    srv->points_completed += r.pts.n;
  }
  srv->inflight_bytes -= s->bytes;
  s->batch.clear();
  s->busy = false;
  srv->cv.notify_all();
}

void scheduler_loop(clue_server* srv) {
  cudaSetDevice(srv->cfg.device);
  std::unique_lock<std::mutex> lock(srv->mu);
  while (true) {
    // retire finished batches
    for (Slot* s : srv->slots)
      if (s->busy && s->done.load()) {
        lock.unlock();
        const bool ok = cudaStreamSynchronize(s->active) == cudaSuccess;
        retire_batch(srv, s, ok);
        lock.lock();
      }
    if (srv->stop) {
      bool busy = false;
      for (Slot* s : srv->slots)
        busy |= s->busy;
      bool pending = false;
      for (auto& pq : srv->queues)
        for (auto& [b, q] : pq)
          pending |= !q.empty();
      if (!busy && !pending)
        return;
    }
    // start a batch if a slot is free
    Slot* free_slot = nullptr;
    int n_busy = 0;
    for (Slot* s : srv->slots) {
      if (s->busy)
        ++n_busy;
      else if (!free_slot)
        free_slot = s;
    }
    int profile = 0, bucket = 0;
    double t_old = 0;
    if (free_slot && oldest_bucket(srv, &profile, &bucket, &t_old)) {
      const double waited_us = (now_s() - t_old) * 1e6;
      const bool small = pending_points(srv, profile) < srv->max_points / 4;
      if (n_busy > 0 && small && waited_us < srv->cfg.linger_us && !srv->stop) {
        srv->cv.wait_for(lock, std::chrono::microseconds(
                                   std::max<int64_t>(1, srv->cfg.linger_us - (int64_t)waited_us)));
        continue;
      }
      std::vector<Request> reqs = take_batch(srv, profile, bucket);
      for (auto& r : reqs)
        srv->state[r.ticket] = kRunning;
      free_slot->busy = true;
      free_slot->bytes = (int64_t)free_slot->ws->bytes;
      srv->inflight_bytes += free_slot->bytes;
      srv->inflight_peak = std::max(srv->inflight_peak, srv->inflight_bytes);
      srv->batches += 1;
      lock.unlock();
      std::vector<Request> keep = reqs;
      clue_status st = launch_batch(srv, free_slot, std::move(reqs));
      if (st != CLUE_OK) {
        free_slot->batch = std::move(keep);
        cudaStreamSynchronize(free_slot->active);
        retire_batch(srv, free_slot, false);
      }
      lock.lock();
      continue;
    }
    srv->cv.wait_for(lock, std::chrono::milliseconds(5));
  }
}

void free_slot(Slot* s) {
  if (s->stream)
    cudaStreamSynchronize(s->stream);
  if (s->stream_hi)
    cudaStreamSynchronize(s->stream_hi);
  for (cudaEvent_t ev : {s->ev_start, s->ev_end})
    if (ev)
      cudaEventDestroy(ev);
  if (s->ws)
    clue_workspace_destroy(s->ws);
  for (void* p : {(void*)s->d_coords, (void*)s->d_weight, (void*)s->d_cluster, (void*)s->d_seed,
                  (void*)s->d_rho, (void*)s->d_nh})
    if (p)
      cudaFree(p);
  for (void* p : {(void*)s->h_coords, (void*)s->h_weight, (void*)s->h_cluster, (void*)s->h_seed,
                  (void*)s->h_rho, (void*)s->h_nh})
    if (p)
      cudaFreeHost(p);
  if (s->stream)
    cudaStreamDestroy(s->stream);
  if (s->stream_hi)
    cudaStreamDestroy(s->stream_hi);
  delete s;
}

}  // namespace

extern "C" {

clue_status clue_server_create(clue_server** out, const clue_server_config* cfg,
                               const clue_server_profile* profiles, int32_t n_profiles) {
  if (!out || !cfg || !profiles || n_profiles <= 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "server config and at least one profile are required");
  if (cfg->max_inflight <= 0 || cfg->max_batch_events <= 0 || cfg->budget_bytes == 0)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "max_inflight, max_batch_events and budget must be positive");
  if (!(cfg->max_batch_ms >= 0.0f) || !(cfg->priority_ms >= 0.0f))
    return fail(CLUE_ERR_INVALID_ARGUMENT, "max_batch_ms and priority_ms must be >= 0");
  int32_t max_dim = 1;
  for (int i = 0; i < n_profiles; ++i) {
    clue_status s = check_params(&profiles[i].params);
    if (s != CLUE_OK)
      return s;
    if (profiles[i].ndim < 1 || profiles[i].ndim > CLUE_MAX_DIM)
      return fail(CLUE_ERR_OUT_OF_RANGE, "profile ndim must be in [1, 10]");
    max_dim = std::max(max_dim, profiles[i].ndim);
  }
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess)
    return fail_cuda(e, "cudaSetDevice");
  auto* srv = new clue_server();
  srv->cfg = *cfg;
  srv->profiles.assign(profiles, profiles + n_profiles);
  srv->queues.resize(n_profiles);
  srv->ns_per_point.assign(n_profiles, 0.0);
  srv->max_dim = max_dim;
  // Device bytes per batch point: workspace scratch plus inputs and outputs.
  const int64_t per_slot = (int64_t)(cfg->budget_bytes / cfg->max_inflight);
  auto slot_bytes = [&](int64_t P, int64_t E) {
    RunShape sh;
    sh.D = max_dim;
    sh.n = P;
    sh.n_events = (int32_t)E;
    sh.n_grids = (int32_t)E;
    sh.n_tiles = tiles_bound(max_dim, P, E);
    sh.n_chunks = (int32_t)(P / 4096 + E + 1);
    return (int64_t)scratch_bytes(sh, false, false, false) + P * (int64_t)(4 * (max_dim + 1) + 16);
  };
  int64_t P = cfg->max_batch_points > 0 ? cfg->max_batch_points : (int64_t)1 << 24;
  while (P > 4096 && slot_bytes(P, cfg->max_batch_events) > per_slot)
    P /= 2;
  if (slot_bytes(P, cfg->max_batch_events) > per_slot) {
    delete srv;
    return fail(CLUE_ERR_OUT_OF_MEMORY, "the memory budget is too small for one batch per slot");
  }
  srv->max_points = P;
  for (int i = 0; i < cfg->max_inflight; ++i) {
    Slot* s = new Slot();
    s->server = srv;
    srv->slots.push_back(s);
    clue_status st = CLUE_OK;
    int prio_low = 0, prio_high = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)) ||
        (e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio_low)) ||
        (e = cudaStreamCreateWithPriority(&s->stream_hi, cudaStreamNonBlocking, prio_high)) ||
        (e = cudaEventCreate(&s->ev_start)) || (e = cudaEventCreate(&s->ev_end)) ||
        (e = cudaMalloc(&s->d_coords, P * max_dim * sizeof(float))) ||
        (e = cudaMalloc(&s->d_weight, P * sizeof(float))) ||
        (e = cudaMalloc(&s->d_cluster, P * sizeof(int32_t))) ||
        (e = cudaMalloc(&s->d_seed, P * sizeof(int32_t))) ||
        (e = cudaMalloc(&s->d_rho, P * sizeof(float))) ||
        (e = cudaMalloc(&s->d_nh, P * sizeof(int32_t))) ||
        (e = cudaMallocHost(&s->h_coords, P * max_dim * sizeof(float))) ||
        (e = cudaMallocHost(&s->h_weight, P * sizeof(float))) ||
        (e = cudaMallocHost(&s->h_cluster, P * sizeof(int32_t))) ||
        (e = cudaMallocHost(&s->h_seed, P * sizeof(int32_t))) ||
        (e = cudaMallocHost(&s->h_rho, P * sizeof(float))) ||
        (e = cudaMallocHost(&s->h_nh, P * sizeof(int32_t))))
      st = fail_cuda(e, "server slot allocation");
    s->active = s->stream;
    if (st == CLUE_OK)
      st = clue_workspace_create(&s->ws, cfg->device);
    if (st == CLUE_OK) {
      // Reserve the largest batch up front: no allocation while serving.
      RunShape sh;
      sh.D = max_dim;
      sh.n = P;
      sh.n_events = cfg->max_batch_events;
      sh.n_grids = cfg->max_batch_events;
      sh.n_tiles = tiles_bound(max_dim, P, cfg->max_batch_events);
      sh.n_chunks = (int32_t)(P / 4096 + cfg->max_batch_events + 1);
      st = ensure_capacity(s->ws, sh, false, false, false, 0);
    }
    if (st != CLUE_OK) {
      for (Slot* x : srv->slots)
        free_slot(x);
      delete srv;
      return st;
    }
  }
  srv->scheduler = std::thread(scheduler_loop, srv);
  *out = srv;
  return CLUE_OK;
}

clue_status clue_server_submit(clue_server* srv, int32_t profile, const clue_points* pts,
                               uint64_t* ticket) {
  if (!srv || !pts)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  if (profile < 0 || profile >= (int32_t)srv->profiles.size())
    return fail(CLUE_ERR_OUT_OF_RANGE, "unknown profile");
  const clue_server_profile& prof = srv->profiles[profile];
  clue_status s = check_points(pts, true, prof.params.metric_kind);
  if (s != CLUE_OK)
    return s;
  if (pts->ndim != prof.ndim)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "event ndim differs from the profile's");
  for (int d = 0; d < pts->ndim; ++d)
    if (pts->sigma[d])
      return fail(CLUE_ERR_INVALID_ARGUMENT, "the server does not take per-point sigma");
  if (pts->density_uncertainty || pts->tags)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "the server does not take uncertainties or tags");
  if (pts->n > srv->max_points)
    return fail(CLUE_ERR_OUT_OF_MEMORY, "event larger than the server's batch capacity");
  Request r;
  r.profile = profile;
  r.pts = *pts;
  r.pinned = is_pinned(pts->weight) && is_pinned(pts->cluster_index);
  for (int d = 0; d < pts->ndim && r.pinned; ++d)
    r.pinned = is_pinned(pts->coords[d]);
  for (const void* o : {(const void*)pts->is_seed, (const void*)pts->rho,
                        (const void*)pts->nearest_higher})
    r.pinned = r.pinned && is_pinned(o);
  r.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    if (srv->stop)
      return fail(CLUE_ERR_RUNTIME, "server is shutting down");
    r.ticket = (uint64_t)srv->state.size();
    srv->state.push_back(kPending);
    srv->t_submit.push_back(r.t_submit);
    srv->t_done.push_back(0.0);
    srv->sizes.push_back(pts->n);
    srv->submitted += 1;
    srv->queues[profile][bucket_of(pts->n)].push_back(r);
  }
  srv->cv.notify_all();
  if (ticket)
    *ticket = r.ticket;
  return CLUE_OK;
}

clue_status clue_server_poll(clue_server* srv, uint64_t ticket) {
  if (!srv)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null server");
  std::lock_guard<std::mutex> lock(srv->mu);
  if (ticket >= srv->state.size())
    return fail(CLUE_ERR_OUT_OF_RANGE, "unknown ticket");
  const uint8_t st = srv->state[ticket];
  if (st == kDone)
    return CLUE_OK;
  if (st == kFailed)
    return fail(CLUE_ERR_RUNTIME, "the batch holding this event failed");
  return CLUE_ERR_NOT_READY;
}

clue_status clue_server_drain(clue_server* srv) {
  if (!srv)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null server");
  std::unique_lock<std::mutex> lock(srv->mu);
  srv->cv.wait(lock, [&] { return srv->completed == srv->submitted; });
  for (uint8_t st : srv->state)
    if (st == kFailed)
      return fail(CLUE_ERR_RUNTIME, "at least one batch failed");
  return CLUE_OK;
}

clue_status clue_server_stats_get(clue_server* srv, clue_server_stats* out) {
  if (!srv || !out)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<double> lat;
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    out->submitted = srv->submitted;
    out->completed = srv->completed;
    out->batches = srv->batches;
    out->points_completed = srv->points_completed;
    out->inflight_bytes_peak = srv->inflight_peak;
    for (size_t i = 0; i < srv->state.size(); ++i)
      if (srv->state[i] == kDone)
        lat.push_back((srv->t_done[i] - srv->t_submit[i]) * 1e3);
  }
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double q) {
    if (lat.empty())
      return 0.0;
    const size_t i = std::min(lat.size() - 1, (size_t)(q * (lat.size() - 1) + 0.5));
    return lat[i];
  };
  out->latency_p50_ms = pct(0.50);
  out->latency_p99_ms = pct(0.99);
  out->latency_max_ms = lat.empty() ? 0.0 : lat.back();
  return CLUE_OK;
}

clue_status clue_server_latencies(clue_server* srv, double* lat, int64_t capacity, int64_t* count) {
  if (!srv)
    return fail(CLUE_ERR_INVALID_ARGUMENT, "null server");
  std::lock_guard<std::mutex> lock(srv->mu);
  const int64_t n = (int64_t)srv->state.size();
  if (count)
    *count = n;
  for (int64_t i = 0; i < n && i < capacity && lat; ++i)
    lat[i] = srv->state[i] == kDone ? (srv->t_done[i] - srv->t_submit[i]) * 1e3 : -1.0;
  return CLUE_OK;
}

clue_status clue_server_destroy(clue_server* srv) {
  if (!srv)
    return CLUE_OK;
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->stop = true;
  }
  srv->cv.notify_all();
  if (srv->scheduler.joinable())
    srv->scheduler.join();
  cudaSetDevice(srv->cfg.device);
  for (Slot* s : srv->slots)
    free_slot(s);
  delete srv;
  return CLUE_OK;
}

}  // extern "C"
