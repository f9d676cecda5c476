// server.cu — the serving loop: admission by device-memory budget, resident
// events and continuous batching.
//
// Threads: any number of submitters, and one scheduler thread that admits
// events, forms batches, starts them on free stream slots and retires finished
// ones. Completion is signalled from the stream by a host function, so the
// scheduler sleeps on a condition variable instead of spinning on the GPU.
//
// Life of an event: submitted (host queue, arrival order) -> admitted (its
// points get a block of the device pool, inside the budget, and are uploaded
// on the upload stream at once; they stay resident until the event completes)
// -> batched with admitted events of the same profile and options, by size ->
// its batch's slot copies the resident points into the batch's planes on the
// device, clusters them and downloads the event's results -> completed (the
// block goes back to the pool).
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

// First-fit allocator over one region [0, size) (device or pinned host memory),
// blocks aligned to 256 bytes; freed blocks merge with their neighbours.
class Pool {
 public:
  void init(char* base, int64_t size) {
    base_ = base;
    size_ = size;
    free_.clear();
    if (size > 0)
      free_[0] = size;
    used_ = 0;
  }
  char* alloc(int64_t bytes) {
    bytes = (bytes + 255) & ~int64_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        const int64_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > bytes)
          free_[off + bytes] = len - bytes;
        used_ += bytes;
        return base_ + off;
      }
    }
    return nullptr;
  }
  void release(char* p, int64_t bytes) {
    if (!p)
      return;
    bytes = (bytes + 255) & ~int64_t(255);
    used_ -= bytes;
    int64_t off = p - base_;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + bytes == next->first) {
      bytes += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += bytes;
        return;
      }
    }
    free_[off] = bytes;
  }
  int64_t size() const { return size_; }
  int64_t used() const { return used_; }

 private:
  char* base_ = nullptr;
  int64_t size_ = 0;
  int64_t used_ = 0;
  std::map<int64_t, int64_t> free_;
};

// Optional per-point inputs of an event: bits 0..9 sigma of dimension d, bit
// 10 density uncertainty, bit 11 tags. Only events with equal options share a
// batch, so a batch carries exactly the planes its events have.
constexpr uint32_t kOptUnc = 1u << 10, kOptTags = 1u << 11;

uint32_t options_of(const clue_points* p) {
  uint32_t m = 0;
  for (int d = 0; d < p->ndim; ++d)
    if (p->sigma[d])
      m |= 1u << d;
  if (p->density_uncertainty)
    m |= kOptUnc;
  if (p->tags)
    m |= kOptTags;
  return m;
}

// Input planes of an event with these options, in their resident order:
// coordinates, weight, sigma of each dimension that has one, uncertainty, tags.
int planes_of(int D, uint32_t opts) {
  return D + 1 + __builtin_popcount(opts & 0x3ffu) + ((opts & kOptUnc) ? 1 : 0) +
         ((opts & kOptTags) ? 1 : 0);
}

const void* plane_src(const clue_points* p, uint32_t opts, int k) {
  const int D = p->ndim;
  if (k < D)
    return p->coords[k];
  if (k == D)
    return p->weight;
  k -= D + 1;
  for (int d = 0; d < D; ++d)
    if (opts & (1u << d)) {
      if (k == 0)
        return p->sigma[d];
      --k;
    }
  if (opts & kOptUnc) {
    if (k == 0)
      return p->density_uncertainty;
    --k;
  }
  return p->tags;
}

struct Request {
  uint64_t ticket;
  int32_t profile;
  uint32_t opts;
  clue_points pts;      // host pointers
  bool in_pinned;       // inputs can be uploaded by DMA from the caller's buffers
  bool out_pinned;      // outputs can be downloaded into the caller's buffers
  double t_submit;
  int64_t bytes = 0;    // resident device bytes (input planes)
  char* dev = nullptr;  // resident block in the device pool
  char* host = nullptr; // pinned staging of pageable inputs (host pool)
  cudaEvent_t uploaded = nullptr;
};

// One entry of the batch assembly table: the event's resident planes start at
// src (plane k at src + k * n words); its points go to offset off of every
// batch plane.
struct AsmEvent {
  const uint32_t* src;
  int32_t n;
  int32_t off;
};

// Copies every event's resident planes into the batch planes (plane k of the
// batch at dst + k * P). Word copies: tags travel as their bit patterns.
__global__ void k_assemble(const AsmEvent* evs, int planes, int64_t P, uint32_t* dst) {
  const AsmEvent e = evs[blockIdx.y];
  const int64_t total = (int64_t)e.n * planes;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i / e.n, j = i - k * e.n;
    dst[k * P + e.off + j] = e.src[i];
  }
}

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
  // device planes of one batch: inputs (up to 2 D + 3 planes of max_points
  // words) and outputs
  uint32_t* d_in = nullptr;
  int32_t* d_cluster = nullptr;
  int32_t* d_seed = nullptr;
  float* d_rho = nullptr;
  int32_t* d_nh = nullptr;
  AsmEvent* d_asm = nullptr;  // assembly table (max_batch_events entries)
  AsmEvent* h_asm = nullptr;  // its pinned staging
  // pinned staging of the outputs of requests whose buffers are pageable
  int32_t* h_cluster = nullptr;
  int32_t* h_seed = nullptr;
  float* h_rho = nullptr;
  int32_t* h_nh = nullptr;
  std::vector<Request> batch;
  std::vector<int64_t> offsets;
  int64_t bytes = 0;  // device bytes the slot holds
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
  int64_t slot_bytes = 0;  // device bytes of all slots
  // Resident events: a device pool inside the budget, and a pinned host pool
  // staging the inputs of pageable requests on their way up.
  char* pool_base = nullptr;
  char* host_base = nullptr;
  Pool pool, host_pool;
  cudaStream_t upload = nullptr;
  std::vector<cudaEvent_t> spare_events;
  // submitted, not yet admitted (arrival order)
  std::deque<Request> waiting;
  // admitted: (profile, options) -> bucket -> FIFO of resident requests
  std::map<std::pair<int32_t, uint32_t>, std::map<int, std::deque<Request>>> queues;
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
  int64_t resident_peak = 0, admission_waits = 0;
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

using QueueKey = std::pair<int32_t, uint32_t>;

// Oldest admitted request over all queues, or false.
bool oldest_bucket(clue_server* srv, QueueKey* key, int* bucket, double* t) {
  bool found = false;
  for (auto& [k, buckets] : srv->queues)
    for (auto& [b, q] : buckets)
      if (!q.empty() && (!found || q.front().t_submit < *t)) {
        found = true;
        *key = k;
        *bucket = b;
        *t = q.front().t_submit;
      }
  return found;
}

// Points of one profile that wait, admitted or not.
int64_t pending_points(clue_server* srv, int profile) {
  int64_t n = 0;
  for (auto& [k, buckets] : srv->queues)
    if (k.first == profile)
      for (auto& [b, q] : buckets)
        for (auto& r : q)
          n += r.pts.n;
  for (auto& r : srv->waiting)
    if (r.profile == profile)
      n += r.pts.n;
  return n;
}

int64_t admitted_points(clue_server* srv, const QueueKey& key) {
  int64_t n = 0;
  auto it = srv->queues.find(key);
  if (it != srv->queues.end())
    for (auto& [b, q] : it->second)
      for (auto& r : q)
        n += r.pts.n;
  return n;
}

// Batches of fewer points have their time dominated by per-launch latency and
// are not used to learn the per-point cost.
constexpr int64_t kCostSamplePoints = 1 << 16;

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

// Takes a batch of admitted requests of `key`, starting from `bucket`, then
// smaller buckets.
std::vector<Request> take_batch(clue_server* srv, const QueueKey& key, int bucket) {
  std::vector<Request> out;
  int64_t pts = 0;
  const int64_t cap = batch_point_cap(srv, key.first);
  auto& qs = srv->queues[key];
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

cudaEvent_t take_event(clue_server* srv) {
  if (!srv->spare_events.empty()) {
    cudaEvent_t e = srv->spare_events.back();
    srv->spare_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

// Admits waiting requests in arrival order while their resident blocks fit the
// pool (and, for pageable inputs, the pinned staging pool): uploads each on
// the upload stream and queues it for batching. Called with the lock held.
clue_status admit(clue_server* srv) {
  while (!srv->waiting.empty()) {
    Request& r = srv->waiting.front();
    char* dev = srv->pool.alloc(r.bytes);
    if (!dev) {
      srv->admission_waits += 1;
      break;
    }
    char* host = nullptr;
    if (!r.in_pinned && !(host = srv->host_pool.alloc(r.bytes))) {
      srv->pool.release(dev, r.bytes);
      srv->admission_waits += 1;
      break;
    }
    cudaEvent_t ev = take_event(srv);
    if (!ev) {
      srv->pool.release(dev, r.bytes);
      srv->host_pool.release(host, r.bytes);
      return fail(CLUE_ERR_CUDA, "upload event");
    }
    const int D = r.pts.ndim;
    const int planes = planes_of(D, r.opts);
    const size_t nb = (size_t)r.pts.n * 4;
    cudaError_t e = cudaSuccess;
    if (r.in_pinned) {
      for (int k = 0; k < planes && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(dev + k * nb, plane_src(&r.pts, r.opts, k), nb, cudaMemcpyHostToDevice,
                            srv->upload);
    } else {
      for (int k = 0; k < planes; ++k)
        std::memcpy(host + k * nb, plane_src(&r.pts, r.opts, k), nb);
      e = cudaMemcpyAsync(dev, host, nb * planes, cudaMemcpyHostToDevice, srv->upload);
    }
    if (e == cudaSuccess)
      e = cudaEventRecord(ev, srv->upload);
    if (e != cudaSuccess) {
      srv->pool.release(dev, r.bytes);
      srv->host_pool.release(host, r.bytes);
      srv->spare_events.push_back(ev);
      return fail_cuda(e, "event upload");
    }
    r.dev = dev;
    r.host = host;
    r.uploaded = ev;
    srv->resident_peak = std::max(srv->resident_peak, srv->pool.used());
    srv->inflight_peak = std::max(srv->inflight_peak, srv->inflight_bytes + srv->pool.used());
    srv->queues[{r.profile, r.opts}][bucket_of(r.pts.n)].push_back(r);
    srv->waiting.pop_front();
  }
  return CLUE_OK;
}

clue_status launch_batch(clue_server* srv, Slot* s) {
  const Request& r0 = s->batch[0];
  const clue_server_profile& prof = srv->profiles[r0.profile];
  const int D = prof.ndim;
  const uint32_t opts = r0.opts;
  const int planes = planes_of(D, opts);
  const int B = (int)s->batch.size();
  std::vector<uint32_t> sizes(B);
  s->offsets.assign(B + 1, 0);
  int32_t n_max = 0;
  for (int e = 0; e < B; ++e) {
    sizes[e] = (uint32_t)s->batch[e].pts.n;
    s->offsets[e + 1] = s->offsets[e] + sizes[e];
    n_max = std::max<int32_t>(n_max, (int32_t)sizes[e]);
  }
  const int64_t P = s->offsets[B];
  bool want_seed = false, want_rho = false, want_nh = false;
  cudaError_t e;
  // A batch holding an event that is expected to run long goes first on the GPU.
  const double ns = srv->ns_per_point[r0.profile];
  const bool urgent = srv->cfg.priority_ms > 0.0f && ns > 0.0 &&
                      (double)n_max * ns * 1e-6 >= srv->cfg.priority_ms;
  s->active = urgent ? s->stream_hi : s->stream;
  s->profile = r0.profile;
  if ((e = cudaEventRecord(s->ev_start, s->active)))
    return fail_cuda(e, "batch start event");
  // the events' points are resident once their uploads are done
  for (const Request& r : s->batch)
    if ((e = cudaStreamWaitEvent(s->active, r.uploaded, 0)))
      return fail_cuda(e, "wait for upload");
  for (int k = 0; k < B; ++k) {
    const Request& r = s->batch[k];
    s->h_asm[k] = AsmEvent{reinterpret_cast<const uint32_t*>(r.dev), r.pts.n, (int32_t)s->offsets[k]};
    want_seed |= r.pts.is_seed != nullptr;
    want_rho |= r.pts.rho != nullptr;
    want_nh |= r.pts.nearest_higher != nullptr;
  }
  if ((e = cudaMemcpyAsync(s->d_asm, s->h_asm, sizeof(AsmEvent) * B, cudaMemcpyHostToDevice, s->active)))
    return fail_cuda(e, "assembly table");
  {
    const int64_t words = (int64_t)n_max * planes;
    const int gx = (int)std::min<int64_t>((words + 255) / 256, 64);
    k_assemble<<<dim3(gx, B), 256, 0, s->active>>>(s->d_asm, planes, P, s->d_in);
    if ((e = cudaGetLastError()))
      return fail_cuda(e, "batch assembly");
  }
  clue_points dev{};
  dev.ndim = D;
  dev.n = (int32_t)P;
  int k = 0;
  for (int d = 0; d < D; ++d)
    dev.coords[d] = reinterpret_cast<const float*>(s->d_in + (k++) * P);
  dev.weight = reinterpret_cast<const float*>(s->d_in + (k++) * P);
  for (int d = 0; d < D; ++d)
    if (opts & (1u << d))
      dev.sigma[d] = reinterpret_cast<const float*>(s->d_in + (k++) * P);
  if (opts & kOptUnc)
    dev.density_uncertainty = reinterpret_cast<const float*>(s->d_in + (k++) * P);
  if (opts & kOptTags)
    dev.tags = s->d_in + (k++) * P;
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
  for (int k2 = 0; k2 < B; ++k2) {
    const Request& r = s->batch[k2];
    const int64_t off = s->offsets[k2];
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
      void* dst = r.out_pinned ? o.user : o.staging;
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

// Copies staged outputs of pageable requests back, completes the tickets and
// returns the events' resident blocks to the pools.
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
    if (ok && !r.out_pinned) {
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
    srv->pool.release(r.dev, r.bytes);
    srv->host_pool.release(r.host, r.bytes);
    if (r.uploaded)
      srv->spare_events.push_back(r.uploaded);
  }
  srv->inflight_bytes -= s->bytes;
  s->batch.clear();
  s->busy = false;
  srv->cv.notify_all();
}

// Fails every request still waiting for admission (the upload path broke).
void fail_waiting(clue_server* srv, const std::string& why) {
  const double t = now_s();
  for (auto& r : srv->waiting) {
    srv->state[r.ticket] = kFailed;
    srv->t_done[r.ticket] = t;
    srv->completed += 1;
  }
  srv->waiting.clear();
  srv->error = why;
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
    // admit what fits the budget
    if (admit(srv) != CLUE_OK)
      fail_waiting(srv, clue_last_error());
    if (srv->stop) {
      bool busy = false;
      for (Slot* s : srv->slots)
        busy |= s->busy;
      bool pending = !srv->waiting.empty();
      for (auto& [k, buckets] : srv->queues)
        for (auto& [b, q] : buckets)
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
    QueueKey key{0, 0};
    int bucket = 0;
    double t_old = 0;
    if (free_slot && oldest_bucket(srv, &key, &bucket, &t_old)) {
      const double waited_us = (now_s() - t_old) * 1e6;
      const bool small = admitted_points(srv, key) < srv->max_points / 4;
      if (n_busy > 0 && small && waited_us < srv->cfg.linger_us && !srv->stop) {
        srv->cv.wait_for(lock, std::chrono::microseconds(
                                   std::max<int64_t>(1, srv->cfg.linger_us - (int64_t)waited_us)));
        continue;
      }
      free_slot->batch = take_batch(srv, key, bucket);
      for (auto& r : free_slot->batch)
        srv->state[r.ticket] = kRunning;
      free_slot->busy = true;
      srv->inflight_bytes += free_slot->bytes;
      srv->inflight_peak = std::max(srv->inflight_peak, srv->inflight_bytes + srv->pool.used());
      srv->batches += 1;
      lock.unlock();
      clue_status st = launch_batch(srv, free_slot);
      if (st != CLUE_OK) {
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
  for (void* p : {(void*)s->d_in, (void*)s->d_cluster, (void*)s->d_seed, (void*)s->d_rho,
                  (void*)s->d_nh, (void*)s->d_asm})
    if (p)
      cudaFree(p);
  for (void* p : {(void*)s->h_cluster, (void*)s->h_seed, (void*)s->h_rho, (void*)s->h_nh,
                  (void*)s->h_asm})
    if (p)
      cudaFreeHost(p);
  if (s->stream)
    cudaStreamDestroy(s->stream);
  if (s->stream_hi)
    cudaStreamDestroy(s->stream_hi);
  delete s;
}

void free_server(clue_server* srv) {
  for (Slot* s : srv->slots)
    free_slot(s);
  if (srv->upload) {
    cudaStreamSynchronize(srv->upload);
    cudaStreamDestroy(srv->upload);
  }
  for (cudaEvent_t e : srv->spare_events)
    cudaEventDestroy(e);
  if (srv->pool_base)
    cudaFree(srv->pool_base);
  if (srv->host_base)
    cudaFreeHost(srv->host_base);
  delete srv;
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
  srv->ns_per_point.assign(n_profiles, 0.0);
  srv->max_dim = max_dim;
  // Device bytes of one slot for batches of P points: workspace scratch (with
  // room for sigma, uncertainty and tags) plus the batch's input and output
  // planes. A batch size derived from the budget gives the slots at most half
  // of it; a given one gives them what it needs. The rest of the budget holds
  // the resident events.
  const int in_planes = 2 * max_dim + 3;
  const int64_t per_slot = cfg->max_batch_points > 0
                               ? (int64_t)(cfg->budget_bytes / cfg->max_inflight)
                               : (int64_t)(cfg->budget_bytes / 2 / cfg->max_inflight);
  auto slot_bytes = [&](int64_t P, int64_t E) {
    RunShape sh;
    sh.D = max_dim;
    sh.n = P;
    sh.n_events = (int32_t)E;
    sh.n_grids = (int32_t)E;
    sh.n_tiles = tiles_bound(max_dim, P, E);
    sh.n_chunks = (int32_t)(P / kChunkPoints + E + 1);
    return (int64_t)scratch_bytes(sh, true, true, true) + P * (int64_t)(4 * (in_planes + 4));
  };
  int64_t P = cfg->max_batch_points > 0 ? cfg->max_batch_points : (int64_t)1 << 24;
  while (cfg->max_batch_points <= 0 && P > 4096 && slot_bytes(P, cfg->max_batch_events) > per_slot)
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
    const size_t E = (size_t)cfg->max_batch_events;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)) ||
        (e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio_low)) ||
        (e = cudaStreamCreateWithPriority(&s->stream_hi, cudaStreamNonBlocking, prio_high)) ||
        (e = cudaEventCreate(&s->ev_start)) || (e = cudaEventCreate(&s->ev_end)) ||
        (e = cudaMalloc(&s->d_in, P * in_planes * sizeof(uint32_t))) ||
        (e = cudaMalloc(&s->d_cluster, P * sizeof(int32_t))) ||
        (e = cudaMalloc(&s->d_seed, P * sizeof(int32_t))) ||
        (e = cudaMalloc(&s->d_rho, P * sizeof(float))) ||
        (e = cudaMalloc(&s->d_nh, P * sizeof(int32_t))) ||
        (e = cudaMalloc(&s->d_asm, E * sizeof(AsmEvent))) ||
        (e = cudaMallocHost(&s->h_asm, E * sizeof(AsmEvent))) ||
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
      sh.n_chunks = (int32_t)(P / kChunkPoints + cfg->max_batch_events + 1);
      st = ensure_capacity(s->ws, sh, true, true, true, 0);
    }
    if (st != CLUE_OK) {
      free_server(srv);
      return st;
    }
    s->bytes = (int64_t)s->ws->bytes + P * (int64_t)(4 * (in_planes + 4)) + (int64_t)(E * sizeof(AsmEvent));
    srv->slot_bytes += s->bytes;
  }
  // The resident pool: the rest of the budget, which must hold at least one
  // event of the largest batch size; pageable inputs stage through a pinned
  // host pool of one full batch per slot (at most 512 MiB, at least one batch).
  const int64_t pool_bytes = (int64_t)cfg->budget_bytes - srv->slot_bytes;
  const int64_t one_batch = P * (int64_t)in_planes * 4;
  const int64_t host_bytes = std::max<int64_t>(one_batch, std::min<int64_t>(one_batch * cfg->max_inflight, (int64_t)512 << 20));
  clue_status st = CLUE_OK;
  if (pool_bytes < P * (int64_t)in_planes * 4 + 256)
    st = fail(CLUE_ERR_OUT_OF_MEMORY, "the memory budget leaves no room for resident events");
  else if ((e = cudaMalloc(&srv->pool_base, pool_bytes)) ||
           (e = cudaMallocHost(&srv->host_base, host_bytes)) ||
           (e = cudaStreamCreateWithFlags(&srv->upload, cudaStreamNonBlocking)))
    st = fail_cuda(e, "server pool allocation");
  if (st != CLUE_OK) {
    free_server(srv);
    return st;
  }
  srv->pool.init(srv->pool_base, pool_bytes);
  srv->host_pool.init(srv->host_base, host_bytes);
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
  Request r;
  r.profile = profile;
  r.pts = *pts;
  r.opts = options_of(pts);
  r.bytes = (int64_t)pts->n * 4 * planes_of(pts->ndim, r.opts);
  if (pts->n > srv->max_points || r.bytes > srv->pool.size())
    return fail(CLUE_ERR_OUT_OF_MEMORY, "event larger than the server's batch capacity");
  r.in_pinned = true;
  for (int k = 0; k < planes_of(pts->ndim, r.opts); ++k)
    r.in_pinned = r.in_pinned && is_pinned(plane_src(pts, r.opts, k));
  r.out_pinned = true;
  for (const void* o : {(const void*)pts->cluster_index, (const void*)pts->is_seed,
                        (const void*)pts->rho, (const void*)pts->nearest_higher})
    r.out_pinned = r.out_pinned && is_pinned(o);
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
    srv->waiting.push_back(r);
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
    out->resident_bytes_peak = srv->resident_peak;
    out->resident_pool_bytes = srv->pool.size();
    out->slot_bytes = srv->slot_bytes;
    out->admission_waits = srv->admission_waits;
    out->max_batch_points = srv->max_points;
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
  free_server(srv);
  return CLUE_OK;
}

}  // extern "C"
