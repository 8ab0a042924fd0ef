// The served form of the C ABI (include/continuum_cuda.h, cc_server_*): a
// request loop on its own host thread with continuous batching over several
// streams, admission against a device-memory budget, and a lighting cache of
// per-light results kept on the device.
//
// Each launch slot owns a stream, an event and pinned host staging for its
// job table and status words. The loop retires finished launches (results
// become cache entries or are freed), then builds the next launch from the
// queued requests (earliest deadline first, or in arrival order): cache
// lookups first, then device memory for the traced lights (evicting unused
// cache entries least recently used), one job per (request, traced light),
// the copies in, one batched launch, and the copies out. Device memory comes
// from a pool owned by the server (the budget reserved in it at creation),
// allocated and freed in stream order.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "capi_internal.h"

using namespace cc_host;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Per-point bytes of one light's results: full and any words, irradiance, fraction.
constexpr uint64_t kResultBytes = 8 + 8 + 4 + 4;
// Jobs a launch slot's pinned job-table staging holds from the start: a
// launch of 2M cones in requests of at least 16k points and 8 lights has 1,024.
constexpr size_t kStagingJobs = 1024;

struct CacheEntry {
  uint64_t key = 0;
  float geometry[12] = {};  // the light record without its radiance
  uint64_t npoints = 0;
  uint32_t scene = 0, hierarchy = 0;
  float prefilter = 0.0f;
  uint8_t* dev = nullptr;   // npoints x (full | any | irradiance | fraction)
  uint64_t bytes = 0;
  int refs = 0;             // launches in flight reading it
  std::list<CacheEntry*>::iterator lru;
};

struct Request {
  uint64_t ticket = 0;
  cc_request req{};
  std::vector<float> lights;  // copied at submission
  Clock::time_point t_submit, t_admit, t_done;
  Clock::time_point deadline;  // admission order: submission + the options' time per cone
  bool done = false;
  int status = CC_OK;
  std::string error;
  cc_request_stats stats{};
  // Set while in a launch.
  std::vector<CacheEntry*> hit;      // per light: the entry serving it, or null
  std::vector<uint8_t*> result;      // per light: the traced result block, or null
  std::vector<float> traced;         // the traced lights' records, compacted (the copy's source)
  float4* d_receivers = nullptr;
  float4* d_lights = nullptr;
  const cc_scene* scene = nullptr;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  bool large = false;                // the launch runs one request above the launch's cone limit
  size_t trace_row = 0;              // the launch's row in the server's trace (when tracing)
  std::vector<Request*> reqs;
  std::vector<void*> scratch;        // freed when the launch retires
  uint64_t scratch_bytes = 0;        // in_use held by the launch besides result blocks
  cc::JobGpu* host_jobs = nullptr;   // pinned
  size_t host_jobs_cap = 0;
  uint32_t* status = nullptr;        // pinned, kCounterWords
};

}  // namespace

struct cc_server {
  cc_context* ctx = nullptr;
  cc_server_options opt{};
  cudaMemPool_t pool = nullptr;
  std::vector<const cc_scene*> scenes;
  std::vector<Slot> slots;

  std::mutex mu;                     // guards everything below
  std::condition_variable wake;      // the loop: new requests or stop
  std::condition_variable finished;  // waiters: a request completed
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread loop;

  std::list<CacheEntry*> lru;        // front: least recently used
  std::multimap<uint64_t, std::unique_ptr<CacheEntry>> cache;  // by key
  uint64_t in_use = 0, peak = 0;
  uint64_t chunk = 1ull << 22;  // cones a launch's split chunk holds at most

  uint64_t completed = 0, refused = 0, launches = 0, cached_lights = 0, traced_lights = 0;
  // CC_SERVER_TRACE set in the environment at creation: one row per launch
  // (ms since creation: admitted, host time to build and enqueue it, retired;
  // its requests and cones; slots busy when admitted), written to stderr
  // when the server is destroyed.
  bool tracing = false;
  std::chrono::steady_clock::time_point t0;
  struct TraceRow {
    double admitted_ms, enqueue_ms, retired_ms;
    uint64_t requests, cones;
    uint32_t busy;
    double part_ms[5];  // host time in: pool allocations, copies in, walk order, kernel launches, copies out
  };
  std::vector<TraceRow> trace;
  double part_ms[5] = {};  // the launch being built (loop thread only)
};

namespace {

uint64_t request_cones(const cc_request& r) { return r.npoints * (uint64_t)r.nlights; }

// Device bytes a request needs while in flight when `traced` of its lights
// are traced: inputs, results, and its share of the launch's scratch.
uint64_t request_bytes(const cc_request& r, uint64_t traced) {
  const uint64_t P = r.npoints;
  return P * 32 + traced * 64 + traced * P * kResultBytes + traced * P * 4 /* redo */ + P * 4 /* order */ +
         cc::batch_order_scratch_bytes(std::max<uint64_t>(P, 1)) + traced * sizeof(cc::JobGpu) + 4096;
}

// A launch's split-path scratch (cone records and masks) for its largest
// chunk, when it traces `cones` cones: chunks hold at most s->chunk.
uint64_t split_bytes(const cc_server* s, uint64_t cones) {
  return std::min(cones, s->chunk) * (sizeof(cc::ConeRecord) + 256);
}

// Host time of a call, added to part `k` of the launch's trace row (when tracing).
struct PartTimer {
  cc_server* s;
  int k;
  Clock::time_point t;
  PartTimer(cc_server* s_, int k_) : s(s_), k(k_), t(s_->tracing ? Clock::now() : Clock::time_point{}) {}
  ~PartTimer() {
    if (s->tracing) s->part_ms[k] += ms_between(t, Clock::now());
  }
};

void* pool_alloc(cc_server* s, uint64_t bytes, cudaStream_t stream, cudaError_t* e) {
  PartTimer timer(s, 0);
  void* p = nullptr;
  *e = cudaMallocFromPoolAsync(&p, std::max<uint64_t>(bytes, 256), s->pool, stream);
  return *e == cudaSuccess ? p : nullptr;
}

CacheEntry* find_entry(cc_server* s, const cc_request& r, const float* light) {
  auto range = s->cache.equal_range(r.cache_key);
  for (auto it = range.first; it != range.second; ++it) {
    CacheEntry* e = it->second.get();
    if (e->npoints == r.npoints && e->scene == r.scene && e->hierarchy == r.hierarchy &&
        e->prefilter == r.prefilter && std::memcmp(e->geometry, light, sizeof(e->geometry)) == 0)
      return e;
  }
  return nullptr;
}

void touch(cc_server* s, CacheEntry* e) {
  s->lru.erase(e->lru);
  e->lru = s->lru.insert(s->lru.end(), e);
}

// Frees unused cache entries, least recently used first, until `need` more
// bytes fit the budget. Returns whether they fit. (s->mu held.)
bool make_room(cc_server* s, uint64_t need, cudaStream_t stream) {
  auto it = s->lru.begin();
  while (s->in_use + need > s->opt.hbm_budget && it != s->lru.end()) {
    CacheEntry* e = *it;
    if (e->refs > 0) {
      ++it;
      continue;
    }
    it = s->lru.erase(it);
    cudaFreeAsync(e->dev, stream);
    s->in_use -= e->bytes;
    auto range = s->cache.equal_range(e->key);
    for (auto c = range.first; c != range.second; ++c)
      if (c->second.get() == e) {
        s->cache.erase(c);
        break;
      }
  }
  return s->in_use + need <= s->opt.hbm_budget;
}

// Marks a request done. (s->mu held.)
void complete_locked(cc_server* s, Request* r, int status, const std::string& error) {
  r->status = status;
  r->error = error;
  r->done = true;
  r->t_done = Clock::now();
  r->stats.queued_ms = ms_between(r->t_submit, r->t_admit);
  r->stats.total_ms = ms_between(r->t_submit, r->t_done);
  if (status == CC_OK) s->completed++;
  s->finished.notify_all();
}

void release_slot(cc_server* s, Slot& slot) {
  for (void* p : slot.scratch) cudaFreeAsync(p, slot.stream);
  s->in_use -= slot.scratch_bytes;
  slot.scratch.clear();
  slot.scratch_bytes = 0;
  slot.reqs.clear();
  slot.busy = false;
}

// Retires a finished launch: traced results become cache entries (or are
// freed), inputs and scratch are freed, and its requests complete. (s->mu held.)
void retire(cc_server* s, Slot& slot) {
  const bool stack = ((slot.status[1] | slot.status[cc::kCounterWords + 1]) & 2u) != 0;
  if (s->tracing && slot.trace_row < s->trace.size())
    s->trace[slot.trace_row].retired_ms = ms_between(s->t0, Clock::now());
  for (Request* r : slot.reqs) {
    for (size_t l = 0; l < r->result.size(); ++l) {
      if (r->hit[l]) r->hit[l]->refs--;
      uint8_t* block = r->result[l];
      if (!block) continue;
      const uint64_t bytes = r->req.npoints * kResultBytes;
      const float* light = r->lights.data() + 16 * l;
      if (r->req.cache_key && !stack && !find_entry(s, r->req, light)) {
        auto e = std::make_unique<CacheEntry>();
        e->key = r->req.cache_key;
        std::memcpy(e->geometry, light, sizeof(e->geometry));
        e->npoints = r->req.npoints;
        e->scene = r->req.scene;
        e->hierarchy = r->req.hierarchy;
        e->prefilter = r->req.prefilter;
        e->dev = block;
        e->bytes = bytes;
        e->lru = s->lru.insert(s->lru.end(), e.get());
        s->cache.emplace(e->key, std::move(e));
      } else {
        cudaFreeAsync(block, slot.stream);
        s->in_use -= bytes;
      }
    }
    cudaFreeAsync(r->d_receivers, slot.stream);
    if (r->d_lights) cudaFreeAsync(r->d_lights, slot.stream);
    complete_locked(s, r, stack ? CC_ERR_STACK : CC_OK, stack ? "a traversal stack overflowed" : "");
  }
  release_slot(s, slot);
}

// Undoes a launch that failed while being built: its requests fail. (Called
// without s->mu.)
void abandon(cc_server* s, Slot& slot, int status, const std::string& error) {
  cudaStreamSynchronize(slot.stream);
  std::lock_guard<std::mutex> g(s->mu);
  for (Request* r : slot.reqs) {
    for (size_t l = 0; l < r->result.size(); ++l) {
      if (r->hit[l]) r->hit[l]->refs--;
      if (r->result[l]) {
        cudaFreeAsync(r->result[l], slot.stream);
        s->in_use -= r->req.npoints * kResultBytes;
      }
    }
    if (r->d_receivers) cudaFreeAsync(r->d_receivers, slot.stream);
    if (r->d_lights) cudaFreeAsync(r->d_lights, slot.stream);
    complete_locked(s, r, status, error);
  }
  release_slot(s, slot);
}

#define SRV_CUDA(call, what)                                                       \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      abandon(s, slot, e_ == cudaErrorMemoryAllocation ? CC_ERR_OOM : CC_ERR_CUDA, \
              std::string(what) + ": " + cudaGetErrorString(e_));                  \
      return;                                                                      \
    }                                                                              \
  } while (0)

// Builds and enqueues one launch on `slot` from the requests admitted to it
// (their memory already counted in in_use). Called without s->mu: the
// requests and the slot belong to the loop thread until the launch retires.
// A launch's jobs of one kind with their starts (packets, cones, points).
struct JobGroup {
  std::vector<cc::JobGpu> jobs;
  std::vector<uint64_t> cones_of;
  uint64_t points = 0, cones = 0, packets = 0;
  void add(cc::JobGpu j, uint64_t P, uint32_t pw) {
    j.packet_start = packets;
    j.cone_start = cones;
    j.point_start = points;
    packets += (P + pw - 1) / pw;
    cones += P;
    points += P;
    jobs.push_back(j);
    cones_of.push_back(P);
  }
};

#define GROUP_CUDA(call, what)                                                     \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      abandon(s, slot, e_ == cudaErrorMemoryAllocation ? CC_ERR_OOM : CC_ERR_CUDA, \
              std::string(what) + ": " + cudaGetErrorString(e_));                  \
      return false;                                                                \
    }                                                                              \
  } while (0)

// Enqueues one group on the slot's stream: exact jobs through the split path
// (cone setup, packet and solo passes, integration, per chunk), prefiltering
// jobs through the prefiltering kernel (walk and integration in one pass).
// Its job table goes up from `staging` (pinned); its counters land in
// `status` (kCounterWords). Returns false once it has abandoned the launch.
bool enqueue_group(cc_server* s, Slot& slot, JobGroup& g, bool splat, cc::JobGpu* staging, uint32_t* status) {
  cudaStream_t st = slot.stream;
  const uint32_t pw = s->opt.points_per_warp;
  cudaError_t e = cudaSuccess;
  std::memcpy(staging, g.jobs.data(), g.jobs.size() * sizeof(cc::JobGpu));
  const uint64_t sort_bytes = cc::batch_order_scratch_bytes(g.points);
  void* d_jobs = pool_alloc(s, g.jobs.size() * sizeof(cc::JobGpu), st, &e);
  GROUP_CUDA(e, "job table");
  slot.scratch.push_back(d_jobs);
  void* d_redo = pool_alloc(s, g.cones * 4, st, &e);
  GROUP_CUDA(e, "redo list");
  slot.scratch.push_back(d_redo);
  void* d_order = pool_alloc(s, g.points * 4, st, &e);
  GROUP_CUDA(e, "walk order");
  slot.scratch.push_back(d_order);
  void* d_sort = pool_alloc(s, sort_bytes, st, &e);
  GROUP_CUDA(e, "sort scratch");
  slot.scratch.push_back(d_sort);
  void* d_counters = pool_alloc(s, cc::kCounterWords * 4, st, &e);
  GROUP_CUDA(e, "counters");
  slot.scratch.push_back(d_counters);
  std::vector<cc::BatchChunk> chunks;
  void* d_records = nullptr;
  void* d_masks = nullptr;
  if (!splat) {
    chunks = cc::batch_chunks(g.cones_of, pw, s->chunk);
    uint64_t slots = 1;
    for (const cc::BatchChunk& k : chunks) slots = std::max(slots, k.cone_count);
    d_records = pool_alloc(s, slots * sizeof(cc::ConeRecord), st, &e);
    GROUP_CUDA(e, "cone records");
    slot.scratch.push_back(d_records);
    d_masks = pool_alloc(s, slots * 256, st, &e);
    GROUP_CUDA(e, "cone masks");
    slot.scratch.push_back(d_masks);
  }
  GROUP_CUDA(cudaMemcpyAsync(d_jobs, staging, g.jobs.size() * sizeof(cc::JobGpu), cudaMemcpyHostToDevice, st),
             "job table upload");
  GROUP_CUDA(cudaMemsetAsync(d_counters, 0, cc::kCounterWords * 4, st), "counter reset");
  cc::BatchLaunch L{};
  L.jobs = static_cast<const cc::JobGpu*>(d_jobs);
  L.njobs = (uint32_t)g.jobs.size();
  L.packets = g.packets;
  L.points = g.points;
  L.pw = pw;
  L.records = static_cast<cc::ConeRecord*>(d_records);
  for (const cc::JobGpu& j : g.jobs) {
    if (j.query.hierarchy < 2) L.flat_levels = 1;
    if (j.scene.xforms) L.inst = 1;  // an instanced scene: the instanced kernel for the launch
  }
  {
    PartTimer timer(s, 2);
    e = cc::batch_order(L, d_sort, sort_bytes, static_cast<uint32_t*>(d_order), st);
  }
  GROUP_CUDA(e, "walk order");
  L.order = static_cast<const uint32_t*>(d_order);
  uint32_t* counters = static_cast<uint32_t*>(d_counters);
  cc::DevOut o{};
  o.redo_count = counters;
  o.error = counters + 1;
  o.next_packet = counters + 2;
  o.next_solo = counters + 3;
  o.redo_list = static_cast<uint32_t*>(d_redo);
  o.redo_capacity = (uint32_t)std::max<uint64_t>(g.cones, 1);
  o.cov_out = static_cast<float*>(d_masks);
  {
    PartTimer timer(s, 3);
    e = splat ? cc::launch_batch_splat(L, o, false, s->ctx->sm_count, (int)s->opt.blocks_per_sm, st)
              : cc::launch_batch(L, o, chunks.data(), chunks.size(), false, s->ctx->sm_count,
                                 (int)s->opt.blocks_per_sm, st);
  }
  GROUP_CUDA(e, "launch");
  GROUP_CUDA(cudaMemcpyAsync(status, counters, cc::kCounterWords * 4, cudaMemcpyDeviceToHost, st), "status");
  return true;
}

// Builds and enqueues one launch on `slot` from the requests admitted to it
// (their memory already counted in in_use). Called without s->mu: the
// requests and the slot belong to the loop thread until the launch retires.
void launch(cc_server* s, Slot& slot) {
  cudaStream_t st = slot.stream;
  JobGroup exact, splat;  // exact cones; prefiltering cones
  const uint32_t pw = s->opt.points_per_warp;
  cc_options d;
  cc_options_default(&d);
  for (Request* r : slot.reqs) {
    const cc_request& q = r->req;
    const uint64_t P = q.npoints;
    cudaError_t e = cudaSuccess;
    r->d_receivers = static_cast<float4*>(pool_alloc(s, P * 32, st, &e));
    SRV_CUDA(e, "request receivers");
    {
      PartTimer timer(s, 1);
      e = cudaMemcpyAsync(r->d_receivers, q.receivers, P * 32, cudaMemcpyHostToDevice, st);
    }
    SRV_CUDA(e, "request receivers");
    r->traced.clear();
    for (size_t l = 0; l < r->result.size(); ++l)
      if (!r->hit[l]) r->traced.insert(r->traced.end(), r->lights.begin() + 16 * l, r->lights.begin() + 16 * (l + 1));
    if (!r->traced.empty()) {
      r->d_lights = static_cast<float4*>(pool_alloc(s, r->traced.size() * 4, st, &e));
      SRV_CUDA(e, "request lights");
      PartTimer timer(s, 1);
      SRV_CUDA(cudaMemcpyAsync(r->d_lights, r->traced.data(), r->traced.size() * 4, cudaMemcpyHostToDevice, st),
               "request lights");
    }
    const cc_scene* sc = r->scene;
    uint32_t t = 0;
    for (size_t l = 0; l < r->result.size(); ++l) {
      if (r->hit[l]) continue;
      uint8_t* block = static_cast<uint8_t*>(pool_alloc(s, P * kResultBytes, st, &e));
      SRV_CUDA(e, "request results");
      r->result[l] = block;
      cc::JobGpu j{};
      j.scene = sc->dev();  // prefiltering requests: coverage made at submission
      j.query.receivers = r->d_receivers;
      j.query.lights = r->d_lights + 4 * t;
      j.query.npoints = P;
      j.query.nlights = 1;
      j.query.hierarchy = q.hierarchy;
      j.query.prefilter = q.prefilter;
      j.query.wide_extent = d.wide_extent;
      j.query.light_cone_cap = d.light_cone_cap;
      j.query.wide_cone_cap = d.wide_cone_cap;
      j.full = reinterpret_cast<uint2*>(block);
      j.any = reinterpret_cast<uint2*>(block + 8 * P);
      j.irradiance = reinterpret_cast<float*>(block + 16 * P);
      j.fraction = reinterpret_cast<float*>(block + 20 * P);
      if (!sc->flat.nodes.empty())
        for (int k = 0; k < 3; ++k) {
          j.lo[k] = sc->flat.nodes[0].lo[k];
          j.hi[k] = sc->flat.nodes[0].hi[k];
        }
      (q.prefilter > 0.0f ? splat : exact).add(j, P, pw);
      ++t;
    }
  }
  // Each group's scratch: job table, redo list, walk order and its sort,
  // counters, and for exact jobs the split path's records and masks for one
  // chunk. The job tables go up from one pinned staging area.
  const size_t njobs = exact.jobs.size() + splat.jobs.size();
  if (njobs && slot.host_jobs_cap < njobs) {
    if (slot.host_jobs) cudaFreeHost(slot.host_jobs);
    slot.host_jobs = nullptr;
    slot.host_jobs_cap = 0;
    SRV_CUDA(cudaMallocHost(&slot.host_jobs, njobs * 2 * sizeof(cc::JobGpu)), "job table staging");
    slot.host_jobs_cap = njobs * 2;
  }
  std::fill(slot.status, slot.status + 2 * cc::kCounterWords, 0u);
  if (!exact.jobs.empty() && !enqueue_group(s, slot, exact, false, slot.host_jobs, slot.status)) return;
  if (!splat.jobs.empty() &&
      !enqueue_group(s, slot, splat, true, slot.host_jobs + exact.jobs.size(), slot.status + cc::kCounterWords))
    return;
  // Results to the requests' host buffers, light-major.
  PartTimer copies_out(s, 4);
  for (Request* r : slot.reqs) {
    const cc_request& q = r->req;
    const uint64_t P = q.npoints;
    for (size_t l = 0; l < r->result.size(); ++l) {
      const uint8_t* src = r->result[l] ? r->result[l] : r->hit[l]->dev;
      if (q.full) SRV_CUDA(cudaMemcpyAsync(q.full + 2 * P * l, src, 8 * P, cudaMemcpyDeviceToHost, st), "results");
      if (q.any) SRV_CUDA(cudaMemcpyAsync(q.any + 2 * P * l, src + 8 * P, 8 * P, cudaMemcpyDeviceToHost, st), "results");
      if (q.irradiance)
        SRV_CUDA(cudaMemcpyAsync(q.irradiance + P * l, src + 16 * P, 4 * P, cudaMemcpyDeviceToHost, st), "results");
      if (q.fraction)
        SRV_CUDA(cudaMemcpyAsync(q.fraction + P * l, src + 20 * P, 4 * P, cudaMemcpyDeviceToHost, st), "results");
    }
  }
  SRV_CUDA(cudaEventRecord(slot.done, st), "launch event");
  std::lock_guard<std::mutex> g(s->mu);
  s->launches++;
}

// Takes queued requests for a launch, earliest deadline first (arrival order
// among equal deadlines), while they fit: the budget (after evicting unused
// cache entries) and the launch's cone limit. The most urgent request that
// does not fit the memory stops the admission (*blocked: it), so that later
// ones cannot keep it waiting; one that does not fit the launch's cone limit
// is left for the next launch (in arrival order: admission stops there).
// Ordered by deadline, requests above the cone limit (each runs alone) hold
// at most all slots but one while a smaller request waits, so that smaller
// requests find a slot instead of queueing behind long launches (with none
// waiting, the last slot keeps the device busy). *large: the launch takes one.
// Returns the requests taken and the bytes their results hold. (s->mu held.)
std::vector<Request*> admit(cc_server* s, cudaStream_t stream, uint64_t* result_bytes, uint64_t* total_bytes,
                            Request** blocked, bool* large) {
  std::vector<Request*> taken;
  uint64_t cones = 0;
  *result_bytes = *total_bytes = 0;
  *blocked = nullptr;
  *large = false;
  uint32_t large_busy = 0;
  for (const Slot& slot : s->slots) large_busy += slot.busy && slot.large;
  bool small_waits = false;  // a queued request within the cone limit (before cache hits)
  for (const Request* r : s->queue) small_waits = small_waits || request_cones(r->req) <= s->opt.max_launch_cones;
  std::vector<Request*> order(s->queue.begin(), s->queue.end());
  std::stable_sort(order.begin(), order.end(),
                   [](const Request* a, const Request* b) { return a->deadline < b->deadline; });
  const bool arrival = s->opt.deadline_ns_per_cone == 0;
  for (Request* r : order) {
    const cc_request& q = r->req;
    // Lighting-cache lookups (entries found stay referenced by this launch).
    std::vector<CacheEntry*> hit(q.nlights, nullptr);
    uint64_t traced = 0;
    for (uint32_t l = 0; l < q.nlights; ++l) {
      if (q.cache_key) hit[l] = find_entry(s, q, r->lights.data() + 16 * l);
      if (!hit[l]) ++traced;
    }
    const uint64_t c = traced * q.npoints;
    if (!taken.empty() && cones + c > s->opt.max_launch_cones) {
      if (arrival) break;
      continue;
    }
    const bool is_large = c > s->opt.max_launch_cones;
    if (!arrival && is_large && small_waits && s->opt.max_inflight > 1 && large_busy + 1 >= s->opt.max_inflight)
      continue;
    for (CacheEntry* e : hit)
      if (e) e->refs++;  // keep them through make_room
    // The request's bytes, and what it adds to the launch's split scratch.
    const uint64_t need = request_bytes(q, traced) + split_bytes(s, cones + c) - split_bytes(s, cones);
    if (!make_room(s, need, stream)) {
      for (CacheEntry* e : hit)
        if (e) e->refs--;
      *blocked = r;
      break;
    }
    for (CacheEntry* e : hit)
      if (e) touch(s, e);
    r->hit = std::move(hit);
    r->result.assign(q.nlights, nullptr);
    r->t_admit = Clock::now();
    r->scene = s->scenes[q.scene];
    r->stats.cached_lights = (uint32_t)(q.nlights - traced);
    s->cached_lights += q.nlights - traced;
    s->traced_lights += traced;
    s->in_use += need;
    s->peak = std::max(s->peak, s->in_use);
    *result_bytes += traced * q.npoints * kResultBytes;
    *total_bytes += need;
    taken.push_back(r);
    cones += c;
    *large = is_large;
  }
  if (!taken.empty()) {
    std::deque<Request*> rest;
    for (Request* r : s->queue)
      if (std::find(taken.begin(), taken.end(), r) == taken.end()) rest.push_back(r);
    s->queue.swap(rest);
  }
  for (Request* r : taken) r->stats.launch_requests = (uint32_t)taken.size();
  return taken;
}

void run_loop(cc_server* s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool any_busy = false;
    for (Slot& slot : s->slots) {
      if (!slot.busy) continue;
      if (cudaEventQuery(slot.done) == cudaSuccess) retire(s, slot);
      else any_busy = true;
    }
    if (s->stop && s->queue.empty() && !any_busy) break;
    Slot* free_slot = nullptr;
    for (Slot& slot : s->slots)
      if (!slot.busy) {
        free_slot = &slot;
        break;
      }
    if (free_slot && !s->queue.empty()) {
      uint64_t result_bytes = 0, total_bytes = 0;
      Request* blocked = nullptr;
      bool large = false;
      std::vector<Request*> taken = admit(s, free_slot->stream, &result_bytes, &total_bytes, &blocked, &large);
      if (!taken.empty()) {
        // Result blocks are released one by one (or kept as cache entries);
        // the rest of the admitted bytes are released with the launch.
        free_slot->scratch_bytes = total_bytes - result_bytes;
        free_slot->reqs = std::move(taken);
        free_slot->busy = true;
        free_slot->large = large;
        const Clock::time_point t_launch = Clock::now();
        if (s->tracing) {
          uint32_t busy = 0;
          uint64_t cones = 0;
          for (const Slot& sl : s->slots) busy += sl.busy;
          for (const Request* r : free_slot->reqs) cones += request_cones(r->req);
          free_slot->trace_row = s->trace.size();
          s->trace.push_back({ms_between(s->t0, t_launch), 0.0, 0.0, free_slot->reqs.size(), cones, busy, {}});
        }
        const size_t row = free_slot->trace_row;
        std::fill(s->part_ms, s->part_ms + 5, 0.0);
        lk.unlock();
        launch(s, *free_slot);
        lk.lock();
        if (s->tracing && row < s->trace.size()) {
          s->trace[row].enqueue_ms = ms_between(t_launch, Clock::now());
          std::copy(s->part_ms, s->part_ms + 5, s->trace[row].part_ms);
        }
        continue;
      }
      if (!any_busy && blocked) {
        // Nothing in flight and the cache emptied, yet the most urgent request
        // does not fit: it never will.
        Request* r = blocked;
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
        s->refused++;
        r->t_admit = Clock::now();
        complete_locked(s, r, CC_ERR_BUSY, "the request does not fit the server's memory budget");
        continue;
      }
    }
    if (any_busy) {
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(100));
      lk.lock();
    } else if (s->queue.empty() && !s->stop) {
      s->wake.wait_for(lk, std::chrono::milliseconds(50));
    }
  }
}

}  // namespace

void cc_server_options_default(cc_server_options* opt) {
  if (!opt) return;
  opt->hbm_budget = 8ull << 30;
  opt->max_inflight = 4;
  opt->max_queue = 256;
  opt->max_launch_cones = 2ull << 20;
  opt->points_per_warp = 32;
  opt->blocks_per_sm = cc::kBlocksPerSm;
  opt->deadline_ns_per_cone = 12;
}

int cc_server_create(cc_context* ctx, const cc_server_options* opt_in, cc_server** out) {
  if (!ctx || !out) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  cc_server_options opt;
  if (opt_in) opt = *opt_in; else cc_server_options_default(&opt);
  if (opt.max_inflight < 1 || opt.max_inflight > 8) return fail(CC_ERR_INVALID, "max_inflight must be 1..8");
  if (opt.points_per_warp < 1 || opt.points_per_warp > 32) return fail(CC_ERR_INVALID, "points_per_warp must be 1..32");
  if (opt.blocks_per_sm < 1 || opt.blocks_per_sm > (uint32_t)cc::kBlocksPerSm)
    return fail(CC_ERR_INVALID, "blocks_per_sm must be 1..8");
  if (opt.max_queue < 1 || opt.hbm_budget == 0 || opt.max_launch_cones == 0)
    return fail(CC_ERR_INVALID, "zero queue, budget or launch size");
  int rc = set_device(ctx);
  if (rc) return rc;
  cc_server* s = new cc_server;
  s->ctx = ctx;
  s->opt = opt;
  s->tracing = std::getenv("CC_SERVER_TRACE") != nullptr;
  s->t0 = Clock::now();
  s->chunk = std::min<uint64_t>(s->chunk, ctx->split_chunk);
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = ~0ull;  // keep freed memory in the pool for reuse
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  s->slots.resize(opt.max_inflight);
  for (Slot& slot : s->slots) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&slot.status, 2 * cc::kCounterWords * sizeof(uint32_t));
    // Job-table staging for launches of up to kStagingJobs jobs, made here:
    // a pinned allocation (or free) while launches run waits for the whole
    // device, so the loop grows it only for a launch of more jobs.
    if (e == cudaSuccess) e = cudaMallocHost(&slot.host_jobs, kStagingJobs * sizeof(cc::JobGpu));
    if (e == cudaSuccess) slot.host_jobs_cap = kStagingJobs;
  }
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "server setup");
    cc_server_destroy(s);
    return rc;
  }
  // The budget is reserved in the pool now (its memory stays in the pool,
  // whose release threshold is unlimited): growing the pool while launches
  // run stalled the loop thread inside cudaMallocFromPoolAsync for up to
  // 1.4 s at a time, with the device idle. Without room for the whole budget
  // the pool grows on demand, as before.
  {
    const Clock::time_point t = Clock::now();
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, opt.hbm_budget, s->pool, s->slots[0].stream) == cudaSuccess) {
      cudaFreeAsync(p, s->slots[0].stream);
      cudaStreamSynchronize(s->slots[0].stream);
    } else {
      cudaGetLastError();  // not an error of the server's
    }
    if (s->tracing) std::fprintf(stderr, "cc_server trace: reserved %.2f GiB in %.1f ms\n",
                                 opt.hbm_budget / 1073741824.0, ms_between(t, Clock::now()));
  }
  s->loop = std::thread(run_loop, s);
  *out = s;
  return CC_OK;
}

int cc_server_destroy(cc_server* s) {
  if (!s) return CC_OK;
  if (s->loop.joinable()) {
    {
      std::lock_guard<std::mutex> g(s->mu);
      s->stop = true;
    }
    s->wake.notify_all();
    s->loop.join();
  }
  cudaSetDevice(s->ctx->device);
  if (!s->slots.empty() && s->slots[0].stream)
    for (auto& kv : s->cache) cudaFreeAsync(kv.second->dev, s->slots[0].stream);
  for (Slot& slot : s->slots) {
    if (slot.stream) cudaStreamSynchronize(slot.stream);
    if (slot.host_jobs) cudaFreeHost(slot.host_jobs);
    if (slot.status) cudaFreeHost(slot.status);
    if (slot.done) cudaEventDestroy(slot.done);
    if (slot.stream) cudaStreamDestroy(slot.stream);
  }
  if (s->pool) cudaMemPoolDestroy(s->pool);
  if (s->tracing) {
    std::fprintf(stderr,
                 "cc_server trace: admitted_ms enqueue_ms retired_ms requests cones slots_busy alloc_ms copy_in_ms "
                 "order_ms kernels_ms copy_out_ms\n");
    for (const auto& t : s->trace)
      std::fprintf(stderr, "cc_server trace: %.2f %.2f %.2f %llu %llu %u %.2f %.2f %.2f %.2f %.2f\n", t.admitted_ms,
                   t.enqueue_ms, t.retired_ms, (unsigned long long)t.requests, (unsigned long long)t.cones, t.busy,
                   t.part_ms[0], t.part_ms[1], t.part_ms[2], t.part_ms[3], t.part_ms[4]);
  }
  delete s;
  return CC_OK;
}

int cc_server_add_scene(cc_server* s, const cc_scene* scene, uint32_t* id) {
  if (!s || !scene) return fail(CC_ERR_INVALID, "null argument");
  if (scene->ctx != s->ctx) return fail(CC_ERR_INVALID, "scene belongs to another context (or to none)");
  std::lock_guard<std::mutex> g(s->mu);
  if (id) *id = (uint32_t)s->scenes.size();
  s->scenes.push_back(scene);
  return CC_OK;
}

int cc_server_submit(cc_server* s, const cc_request* req, uint64_t* ticket) {
  if (!s || !req) return fail(CC_ERR_INVALID, "null argument");
  if ((req->npoints && !req->receivers) || (req->nlights && !req->lights))
    return fail(CC_ERR_INVALID, "null inputs");
  if (req->hierarchy > 2) return fail(CC_ERR_INVALID, "hierarchy must be 0, 1 or 2");
  if (!(req->prefilter >= 0.0f)) return fail(CC_ERR_INVALID, "prefilter must be >= 0");
  if (req->prefilter > 0.0f && req->hierarchy != 2) return fail(CC_ERR_INVALID, "prefiltered cones need hierarchy 2");
  if (req->npoints >= (1ull << 31)) return fail(CC_ERR_INVALID, "more than 2^31 - 1 points in one request");
  if (request_cones(*req) >= 0xffffffffull) return fail(CC_ERR_INVALID, "more than 2^32 - 1 cones in one request");
  auto r = std::make_unique<Request>();
  r->req = *req;
  r->lights.assign(req->lights, req->lights + 16 * (size_t)req->nlights);
  r->t_submit = Clock::now();
  r->deadline = r->t_submit + std::chrono::nanoseconds(request_cones(*req) * s->opt.deadline_ns_per_cone);
  std::lock_guard<std::mutex> g(s->mu);
  if (req->scene >= s->scenes.size()) return fail(CC_ERR_INVALID, "unknown scene");
  if (req->prefilter > 0.0f) {
    // The scene's coverage samples, made before the request can be launched
    // (submissions are serialized by the lock; exact launches never read
    // them).
    int rc = set_device(s->ctx);
    if (rc) return rc;
    if ((rc = cc_host::scene_coverage(const_cast<cc_scene*>(s->scenes[req->scene])))) return rc;
  }
  if (s->queue.size() >= s->opt.max_queue) {
    s->refused++;
    return fail(CC_ERR_BUSY, "the server's queue is full");
  }
  if (request_bytes(*req, req->nlights) + split_bytes(s, request_cones(*req)) > s->opt.hbm_budget) {
    s->refused++;
    return fail(CC_ERR_BUSY, "the request alone exceeds the server's memory budget");
  }
  r->ticket = s->next_ticket++;
  if (ticket) *ticket = r->ticket;
  s->queue.push_back(r.get());
  s->requests.emplace(r->ticket, std::move(r));
  s->wake.notify_all();
  return CC_OK;
}

int cc_server_wait(cc_server* s, uint64_t ticket, uint32_t timeout_ms, cc_request_stats* stats) {
  if (!s) return fail(CC_ERR_INVALID, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return fail(CC_ERR_INVALID, "unknown ticket");
  Request* r = it->second.get();
  if (!s->finished.wait_for(lk, std::chrono::milliseconds(timeout_ms), [r] { return r->done; }))
    return fail(CC_ERR_TIMEOUT, "the request has not finished");
  const int status = r->status;
  const std::string error = r->error;
  if (stats) *stats = r->stats;
  s->requests.erase(it);
  if (status != CC_OK) return fail(status, error);
  return CC_OK;
}

int cc_server_stats(cc_server* s, uint64_t out8[8]) {
  if (!s || !out8) return fail(CC_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(s->mu);
  out8[0] = s->completed;
  out8[1] = s->refused;
  out8[2] = s->launches;
  out8[3] = s->cached_lights;
  out8[4] = s->traced_lights;
  out8[5] = s->in_use;
  out8[6] = s->peak;
  out8[7] = s->cache.size();
  return CC_OK;
}
