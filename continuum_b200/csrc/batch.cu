// The batched form of the C ABI (include/continuum_cuda.h, cc_batch_*): a job
// table on the device, one Morton sort over every job's points and one
// persistent launch over every job's packets, optionally replayed from a
// captured CUDA graph, and an autotuner over the launch configuration.
#include <chrono>
#include <thread>

#include "capi_internal.h"

using namespace cc_host;

struct cc_batch {
  cc_context* ctx = nullptr;
  std::vector<cc::JobGpu> jobs;  // host copy; the starts are set by prepare()
  bool count_work = false;       // some job wants work counters
  bool instanced = false;        // some job's scene is instanced
  // Update jobs (cc_batch_add_update): the job and its stale bytes. Each
  // submission lists the stale cones of the job's grid in its walk order
  // (its slice of upd_list at the job's first cone, its length in
  // upd_count[k]) and walks only those.
  struct Update {
    uint32_t job;
    const uint8_t* stale;
  };
  std::vector<Update> updates;
  DevBuf upd_perm, upd_flags, upd_list, upd_count, upd_temp;
  // Prefiltering jobs (cc_options.prefilter > 0): a table of their own,
  // walked by the prefiltering kernel (which integrates in the walk) in a
  // second launch after the exact jobs' split path, with its own walk order,
  // re-walk list and counters (words 4-7).
  std::vector<cc::JobGpu> splat_jobs;
  bool splat_instanced = false;
  uint64_t splat_points = 0, splat_cones = 0, splat_packets = 0;
  DevBuf splat_table, splat_redo, splat_order, splat_sort_scratch;
  uint64_t points = 0, cones = 0;
  // Device state, sized by prepare().
  DevBuf job_table, redo, order, sort_scratch, counters;
  DevBuf records, masks;               // the split path's scratch, one chunk
  std::vector<cc::BatchChunk> chunks;  // the split path's chunks, set by prepare()
  uint32_t* status = nullptr;    // pinned: the counters (both launches') copied back after each submission
  cudaEvent_t done = nullptr;
  bool prepared = false;
  uint32_t prepared_pw = 0;
  uint64_t prepared_chunk = 0;
  uint64_t packets = 0;
  // The captured graph and the options it was captured with.
  cudaGraphExec_t graph = nullptr;
  cc_batch_options graph_opt{};
  bool submitted = false;
};

namespace {

bool same(const cc_batch_options& a, const cc_batch_options& b) {
  return a.points_per_warp == b.points_per_warp && a.blocks_per_sm == b.blocks_per_sm && a.flags == b.flags;
}

void drop_graph(cc_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

int check_options(const cc_batch_options& o) {
  if (o.points_per_warp < 1 || o.points_per_warp > 32) return fail(CC_ERR_INVALID, "points_per_warp must be 1..32");
  if (o.blocks_per_sm < 1 || o.blocks_per_sm > (uint32_t)cc::kBlocksPerSm)
    return fail(CC_ERR_INVALID, "blocks_per_sm must be 1..8");
  if (o.flags & ~(CC_KEEP_ORDER | CC_NO_REDO | CC_BATCH_GRAPH)) return fail(CC_ERR_INVALID, "unknown batch flag");
  return CC_OK;
}

// Sets each job's packet, cone and point starts for `pw` cones per packet,
// sizes the device buffers and uploads the job table. The previous
// submission has finished.
int prepare(cc_batch* b, uint32_t pw) {
  if (b->prepared && b->prepared_pw == pw && b->prepared_chunk == b->ctx->split_chunk) return CC_OK;
  drop_graph(b);
  uint64_t packet = 0, cone = 0, point = 0;
  std::vector<uint64_t> job_cones;
  for (cc::JobGpu& j : b->jobs) {
    const uint64_t c = j.query.npoints * (uint64_t)j.query.nlights;
    job_cones.push_back(c);
    j.packet_start = packet;
    j.cone_start = cone;
    j.point_start = point;
    packet += (c + pw - 1) / pw;
    cone += c;
    point += j.query.npoints;
  }
  b->packets = packet;
  b->chunks = cc::batch_chunks(job_cones, pw, b->ctx->split_chunk);
  if (!b->updates.empty()) {
    size_t temp = 256;
    for (const cc_batch::Update& u : b->updates)
      temp = std::max(temp, cc::stale_list_scratch_bytes(job_cones[u.job]));
    CC_CUDA(b->upd_perm.reserve(std::max<uint64_t>(cone, 1) * 4), "batch update scratch");
    CC_CUDA(b->upd_flags.reserve(std::max<uint64_t>(cone, 1)), "batch update scratch");
    CC_CUDA(b->upd_list.reserve(std::max<uint64_t>(cone, 1) * 4), "batch update lists");
    CC_CUDA(b->upd_count.reserve(b->updates.size() * 4), "batch update counts");
    CC_CUDA(b->upd_temp.reserve(temp), "batch update scratch");
    uint32_t* list = static_cast<uint32_t*>(b->upd_list.ptr);
    uint32_t* count = static_cast<uint32_t*>(b->upd_count.ptr);
    for (size_t k = 0; k < b->updates.size(); ++k) {
      cc::JobGpu& j = b->jobs[b->updates[k].job];
      j.query.cones = list + j.cone_start;
      j.query.cones_count = count + k;
    }
  }
  uint64_t slots = 1;
  for (const cc::BatchChunk& k : b->chunks) slots = std::max(slots, k.cone_count);
  CC_CUDA(b->records.reserve(slots * sizeof(cc::ConeRecord)), "batch cone records");
  CC_CUDA(b->masks.reserve(slots * 256), "batch cone masks");
  CC_CUDA(b->job_table.reserve(std::max<size_t>(b->jobs.size(), 1) * sizeof(cc::JobGpu)), "batch job table");
  CC_CUDA(b->redo.reserve(std::max<uint64_t>(cone, 1) * 4), "batch redo list");
  CC_CUDA(b->order.reserve(std::max<uint64_t>(point, 1) * 4), "batch walk order");
  CC_CUDA(b->sort_scratch.reserve(cc::batch_order_scratch_bytes(std::max<uint64_t>(point, 1))), "batch sort scratch");
  CC_CUDA(b->counters.reserve(2 * cc::kCounterWords * sizeof(uint32_t)), "batch counters");
  if (!b->jobs.empty())
    CC_CUDA(cudaMemcpy(b->job_table.ptr, b->jobs.data(), b->jobs.size() * sizeof(cc::JobGpu), cudaMemcpyHostToDevice),
            "batch job table upload");
  if (!b->splat_jobs.empty()) {
    uint64_t sp = 0, sc = 0, spt = 0;
    for (cc::JobGpu& j : b->splat_jobs) {
      const uint64_t c = j.query.npoints * (uint64_t)j.query.nlights;
      j.packet_start = sp;
      j.cone_start = sc;
      j.point_start = spt;
      sp += (c + pw - 1) / pw;
      sc += c;
      spt += j.query.npoints;
    }
    b->splat_packets = sp;
    CC_CUDA(b->splat_table.reserve(b->splat_jobs.size() * sizeof(cc::JobGpu)), "batch prefiltering job table");
    CC_CUDA(b->splat_redo.reserve(std::max<uint64_t>(sc, 1) * 4), "batch prefiltering redo list");
    CC_CUDA(b->splat_order.reserve(std::max<uint64_t>(spt, 1) * 4), "batch prefiltering walk order");
    CC_CUDA(b->splat_sort_scratch.reserve(cc::batch_order_scratch_bytes(std::max<uint64_t>(spt, 1))),
            "batch prefiltering sort scratch");
    CC_CUDA(cudaMemcpy(b->splat_table.ptr, b->splat_jobs.data(), b->splat_jobs.size() * sizeof(cc::JobGpu),
                       cudaMemcpyHostToDevice),
            "batch prefiltering job table upload");
  }
  b->prepared = true;
  b->prepared_pw = pw;
  b->prepared_chunk = b->ctx->split_chunk;
  return CC_OK;
}

// The submission's work on `stream`: counter reset, walk order, the packet
// and solo passes, and the counters' copy to pinned host memory.
int enqueue(cc_batch* b, const cc_batch_options& opt, cudaStream_t stream) {
  uint32_t* counters = static_cast<uint32_t*>(b->counters.ptr);
  CC_CUDA(cudaMemsetAsync(counters, 0, 2 * cc::kCounterWords * sizeof(uint32_t), stream), "batch counter reset");
  cc::BatchLaunch L{};
  L.jobs = static_cast<const cc::JobGpu*>(b->job_table.ptr);
  L.njobs = (uint32_t)b->jobs.size();
  L.packets = b->packets;
  L.points = b->points;
  L.pw = opt.points_per_warp;
  L.order = nullptr;
  L.records = static_cast<cc::ConeRecord*>(b->records.ptr);
  for (const cc::JobGpu& j : b->jobs)
    if (j.query.hierarchy < 2) L.flat_levels = 1;
  L.inst = b->instanced ? 1u : 0u;
  if (!(opt.flags & CC_KEEP_ORDER) && b->points > 0) {
    CC_CUDA(cc::batch_order(L, b->sort_scratch.ptr, b->sort_scratch.size, static_cast<uint32_t*>(b->order.ptr),
                            stream),
            "batch walk order");
    L.order = static_cast<const uint32_t*>(b->order.ptr);
  }
  // Update jobs: their stale cones as lists, each light's in the walk order.
  for (size_t k = 0; k < b->updates.size(); ++k) {
    const cc::JobGpu& j = b->jobs[b->updates[k].job];
    const uint64_t at = j.cone_start;
    CC_CUDA(cc::stale_list(L.order ? L.order + j.point_start : nullptr, b->updates[k].stale, j.query.npoints,
                           j.query.nlights, static_cast<uint32_t*>(b->upd_perm.ptr) + at,
                           static_cast<uint8_t*>(b->upd_flags.ptr) + at, static_cast<uint32_t*>(b->upd_list.ptr) + at,
                           static_cast<uint32_t*>(b->upd_count.ptr) + k, b->upd_temp.ptr, b->upd_temp.size, stream),
            "batch update list");
  }
  cc::DevOut o{};
  o.redo_count = counters;
  o.error = counters + 1;
  o.next_packet = counters + 2;
  o.next_solo = counters + 3;
  if (!(opt.flags & CC_NO_REDO)) {
    o.redo_list = static_cast<uint32_t*>(b->redo.ptr);
    o.redo_capacity = (uint32_t)std::max<uint64_t>(b->cones, 1);
  }
  o.cov_out = static_cast<float*>(b->masks.ptr);
  if (!b->jobs.empty())
    CC_CUDA(cc::launch_batch(L, o, b->chunks.data(), b->chunks.size(), b->count_work, b->ctx->sm_count,
                             (int)opt.blocks_per_sm, stream),
            "batch launch");
  if (!b->splat_jobs.empty()) {
    cc::BatchLaunch S{};
    S.jobs = static_cast<const cc::JobGpu*>(b->splat_table.ptr);
    S.njobs = (uint32_t)b->splat_jobs.size();
    S.packets = b->splat_packets;
    S.points = b->splat_points;
    S.pw = opt.points_per_warp;
    S.inst = b->splat_instanced ? 1u : 0u;
    if (!(opt.flags & CC_KEEP_ORDER) && b->splat_points > 0) {
      CC_CUDA(cc::batch_order(S, b->splat_sort_scratch.ptr, b->splat_sort_scratch.size,
                              static_cast<uint32_t*>(b->splat_order.ptr), stream),
              "batch prefiltering walk order");
      S.order = static_cast<const uint32_t*>(b->splat_order.ptr);
    }
    cc::DevOut so{};
    uint32_t* sc = counters + cc::kCounterWords;
    so.redo_count = sc;
    so.error = sc + 1;
    so.next_packet = sc + 2;
    so.next_solo = sc + 3;
    if (!(opt.flags & CC_NO_REDO)) {
      so.redo_list = static_cast<uint32_t*>(b->splat_redo.ptr);
      so.redo_capacity = (uint32_t)std::max<uint64_t>(b->splat_cones, 1);
    }
    CC_CUDA(cc::launch_batch_splat(S, so, b->count_work, b->ctx->sm_count, (int)opt.blocks_per_sm, stream),
            "batch prefiltering launch");
  }
  CC_CUDA(cudaMemcpyAsync(b->status, counters, 2 * cc::kCounterWords * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                          stream),
          "batch status copy");
  return CC_OK;
}

int submit(cc_batch* b, const cc_batch_options& opt, cudaStream_t stream) {
  int rc = prepare(b, opt.points_per_warp);
  if (rc) return rc;
  if (opt.flags & CC_BATCH_GRAPH) {
    if (b->graph && same(b->graph_opt, opt)) {
      CC_CUDA(cudaGraphLaunch(b->graph, stream), "batch graph launch");
    } else {
      drop_graph(b);
      // Run directly (this loads every kernel's module and sets their
      // attributes), then capture the same work for later submissions.
      rc = enqueue(b, opt, stream);
      if (rc) return rc;
      CC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "batch graph capture");
      rc = enqueue(b, opt, stream);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(stream, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
      e = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        b->graph = nullptr;
        return cuda_fail(e, "batch graph instantiate");
      }
      b->graph_opt = opt;
    }
  } else {
    rc = enqueue(b, opt, stream);
    if (rc) return rc;
  }
  CC_CUDA(cudaEventRecord(b->done, stream), "batch event");
  b->submitted = true;
  return CC_OK;
}

int wait_done(cc_batch* b, uint32_t timeout_ms) {
  if (!b->submitted) return CC_OK;
  const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  for (;;) {
    cudaError_t e = cudaEventQuery(b->done);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_fail(e, "batch");
    if (std::chrono::steady_clock::now() >= until) return fail(CC_ERR_TIMEOUT, "the batch has not finished");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  const uint32_t error = b->status[1] | b->status[cc::kCounterWords + 1];
  if (error & 2u) return fail(CC_ERR_STACK, "a traversal stack overflowed");
  if (error & 1u) return fail(CC_ERR_INVALID, "solo re-walk list overflowed");
  return CC_OK;
}

}  // namespace

void cc_batch_options_default(cc_batch_options* opt) {
  if (!opt) return;
  opt->points_per_warp = 32;
  opt->blocks_per_sm = cc::kBlocksPerSm;
  opt->flags = CC_BATCH_GRAPH;
}

int cc_batch_create(cc_context* ctx, cc_batch** out) {
  if (!ctx || !out) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  int rc = set_device(ctx);
  if (rc) return rc;
  cc_batch* b = new cc_batch;
  b->ctx = ctx;
  cudaError_t e = cudaMallocHost(&b->status, 2 * cc::kCounterWords * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "batch setup");
    cc_batch_destroy(b);
    return rc;
  }
  std::fill(b->status, b->status + 2 * cc::kCounterWords, 0u);
  *out = b;
  return CC_OK;
}

int cc_batch_destroy(cc_batch* b) {
  if (!b) return CC_OK;
  cudaSetDevice(b->ctx->device);
  if (b->submitted && b->done) cudaEventSynchronize(b->done);
  drop_graph(b);
  for (DevBuf* d : {&b->job_table, &b->redo, &b->order, &b->sort_scratch, &b->counters, &b->records, &b->masks})
    d->release();
  if (b->status) cudaFreeHost(b->status);
  if (b->done) cudaEventDestroy(b->done);
  delete b;
  return CC_OK;
}

int cc_batch_clear(cc_batch* b) {
  if (!b) return fail(CC_ERR_INVALID, "null argument");
  int rc = set_device(b->ctx);
  if (rc) return rc;
  if (b->submitted) CC_CUDA(cudaEventSynchronize(b->done), "batch");
  drop_graph(b);
  b->jobs.clear();
  b->updates.clear();
  b->instanced = false;
  b->splat_jobs.clear();
  b->splat_instanced = false;
  b->splat_points = b->splat_cones = b->splat_packets = 0;
  b->count_work = false;
  b->points = b->cones = 0;
  b->prepared = false;
  return CC_OK;
}

namespace {

// A job of every cone of its grid, or (stale non-null) an update job.
int add_job(cc_batch* b, const cc_scene* scene, const float* receivers, uint64_t npoints, const float* lights,
            uint32_t nlights, const uint8_t* stale, const cc_options* opt_in, const cc_outputs* out, uint32_t* job) {
  if (!b || !scene || !out) return fail(CC_ERR_INVALID, "null argument");
  if (scene->ctx != b->ctx) return fail(CC_ERR_INVALID, "scene belongs to another context (or to none)");
  if ((npoints && !receivers) || (nlights && !lights)) return fail(CC_ERR_INVALID, "null inputs");
  if (stale && (out->partial || out->work))
    return fail(CC_ERR_INVALID, "an update job writes full, any, irradiance and fraction only");
  cc_options opt;
  if (opt_in) opt = *opt_in; else cc_options_default(&opt);
  if (opt.hierarchy > 2) return fail(CC_ERR_INVALID, "hierarchy must be 0, 1 or 2");
  if (!(opt.prefilter >= 0.0f)) return fail(CC_ERR_INVALID, "prefilter must be >= 0");
  const bool splat = opt.prefilter > 0.0f;
  if (splat && opt.hierarchy != 2) return fail(CC_ERR_INVALID, "prefiltered cones need hierarchy 2");
  if (splat && stale) return fail(CC_ERR_INVALID, "update jobs take exact cones (prefilter 0)");
  if (npoints >= (1ull << 31)) return fail(CC_ERR_INVALID, "more than 2^31 - 1 points in one job");
  const uint64_t cones = npoints * (uint64_t)nlights;
  if (b->cones + b->splat_cones + cones >= 0xffffffffull)
    return fail(CC_ERR_INVALID, "more than 2^32 - 1 cones in one batch");
  if (b->jobs.size() >= 0xfffffffeull) return fail(CC_ERR_INVALID, "too many jobs");
  auto misaligned = [](const void* p, uintptr_t a) { return p && (reinterpret_cast<uintptr_t>(p) % a) != 0; };
  if (misaligned(receivers, 16) || misaligned(lights, 16) || misaligned(out->partial, 16) ||
      misaligned(out->work, 16) || misaligned(out->full, 8) || misaligned(out->any, 8) ||
      misaligned(out->irradiance, 4) || misaligned(out->fraction, 4))
    return fail(CC_ERR_INVALID, "device buffers must be aligned (receivers, lights, partial, work: 16 B; full, any: 8 B)");
  if (b->submitted) {
    int rc = set_device(b->ctx);
    if (rc) return rc;
    CC_CUDA(cudaEventSynchronize(b->done), "batch");
  }
  if (splat) {
    // The scene's coverage samples on the device (as a prefiltered
    // cc_visibility call makes them).
    int rc = set_device(b->ctx);
    if (rc) return rc;
    if ((rc = cc_host::scene_coverage(const_cast<cc_scene*>(scene)))) return rc;
  }
  cc::JobGpu j{};
  j.scene = scene->dev();
  if (splat && (opt.flags & CC_NO_OBJECT_PREFILTER)) j.scene.obj_cov = nullptr;
  j.query.prefilter = opt.prefilter;
  j.query.receivers = reinterpret_cast<const float4*>(receivers);
  j.query.lights = reinterpret_cast<const float4*>(lights);
  j.query.npoints = npoints;
  j.query.nlights = nlights;
  j.query.hierarchy = opt.hierarchy;
  j.query.wide_extent = opt.wide_extent;
  j.query.light_cone_cap = opt.light_cone_cap;
  j.query.wide_cone_cap = opt.wide_cone_cap;
  j.query.order = nullptr;
  j.full = reinterpret_cast<uint2*>(out->full);
  j.any = reinterpret_cast<uint2*>(out->any);
  j.partial = out->partial;
  j.irradiance = out->irradiance;
  j.fraction = out->fraction;
  j.work = reinterpret_cast<uint4*>(out->work);
  if (!scene->flat.nodes.empty()) {
    for (int k = 0; k < 3; ++k) {
      j.lo[k] = scene->flat.nodes[0].lo[k];
      j.hi[k] = scene->flat.nodes[0].hi[k];
    }
  }
  if (job) *job = (uint32_t)(b->jobs.size() + b->splat_jobs.size());
  b->count_work = b->count_work || out->work != nullptr;
  b->prepared = false;
  if (splat) {
    b->splat_jobs.push_back(j);
    b->splat_instanced = b->splat_instanced || scene->xforms != nullptr;
    b->splat_points += npoints;
    b->splat_cones += cones;
    drop_graph(b);
    return CC_OK;
  }
  if (stale) b->updates.push_back({(uint32_t)b->jobs.size(), stale});
  b->jobs.push_back(j);
  b->instanced = b->instanced || scene->xforms != nullptr;
  b->points += npoints;
  b->cones += cones;
  drop_graph(b);
  return CC_OK;
}

}  // namespace

int cc_batch_add(cc_batch* b, const cc_scene* scene, const float* receivers, uint64_t npoints, const float* lights,
                 uint32_t nlights, const cc_options* opt_in, const cc_outputs* out, uint32_t* job) {
  return add_job(b, scene, receivers, npoints, lights, nlights, nullptr, opt_in, out, job);
}

int cc_batch_add_update(cc_batch* b, const cc_scene* scene, const float* receivers, uint64_t npoints,
                        const float* lights, uint32_t nlights, const uint8_t* stale, const cc_options* opt_in,
                        const cc_outputs* out, uint32_t* job) {
  if (!stale) return fail(CC_ERR_INVALID, "null stale flags");
  return add_job(b, scene, receivers, npoints, lights, nlights, stale, opt_in, out, job);
}

int cc_batch_submit(cc_batch* b, const cc_batch_options* opt_in, void* stream_in) {
  if (!b) return fail(CC_ERR_INVALID, "null argument");
  cc_batch_options opt;
  if (opt_in) opt = *opt_in; else cc_batch_options_default(&opt);
  int rc = check_options(opt);
  if (rc) return rc;
  rc = set_device(b->ctx);
  if (rc) return rc;
  cudaStream_t stream = stream_in ? (cudaStream_t)stream_in : b->ctx->stream;
  // The status words and the job table are reused: the previous submission
  // must be done before they change.
  if (b->submitted) CC_CUDA(cudaEventSynchronize(b->done), "batch");
  return submit(b, opt, stream);
}

int cc_batch_wait(cc_batch* b, uint32_t timeout_ms) {
  if (!b) return fail(CC_ERR_INVALID, "null argument");
  int rc = set_device(b->ctx);
  if (rc) return rc;
  return wait_done(b, timeout_ms);
}

int cc_batch_tune(cc_batch* b, const cc_batch_options* base, uint32_t reps, cc_batch_options* best, float* ms_out,
                  uint32_t max_candidates) {
  if (!b || !best) return -fail(CC_ERR_INVALID, "null argument");
  if (reps < 1) reps = 1;
  int rc = set_device(b->ctx);
  if (rc) return -rc;
  const uint32_t keep = base ? (base->flags & (CC_BATCH_GRAPH | CC_NO_REDO)) : CC_BATCH_GRAPH;
  std::vector<cc_batch_options> cands;
  for (uint32_t pw : {8u, 16u, 32u})
    for (uint32_t order : {0u, (uint32_t)CC_KEEP_ORDER})
      for (uint32_t bps : {4u, 8u}) cands.push_back({pw, bps, (keep & CC_NO_REDO) | order});
  cudaStream_t stream = b->ctx->stream;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  CC_CUDA(cudaEventCreate(&t0), "tune event");
  cudaError_t e = cudaEventCreate(&t1);
  if (e != cudaSuccess) {
    cudaEventDestroy(t0);
    return -cuda_fail(e, "tune event");
  }
  if (b->submitted) cudaEventSynchronize(b->done);
  float best_ms = 0.0f;
  int best_i = -1;
  for (size_t i = 0; i < cands.size() && rc == CC_OK; ++i) {
    // The first run of a candidate may also size buffers and upload the job
    // table; the best of `reps` runs is kept.
    float cand_ms = 0.0f;
    for (uint32_t r = 0; r < reps && rc == CC_OK; ++r) {
      rc = prepare(b, cands[i].points_per_warp);
      if (rc) break;
      cudaEventRecord(t0, stream);
      rc = submit(b, cands[i], stream);
      cudaEventRecord(t1, stream);
      if (rc == CC_OK) rc = wait_done(b, 600000);
      float ms = 0.0f;
      if (rc == CC_OK && cudaEventElapsedTime(&ms, t0, t1) == cudaSuccess && (r == 0 || ms < cand_ms)) cand_ms = ms;
    }
    if (rc != CC_OK) break;
    if (ms_out && i < max_candidates) ms_out[i] = cand_ms;
    if (best_i < 0 || cand_ms < best_ms) {
      best_ms = cand_ms;
      best_i = (int)i;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (rc != CC_OK) return -rc;
  *best = cands[best_i];
  best->flags |= keep & CC_BATCH_GRAPH;
  return (int)cands.size();
}

int cc_batch_sizes(const cc_batch* b, uint64_t out4[4]) {
  if (!b || !out4) return fail(CC_ERR_INVALID, "null argument");
  out4[0] = b->jobs.size() + b->splat_jobs.size();
  out4[1] = b->points + b->splat_points;
  out4[2] = b->cones + b->splat_cones;
  out4[3] = b->job_table.size + b->redo.size + b->order.size + b->sort_scratch.size + b->counters.size +
            b->records.size + b->masks.size + b->splat_table.size + b->splat_redo.size + b->splat_order.size +
            b->splat_sort_scratch.size;
  return CC_OK;
}
