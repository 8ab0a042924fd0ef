// The lighting cache's bake: the page manager (cache_plan.cpp) plans each
// frame's pages; their listed texels with a surface become the receivers of
// one visibility launch over every light, and a scatter kernel writes the
// results into the pool with vc_bake's semantics (mask_cones.wgsl:3433-3554):
// the visible fraction of the unshadowed light (`light_ratio`, :3505-3510,
// 1 for an empty cone, 0 for a full one, the kernel's `fraction`) or the
// shadowed light (:3527-3531), 0 for a texel without a surface, nothing for
// one outside its chart's grid. A light below a texel's horizon gives the
// share seen past the texel's own triangle (`back`, :3476-3494;
// CC_BACK_FACING) and no light.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <vector>

#include "cache_plan.h"
#include "capi_internal.h"

using cc_host::fail;
using cc_host::cuda_fail;

namespace {

constexpr uint32_t kNoSurface = 0xffffffffu;

// One listed texel: its pool row and its receiver (kNoSurface: none).
struct TexelOut {
  uint32_t pool_row;
  uint32_t receiver;
};

// pool[row * L + l] for every listed texel and light: the receiver's result,
// or 0 for a texel without a surface.
__global__ void scatter_pool(const TexelOut* __restrict__ texels, uint32_t n, uint32_t nlights, uint32_t npoints,
                             const float* __restrict__ value, float* __restrict__ pool) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)n * nlights) return;
  const uint32_t t = (uint32_t)(i % n), l = (uint32_t)(i / n);
  const TexelOut e = texels[t];
  const float v = e.receiver == kNoSurface ? 0.0f : value[(uint64_t)l * npoints + e.receiver];
  pool[(uint64_t)e.pool_row * nlights + l] = v;
}

cc_bake::Options plan_options(const cc_cache_options& o, uint32_t nlights) {
  cc_bake::Options p;
  p.pages = o.pages;
  p.lights = nlights;
  p.bake_budget = o.bake_budget;
  p.frame_target_ms = o.frame_target_ms;
  p.frame_budget_ms = o.frame_budget_ms;
  p.floor_overrun = o.floor_overrun;
  return p;
}

int check_options(const cc_cache_options* opt, uint32_t nlights) {
  if (!opt) return fail(CC_ERR_INVALID, "null options");
  if (opt->pages == 0 || opt->pages > (1u << 26)) return fail(CC_ERR_INVALID, "pages must be 1..2^26");
  if (opt->bake_budget == 0) return fail(CC_ERR_INVALID, "bake_budget must be positive");
  if (nlights == 0 || nlights > (1u << 20)) return fail(CC_ERR_INVALID, "nlights must be 1..2^20");
  if (!(opt->frame_target_ms >= 0.0f) || !(opt->frame_budget_ms >= 0.0f) || !(opt->floor_overrun >= 0.0f))
    return fail(CC_ERR_INVALID, "frame_target_ms, frame_budget_ms and floor_overrun must be >= 0");
  return CC_OK;
}

std::vector<cc_bake::Request> requests_of(const cc_page_request* r, uint32_t n) {
  std::vector<cc_bake::Request> out(n);
  for (uint32_t i = 0; i < n; ++i) {
    out[i].key = cc_bake::Key{{r[i].key[0], r[i].key[1], r[i].key[2]}};
    out[i].priority = r[i].priority;
    out[i].inside[0] = r[i].inside[0];
    out[i].inside[1] = r[i].inside[1];
  }
  return out;
}

cc_bake::Timing timing_of(const cc_cache_frame_info* info) {
  cc_bake::Timing t;
  if (info) {
    t.has_period = info->period_ms > 0.0f;
    t.period_ms = info->period_ms;
    t.gpu_waited = info->gpu_waited != 0;
    t.render_ms = info->render_ms;
  }
  return t;
}

void fill_stats(const cc_bake::Planner& p, float last_bake_ms, cc_cache_stats* s) {
  if (!s) return;
  s->budget = p.budget();
  s->frame = p.frame();
  s->pages_planned = (uint32_t)p.planned().size();
  s->jobs = (uint32_t)(p.jobs().size() / 2);
  s->spent = p.spent();
  s->resident = p.resident();
  s->evicted = p.evicted();
  s->last_bake_ms = last_bake_ms;
}

int64_t copy_jobs(const cc_bake::Planner& p, uint32_t* jobs2, uint64_t max_jobs, uint32_t* page_slots,
                  uint32_t max_pages) {
  const std::vector<uint32_t>& j = p.jobs();
  const uint64_t n = j.size() / 2;
  if (jobs2) std::memcpy(jobs2, j.data(), std::min<uint64_t>(n, max_jobs) * 2 * sizeof(uint32_t));
  if (page_slots)
    for (uint32_t i = 0; i < std::min<uint32_t>(max_pages, (uint32_t)p.planned().size()); ++i)
      page_slots[i] = p.planned()[i].slot;
  return (int64_t)n;
}

// Grows a buffer to at least `bytes`, at least doubling it: frame sizes vary
// a little, and each reallocation would stall the device.
cudaError_t grow(cc_host::DevBuf& b, size_t bytes) {
  if (bytes <= b.size) return cudaSuccess;
  return b.reserve(std::max(bytes, 2 * b.size));
}

// The most texels one frame can list: a page costs its inside texels times
// the lights and lists at most 4 texels per inside texel (inside 1 x 1 lists
// 2 x 2); the first page always fits.
uint64_t listed_bound(uint32_t bake_budget, uint32_t nlights) {
  return 4ull * bake_budget / nlights + bake_budget % nlights + cc_bake::kPageTexels;
}

}  // namespace

struct cc_planner {
  std::unique_ptr<cc_bake::Planner> plan;
};

struct cc_cache {
  cc_context* ctx = nullptr;
  const cc_scene* scene = nullptr;
  cc_cache_options opt{};
  uint32_t nlights = 0;
  std::unique_ptr<cc_bake::Planner> plan;
  float* pool = nullptr;   // pages * 81 * nlights
  float4* lights = nullptr;
  cc_host::DevBuf receivers, texels, value;
  float* host_receivers = nullptr;  // pinned staging
  size_t host_receivers_cap = 0;
  TexelOut* host_texels = nullptr;
  size_t host_texels_cap = 0;
  cudaEvent_t start = nullptr, end = nullptr;
  bool pending = false;    // a bake's events are recorded and not yet read
  float pending_units = 0;
  float last_bake_ms = -1.0f;
};

// Sizes the staging and device buffers of a frame listing `listed` texels
// (their growth, inside a frame, would stall the device and the host).
static int size_buffers(cc_cache* c, uint64_t listed) {
  if (c->host_texels_cap < listed) {
    const size_t cap = std::max<size_t>(listed, 2 * c->host_texels_cap);
    if (c->host_texels) cudaFreeHost(c->host_texels);
    c->host_texels = nullptr;
    c->host_texels_cap = 0;
    CC_CUDA(cudaMallocHost(&c->host_texels, cap * sizeof(TexelOut)), "texel staging");
    c->host_texels_cap = cap;
  }
  if (c->host_receivers_cap < listed) {
    const size_t cap = std::max<size_t>(listed, 2 * c->host_receivers_cap);
    if (c->host_receivers) cudaFreeHost(c->host_receivers);
    c->host_receivers = nullptr;
    c->host_receivers_cap = 0;
    CC_CUDA(cudaMallocHost(&c->host_receivers, cap * 32), "receiver staging");
    c->host_receivers_cap = cap;
  }
  const uint64_t ncones = listed * c->nlights;
  CC_CUDA(grow(c->texels, (size_t)listed * sizeof(TexelOut)), "texel list");
  CC_CUDA(grow(c->value, std::max<size_t>((size_t)ncones * sizeof(float), 4)), "bake values");
  CC_CUDA(grow(c->receivers, (size_t)listed * 32), "bake receivers");
  CC_CUDA(grow(c->ctx->redo, std::max<uint64_t>(ncones, 1) * 4), "redo list");
  CC_CUDA(grow(c->ctx->order, (size_t)listed * sizeof(uint32_t)), "walk order");
  CC_CUDA(grow(c->ctx->sort_scratch, cc::walk_order_scratch_bytes(listed)), "walk order scratch");
  return CC_OK;
}

extern "C" {

void cc_cache_options_default(cc_cache_options* opt) {
  if (!opt) return;
  opt->pages = 1u << 16;
  opt->bake_budget = 1u << 20;
  opt->frame_target_ms = 0.0f;
  opt->frame_budget_ms = 0.0f;
  opt->floor_overrun = 0.25f;
  opt->light_ratio = 1;
}

int cc_planner_create(const cc_cache_options* opt, uint32_t nlights, cc_planner** out) {
  if (!out) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  int rc = check_options(opt, nlights);
  if (rc) return rc;
  auto* p = new cc_planner;
  p->plan.reset(new cc_bake::Planner(plan_options(*opt, nlights)));
  *out = p;
  return CC_OK;
}

int cc_planner_destroy(cc_planner* p) {
  delete p;
  return CC_OK;
}

int cc_planner_frame(cc_planner* p, const cc_page_request* requests, uint32_t nrequests,
                     const cc_cache_frame_info* info, float bake_ms, cc_cache_stats* stats) {
  if (!p || (nrequests && !requests)) return fail(CC_ERR_INVALID, "null argument");
  const float units = (float)p->plan->spent();
  p->plan->begin_frame(timing_of(info), bake_ms, units);
  p->plan->plan(requests_of(requests, nrequests));
  fill_stats(*p->plan, bake_ms, stats);
  p->plan->end_frame();
  return CC_OK;
}

int64_t cc_planner_jobs(cc_planner* p, uint32_t* jobs2, uint64_t max_jobs, uint32_t* page_slots, uint32_t max_pages) {
  if (!p) return -(int64_t)fail(CC_ERR_INVALID, "null planner");
  return copy_jobs(*p->plan, jobs2, max_jobs, page_slots, max_pages);
}

int64_t cc_planner_slot(cc_planner* p, const uint32_t key[3]) {
  if (!p || !key) return -1;
  const uint32_t s = p->plan->slot_of(cc_bake::Key{{key[0], key[1], key[2]}});
  return s == cc_bake::kEmpty ? -1 : (int64_t)s;
}

int cc_cache_create(cc_context* ctx, const cc_scene* scene, const float* lights, uint32_t nlights,
                    const cc_cache_options* opt_in, cc_cache** out) {
  if (!out) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  if (!ctx || !scene || !lights) return fail(CC_ERR_INVALID, "null argument");
  if (scene->ctx != ctx) return fail(CC_ERR_INVALID, "scene belongs to another context (or to none)");
  cc_cache_options opt;
  if (opt_in) opt = *opt_in; else cc_cache_options_default(&opt);
  int rc = check_options(&opt, nlights);
  if (rc) return rc;
  rc = cc_host::set_device(ctx);
  if (rc) return rc;
  std::unique_ptr<cc_cache> c(new cc_cache);
  c->ctx = ctx;
  c->scene = scene;
  c->opt = opt;
  c->nlights = nlights;
  c->plan.reset(new cc_bake::Planner(plan_options(opt, nlights)));
  const size_t pool_bytes = (size_t)opt.pages * cc_bake::kPageTexels * nlights * sizeof(float);
  cudaError_t e = cudaMalloc(&c->pool, pool_bytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->pool, 0, pool_bytes, ctx->stream);
  if (e == cudaSuccess) e = cudaMalloc(&c->lights, (size_t)nlights * 64);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->lights, lights, (size_t)nlights * 64, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaEventCreate(&c->start);
  if (e == cudaSuccess) e = cudaEventCreate(&c->end);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cc_cache_destroy(c.release());
    return cuda_fail(e, "cache pool and lights");
  }
  // Buffers for a full frame up front (at most 16M texels; beyond, a frame
  // that needs more grows them).
  rc = size_buffers(c.get(), std::min<uint64_t>(listed_bound(opt.bake_budget, nlights), 1ull << 24));
  if (rc) {
    cc_cache_destroy(c.release());
    return rc;
  }
  *out = c.release();
  return CC_OK;
}

int cc_cache_destroy(cc_cache* c) {
  if (!c) return CC_OK;
  cc_host::set_device(c->ctx);
  cudaStreamSynchronize(c->ctx->stream);
  if (c->pool) cudaFree(c->pool);
  if (c->lights) cudaFree(c->lights);
  c->receivers.release();
  c->texels.release();
  c->value.release();
  if (c->host_receivers) cudaFreeHost(c->host_receivers);
  if (c->host_texels) cudaFreeHost(c->host_texels);
  if (c->start) cudaEventDestroy(c->start);
  if (c->end) cudaEventDestroy(c->end);
  delete c;
  return CC_OK;
}

int cc_cache_frame(cc_cache* c, const cc_page_request* requests, uint32_t nrequests, const cc_cache_frame_info* info,
                   cc_cache_stats* stats) {
  if (!c || (nrequests && !requests)) return fail(CC_ERR_INVALID, "null argument");
  int rc = cc_host::set_device(c->ctx);
  if (rc) return rc;
  cudaStream_t stream = c->ctx->stream;
  // The previous bake: its GPU time feeds the budget, and its staging
  // buffers are free again once it is done.
  float bake_ms = -1.0f, units = 0.0f;
  if (c->pending) {
    CC_CUDA(cudaEventSynchronize(c->end), "previous bake");
    CC_CUDA(cudaEventElapsedTime(&bake_ms, c->start, c->end), "bake time");
    units = c->pending_units;
    c->pending = false;
    c->last_bake_ms = bake_ms;
  }
  cc_bake::Planner& p = *c->plan;
  p.begin_frame(timing_of(info), bake_ms, units);
  p.plan(requests_of(requests, nrequests));
  const std::vector<cc_bake::Planned>& planned = p.planned();
  // The planned pages' listed texels: receivers for those with a surface.
  uint64_t listed = 0;
  for (const auto& pl : planned) listed += (uint64_t)pl.listed[0] * pl.listed[1];
  if (listed) {
    for (const auto& pl : planned)
      if (!requests[pl.request].texels) {
        p.end_frame();
        return fail(CC_ERR_INVALID, "a planned page's request has no texels");
      }
    rc = size_buffers(c, listed);
    if (rc) {
      p.end_frame();
      return rc;
    }
    uint32_t ntexels = 0, npoints = 0;
    for (const auto& pl : planned) {
      const float* tx = requests[pl.request].texels;
      for (uint32_t y = 0; y < pl.listed[1]; ++y)
        for (uint32_t x = 0; x < pl.listed[0]; ++x) {
          const uint32_t k = y * cc_bake::kStride + x;
          const float* r = tx + 8 * k;
          const float flag = r[3];
          if (!(flag >= 0.5f)) continue;  // outside the chart's grid: not written
          TexelOut& e = c->host_texels[ntexels++];
          e.pool_row = pl.slot * cc_bake::kPageTexels + k;
          e.receiver = kNoSurface;
          if (flag >= 1.5f) {
            float* d = c->host_receivers + 8 * (size_t)npoints;
            d[0] = r[0], d[1] = r[1], d[2] = r[2], d[3] = 0.0f;
            d[4] = r[4], d[5] = r[5], d[6] = r[6], d[7] = r[7];  // the texel's own triangle + 1 (bits)
            e.receiver = npoints++;
          }
        }
    }
    CC_CUDA(cudaEventRecord(c->start, stream), "bake timing");
    if (ntexels) {
      CC_CUDA(cudaMemcpyAsync(c->texels.ptr, c->host_texels, (size_t)ntexels * sizeof(TexelOut),
                              cudaMemcpyHostToDevice, stream),
              "texel list upload");
      if (npoints) {
        CC_CUDA(cudaMemcpyAsync(c->receivers.ptr, c->host_receivers, (size_t)npoints * 32, cudaMemcpyHostToDevice,
                                stream),
                "bake receivers upload");
        cc_options vo;
        cc_options_default(&vo);
        vo.flags = CC_DEVICE_POINTERS;
        // A light below a texel's horizon: the share seen past the texel's
        // own triangle (vc_bake's `back`, :3476-3494), for texels that name
        // it, in scenes without instancing.
        if (c->scene->flat.xforms.empty()) vo.flags |= CC_BACK_FACING;
        cc_outputs out{};
        float* v = static_cast<float*>(c->value.ptr);
        if (c->opt.light_ratio) out.fraction = v; else out.irradiance = v;
        rc = cc_visibility(c->ctx, c->scene, static_cast<const float*>(c->receivers.ptr), npoints,
                           reinterpret_cast<const float*>(c->lights), c->nlights, &vo, &out, stream);
        if (rc) {
          p.end_frame();
          return rc;
        }
      }
      const uint64_t threads = (uint64_t)ntexels * c->nlights;
      scatter_pool<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(
          static_cast<const TexelOut*>(c->texels.ptr), ntexels, c->nlights, npoints,
          static_cast<const float*>(c->value.ptr), c->pool);
      CC_CUDA(cudaGetLastError(), "pool scatter");
    }
    CC_CUDA(cudaEventRecord(c->end, stream), "bake timing");
    c->pending = true;
    c->pending_units = (float)p.spent();
  }
  fill_stats(p, c->last_bake_ms, stats);
  p.end_frame();
  return CC_OK;
}

int cc_cache_read(cc_cache* c, const uint32_t key[3], float* out) {
  if (!c || !key || !out) return fail(CC_ERR_INVALID, "null argument");
  const uint32_t slot = c->plan->slot_of(cc_bake::Key{{key[0], key[1], key[2]}});
  if (slot == cc_bake::kEmpty) return fail(CC_ERR_INVALID, "the page is not resident");
  int rc = cc_host::set_device(c->ctx);
  if (rc) return rc;
  const size_t n = (size_t)cc_bake::kPageTexels * c->nlights;
  CC_CUDA(cudaMemcpyAsync(out, c->pool + (size_t)slot * n, n * sizeof(float), cudaMemcpyDeviceToHost, c->ctx->stream),
          "pool read");
  CC_CUDA(cudaStreamSynchronize(c->ctx->stream), "pool read");
  return CC_OK;
}

int cc_cache_pool(cc_cache* c, float** pool, uint32_t* channels) {
  if (!c) return fail(CC_ERR_INVALID, "null cache");
  if (pool) *pool = c->pool;
  if (channels) *channels = c->nlights;
  return CC_OK;
}

int64_t cc_cache_jobs(cc_cache* c, uint32_t* jobs2, uint64_t max_jobs, uint32_t* page_slots, uint32_t max_pages) {
  if (!c) return -(int64_t)fail(CC_ERR_INVALID, "null cache");
  return copy_jobs(*c->plan, jobs2, max_jobs, page_slots, max_pages);
}

}  // extern "C"
