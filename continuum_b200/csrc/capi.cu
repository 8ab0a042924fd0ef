// The C ABI (include/continuum_cuda.h): contexts, resident scenes, and the
// visibility calls. Host code; the kernels are in visibility.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "capi_internal.h"

namespace cc_host {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  g_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? CC_ERR_OOM : CC_ERR_CUDA;
}

int set_device(cc_context* ctx) {
  CC_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  return CC_OK;
}

}  // namespace cc_host

using namespace cc_host;

namespace {

// The fraction of each bin of a sphere light's window inside the inscribed
// disk (the reference's DISK table, mask_cones.wgsl:888-897): for the
// circle of radius 4 bins centred on the 8x8 grid, each cell's area inside
// it, integrated column by column with the exact chord, rounded to the six
// decimals the reference's table carries.
void disk_table(float* out) {
  const int kSteps = 20000;
  for (int b = 0; b < 64; ++b) {
    const int col = b % 8, row = b / 8;
    double area = 0.0;
    for (int i = 0; i < kSteps; ++i) {
      const double x = col + (i + 0.5) / kSteps - 4.0;
      const double h2 = 16.0 - x * x;
      if (h2 <= 0.0) continue;
      const double h = std::sqrt(h2);
      const double lo = std::max(row - 4.0, -h), hi = std::min(row + 1.0 - 4.0, h);
      if (hi > lo) area += (hi - lo) / kSteps;
    }
    out[b] = (float)(std::round(area * 1e6) / 1e6);
  }
}

// Repacks NodeGpu (48 bytes) into two float4 (lo.xyz | a, hi.xyz | b).
std::vector<float4> repack(const std::vector<cc::NodeGpu>& nodes) {
  std::vector<float4> out(2 * nodes.size());
  for (size_t i = 0; i < nodes.size(); ++i) {
    const cc::NodeGpu& n = nodes[i];
    uint32_t a = n.info[0], b = n.info[1];
    float fa, fb;
    std::memcpy(&fa, &a, 4);
    std::memcpy(&fb, &b, 4);
    out[2 * i] = make_float4(n.lo[0], n.lo[1], n.lo[2], fa);
    out[2 * i + 1] = make_float4(n.hi[0], n.hi[1], n.hi[2], fb);
  }
  return out;
}

template <class T>
int upload(const std::vector<T>& host, T** dev, uint64_t& bytes, const char* what) {
  size_t n = std::max<size_t>(host.size(), 1) * sizeof(T);
  CC_CUDA(cudaMalloc(dev, n), what);
  if (!host.empty()) CC_CUDA(cudaMemcpy(*dev, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), what);
  bytes += n;
  return CC_OK;
}

void free_scene_device(cc_scene* s) {
  cudaFree(s->tris);
  cudaFree(s->meshes);
  cudaFree(s->nodes);
  cudaFree(s->items);
  cudaFree(s->blas);
  cudaFree(s->xforms);
  cudaFree(s->blas_cov);
  cudaFree(s->obj_cov);
  cudaFree(s->tri_slot);
  s->tri_slot = nullptr;
  s->blas_cov = nullptr;
  s->obj_cov = nullptr;
  s->coverage_ready = false;
  s->xforms = nullptr;
  s->tris = nullptr;
  s->meshes = nullptr;
  s->nodes = nullptr;
  s->items = nullptr;
  s->blas = nullptr;
}

int upload_scene(cc_scene* s) {
  const cc::FlatScene& f = s->flat;
  // Triangles in leaf order: slot k holds triangle blas_items[k], so a
  // triangle-hierarchy leaf's items are slots. Each mesh's items permute its
  // own range, so a mesh's range of slots still holds exactly its triangles.
  const size_t ntris = f.tris.size() / 12;
  std::vector<float4> tris(3 * ntris);
  for (size_t k = 0; k < ntris; ++k) {
    const size_t t = (!f.blas.empty() && k < f.blas_items.size()) ? f.blas_items[k] : k;
    for (int v = 0; v < 3; ++v) {
      const float* p = &f.tris[12 * t + 4 * v];
      tris[3 * k + v] = make_float4(p[0], p[1], p[2], p[3]);
    }
  }
  std::vector<uint4> meshes(f.nmeshes);
  for (uint32_t m = 0; m < f.nmeshes; ++m)
    meshes[m] = make_uint4(f.ranges[4 * m], f.ranges[4 * m + 1], f.ranges[4 * m + 2], f.ranges[4 * m + 3]);
  // Without meshes the object hierarchy is one leaf holding mesh 0, which
  // must then be an empty range (as flatten pads it, hierarchy.rs:57-59).
  if (meshes.empty()) meshes.push_back(make_uint4(0u, 0u, CC_NONE, CC_NONE));
  int rc;
  if ((rc = upload(tris, &s->tris, s->bytes, "scene triangles"))) return rc;
  if ((rc = upload(meshes, &s->meshes, s->bytes, "scene meshes"))) return rc;
  if ((rc = upload(repack(f.nodes), &s->nodes, s->bytes, "scene nodes"))) return rc;
  if ((rc = upload(f.items, &s->items, s->bytes, "scene items"))) return rc;
  if ((rc = upload(repack(f.blas), &s->blas, s->bytes, "scene triangle nodes"))) return rc;
  if (!f.xforms.empty()) {
    std::vector<float4> x(f.xforms.size() / 4);
    for (size_t i = 0; i < x.size(); ++i)
      x[i] = make_float4(f.xforms[4 * i], f.xforms[4 * i + 1], f.xforms[4 * i + 2], f.xforms[4 * i + 3]);
    if ((rc = upload(x, &s->xforms, s->bytes, "scene transforms"))) return rc;
  }
  return CC_OK;
}

// The prefiltered cones' coverage samples of every triangle-hierarchy node
// and, for instanced scenes, every object-hierarchy node (built on the host
// from the scene's own arrays as the reference builds them, then uploaded).
int ensure_coverage(cc_scene* s) {
  if (s->coverage_ready) return CC_OK;
  const std::vector<float> blas = cc::blas_coverage(s->flat);
  int rc;
  if (!blas.empty() && (rc = upload(blas, &s->blas_cov, s->bytes, "triangle-node coverage"))) return rc;
  if (!s->flat.xforms.empty()) {
    const std::vector<float> obj = cc::object_coverage(s->flat, blas);
    if (!obj.empty() && (rc = upload(obj, &s->obj_cov, s->bytes, "object-node coverage"))) return rc;
  }
  s->coverage_ready = true;
  return CC_OK;
}

// Each triangle's slot on the device (the inverse of the leaf order in which
// upload_scene stores the triangles), for CC_BACK_FACING's own triangles.
int ensure_slots(cc_scene* s) {
  if (s->tri_slot) return CC_OK;
  const cc::FlatScene& f = s->flat;
  const size_t ntris = f.tris.size() / 12;
  std::vector<uint32_t> slot(std::max<size_t>(ntris, 1), 0u);
  for (size_t k = 0; k < ntris; ++k) {
    const size_t t = (!f.blas.empty() && k < f.blas_items.size()) ? f.blas_items[k] : k;
    slot[t] = (uint32_t)k;
  }
  return upload(slot, &s->tri_slot, s->bytes, "triangle slots");
}

int validate_flat(const cc::FlatScene& f) {
  const uint64_t ntris = f.tris.size() / 12;
  for (uint32_t m = 0; m < f.nmeshes; ++m) {
    const uint32_t* r = &f.ranges[4 * m];
    if ((uint64_t)r[0] + r[1] > ntris) return fail(CC_ERR_INVALID, "mesh range beyond the triangles");
    if (r[2] != CC_NONE && r[2] >= f.blas.size()) return fail(CC_ERR_INVALID, "mesh hierarchy root out of range");
    if (r[3] != CC_NONE) {
      if ((uint64_t)r[3] * 16 + 16 > f.xforms.size()) return fail(CC_ERR_INVALID, "object transform out of range");
      const float* x = &f.xforms[16 * (size_t)r[3]];
      if (!(x[12] > 0.0f) || !std::isfinite(x[12]) || !std::isfinite(x[13]))
        return fail(CC_ERR_INVALID, "object transforms need a positive finite scale");
    }
  }
  auto check_nodes = [&](const std::vector<cc::NodeGpu>& nodes, uint64_t nitems, const char* what) {
    for (size_t i = 0; i < nodes.size(); ++i) {
      const cc::NodeGpu& n = nodes[i];
      if (n.info[1] > 0) {
        if ((uint64_t)n.info[0] + n.info[1] > nitems) return fail(CC_ERR_INVALID, std::string(what) + ": leaf beyond its items");
      } else if ((uint64_t)n.info[0] + 1 >= nodes.size() || n.info[0] <= i) {
        return fail(CC_ERR_INVALID, std::string(what) + ": child index out of range");
      }
    }
    return CC_OK;
  };
  int rc;
  if ((rc = check_nodes(f.blas, f.blas_items.size(), "triangle hierarchy"))) return rc;
  if ((rc = check_nodes(f.nodes, f.items.size(), "object hierarchy"))) return rc;
  for (uint32_t t : f.blas_items)
    if (t >= ntris) return fail(CC_ERR_INVALID, "triangle hierarchy item out of range");
  // Each mesh's leaf items must permute its own triangle range (as flatten
  // lays them out, hierarchy.rs:38-45); the device stores triangles in that
  // order.
  if (!f.blas.empty()) {
    if (f.blas_items.size() != ntris) return fail(CC_ERR_INVALID, "triangle hierarchy items must cover every triangle");
    std::vector<uint8_t> seen(ntris, 0);
    std::vector<uint8_t> checked(ntris + 1, 0);  // objects placing one geometry share its range
    for (uint32_t m = 0; m < f.nmeshes; ++m) {
      const uint32_t first = f.ranges[4 * m], count = f.ranges[4 * m + 1];
      if (count == 0 || checked[first]) continue;
      checked[first] = 1;
      for (uint64_t k = first; k < (uint64_t)first + count; ++k) {
        const uint32_t t = f.blas_items[k];
        if (t < first || t >= (uint64_t)first + count || seen[t])
          return fail(CC_ERR_INVALID, "a mesh's triangle hierarchy items must permute its triangle range");
        seen[t] = 1;
      }
    }
  }
  for (const auto* nodes : {&f.blas, &f.nodes})
    for (const cc::NodeGpu& n : *nodes)
      if (n.info[1] > 15 || n.info[0] >= (1u << 26))
        return fail(CC_ERR_INVALID, "hierarchy leaves hold at most 15 items and indices stay below 2^26");
  for (uint32_t m : f.items)
    if (m >= std::max<uint32_t>(f.nmeshes, 1)) return fail(CC_ERR_INVALID, "object hierarchy item out of range");
  if (f.nodes.empty()) return fail(CC_ERR_INVALID, "empty object hierarchy");
  return CC_OK;
}

int threads_for_build() {
  unsigned n = std::thread::hardware_concurrency();
  return n ? (int)std::min(n, 32u) : 4;
}

}  // namespace

int cc_host::scene_coverage(cc_scene* s) { return ensure_coverage(s); }

extern "C" {

const char* cc_last_error(void) { return g_error.c_str(); }

void cc_options_default(cc_options* opt) {
  if (!opt) return;
  opt->hierarchy = 2;
  opt->wide_extent = 8.0f;
  opt->light_cone_cap = 4096;
  opt->wide_cone_cap = 512;
  opt->points_per_warp = 32;
  opt->flags = 0;
  opt->prefilter = 0.0f;
}

int cc_context_create(int device, cc_context** out) {
  if (!out) return fail(CC_ERR_INVALID, "null output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(CC_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= n) return fail(CC_ERR_INVALID, "device index out of range");
  cc_context* ctx = new cc_context;
  ctx->device = device;
  int rc = set_device(ctx);
  if (rc) {
    delete ctx;
    return rc;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) ctx->sm_count = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->walked, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->copied, cudaEventDisableTiming);
  float disk[64];
  disk_table(disk);
  if (e == cudaSuccess) e = cc::upload_disk_table(disk);
  if (e == cudaSuccess) e = ctx->counters.reserve(cc::kCounterWords * sizeof(uint32_t));
  ctx->marks.assign(3 * cc_context::kTimingRing, nullptr);
  for (auto& ev : ctx->marks)
    if (e == cudaSuccess) e = cudaEventCreate(&ev);
  if (e != cudaSuccess) {
    int code = cuda_fail(e, "context setup");
    cc_context_destroy(ctx);
    return code;
  }
  *out = ctx;
  return CC_OK;
}

int cc_context_set_split_chunk(cc_context* ctx, uint64_t cones) {
  if (!ctx) return fail(CC_ERR_INVALID, "null context");
  if (cones < 32 || cones > (1ull << 31)) return fail(CC_ERR_INVALID, "split chunk must hold 32 .. 2^31 cones");
  ctx->split_chunk = cones;
  return CC_OK;
}

int cc_context_destroy(cc_context* ctx) {
  if (!ctx) return CC_OK;
  cudaSetDevice(ctx->device);
  for (DevBuf* b : {&ctx->receivers, &ctx->lights, &ctx->full, &ctx->any, &ctx->partial, &ctx->irradiance,
                    &ctx->fraction, &ctx->work, &ctx->redo, &ctx->order, &ctx->sort_scratch, &ctx->records, &ctx->masks,
                    &ctx->counters, &ctx->move_xforms, &ctx->stale_tables, &ctx->upd_perm, &ctx->upd_flags,
                    &ctx->upd_list, &ctx->upd_count, &ctx->upd_order, &ctx->upd_temp})
    b->release();
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->walked) cudaEventDestroy(ctx->walked);
  if (ctx->copied) cudaEventDestroy(ctx->copied);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  for (auto ev : ctx->marks)
    if (ev) cudaEventDestroy(ev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return CC_OK;
}

int cc_scene_upload(cc_context* ctx, const cc_flat_scene* fl, cc_scene** out) {
  if (!ctx || !fl || !out) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  if (fl->ntris && !fl->tris) return fail(CC_ERR_INVALID, "null triangles");
  if (!fl->ranges || !fl->nodes || !fl->items || fl->nnodes == 0)
    return fail(CC_ERR_INVALID, "a flat scene needs ranges, nodes and items");
  cc_scene* s = new cc_scene;
  s->ctx = ctx;
  cc::FlatScene& f = s->flat;
  f.nmeshes = fl->nmeshes;
  f.tris.assign(fl->tris, fl->tris + (size_t)fl->ntris * 12);
  f.ranges.assign(fl->ranges, fl->ranges + (size_t)fl->nmeshes * 4);
  const cc::NodeGpu* b = static_cast<const cc::NodeGpu*>(fl->blas);
  if (fl->nblas && !b) {
    delete s;
    return fail(CC_ERR_INVALID, "null triangle hierarchy");
  }
  if (b) f.blas.assign(b, b + fl->nblas);
  if (fl->blas_items) f.blas_items.assign(fl->blas_items, fl->blas_items + fl->nblas_items);
  const cc::NodeGpu* n = static_cast<const cc::NodeGpu*>(fl->nodes);
  f.nodes.assign(n, n + fl->nnodes);
  f.items.assign(fl->items, fl->items + fl->nitems);
  if (fl->nxforms) {
    if (!fl->xforms) {
      delete s;
      return fail(CC_ERR_INVALID, "null transforms");
    }
    f.xforms.assign(fl->xforms, fl->xforms + (size_t)fl->nxforms * 16);
  }
  int rc = validate_flat(f);
  if (!rc) rc = set_device(ctx);
  if (!rc) rc = upload_scene(s);
  if (rc) {
    free_scene_device(s);
    delete s;
    return rc;
  }
  *out = s;
  return CC_OK;
}

int cc_scene_build(cc_context* ctx, const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes,
                   cc_scene** out) {
  if (!out || (nmeshes && !mesh_counts)) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  uint64_t total = 0;
  for (uint32_t m = 0; m < nmeshes; ++m) total += mesh_counts[m];
  if (total && !tri9) return fail(CC_ERR_INVALID, "null triangles");
  if (total >= 0xffffffffull) return fail(CC_ERR_INVALID, "too many triangles");
  cc_scene* s = new cc_scene;
  s->ctx = ctx;
  cc::build_flat_scene(tri9, mesh_counts, nmeshes, s->flat, threads_for_build());
  if (s->flat.blas.size() >= (1u << 26) || s->flat.nodes.size() >= (1u << 26) || total >= (1u << 26)) {
    delete s;
    return fail(CC_ERR_INVALID, "a scene holds fewer than 2^26 triangles and hierarchy nodes");
  }
  if (!ctx) {  // host-only scene
    *out = s;
    return CC_OK;
  }
  int rc = set_device(ctx);
  if (!rc) rc = upload_scene(s);
  if (rc) {
    free_scene_device(s);
    delete s;
    return rc;
  }
  *out = s;
  return CC_OK;
}

int cc_scene_build_instanced(cc_context* ctx, const float* tri9, const uint32_t* geometry_counts,
                             uint32_t ngeometries, const cc_instance* instances, uint32_t ninstances,
                             const uint32_t* movable, uint32_t nmovable, cc_scene** out) {
  static_assert(sizeof(cc_instance) == sizeof(cc::Instance), "cc_instance is cc::Instance");
  if (!out || (ngeometries && !geometry_counts) || (ninstances && !instances)) return fail(CC_ERR_INVALID, "null argument");
  *out = nullptr;
  uint64_t total = 0;
  for (uint32_t g = 0; g < ngeometries; ++g) total += geometry_counts[g];
  if (total && !tri9) return fail(CC_ERR_INVALID, "null triangles");
  if (ninstances >= (1u << 26)) return fail(CC_ERR_INVALID, "fewer than 2^26 instances");
  for (uint32_t k = 0; k < ninstances; ++k) {
    const cc_instance& o = instances[k];
    if (o.geometry >= ngeometries) return fail(CC_ERR_INVALID, "instance geometry out of range");
    if (!(o.scale > 0.0f) || !std::isfinite(o.scale)) return fail(CC_ERR_INVALID, "instance scale must be positive");
    // The rotation must be orthonormal (Placement, hierarchy.rs:258-270).
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const float d = o.rotation[3 * i] * o.rotation[3 * j] + o.rotation[3 * i + 1] * o.rotation[3 * j + 1] +
                        o.rotation[3 * i + 2] * o.rotation[3 * j + 2];
        if (!(std::fabs(d - (i == j ? 1.0f : 0.0f)) < 1e-4f)) return fail(CC_ERR_INVALID, "instance rotation is not orthonormal");
      }
  }
  if (total >= (1u << 26)) return fail(CC_ERR_INVALID, "a scene holds fewer than 2^26 triangles and hierarchy nodes");
  if (nmovable) {
    if (!movable) return fail(CC_ERR_INVALID, "null movable list");
    if (nmovable >= ninstances) return fail(CC_ERR_INVALID, "a scene with movers needs a static object");
    std::vector<uint8_t> seen(ninstances, 0);
    for (uint32_t i = 0; i < nmovable; ++i) {
      if (movable[i] >= ninstances || seen[movable[i]]) return fail(CC_ERR_INVALID, "movable objects must be distinct objects");
      seen[movable[i]] = 1;
    }
  }
  cc_scene* s = new cc_scene;
  s->ctx = ctx;
  cc::build_instanced_scene(tri9, geometry_counts, ngeometries, reinterpret_cast<const cc::Instance*>(instances),
                            ninstances, movable, nmovable, s->flat, threads_for_build());
  if (s->flat.blas.size() >= (1u << 26) || s->flat.nodes.size() >= (1u << 26)) {
    delete s;
    return fail(CC_ERR_INVALID, "a scene holds fewer than 2^26 triangles and hierarchy nodes");
  }
  if (!ctx) {  // host-only scene
    *out = s;
    return CC_OK;
  }
  int rc = set_device(ctx);
  if (!rc) rc = upload_scene(s);
  if (rc) {
    free_scene_device(s);
    delete s;
    return rc;
  }
  *out = s;
  return CC_OK;
}

uint64_t cc_scene_transforms(const cc_scene* s, float* out16, uint64_t max_transforms) {
  if (!s) return 0;
  const uint64_t n = s->flat.xforms.size() / 16;
  if (out16) std::memcpy(out16, s->flat.xforms.data(), std::min(n, max_transforms) * 16 * sizeof(float));
  return n;
}

int cc_scene_destroy(cc_scene* s) {
  if (!s) return CC_OK;
  if (s->ctx) {
    cudaSetDevice(s->ctx->device);
    free_scene_device(s);
  }
  delete s;
  return CC_OK;
}

int cc_scene_sizes(const cc_scene* s, uint64_t out6[6]) {
  if (!s || !out6) return fail(CC_ERR_INVALID, "null argument");
  out6[0] = s->flat.tris.size() / 12;
  out6[1] = s->flat.nmeshes;
  out6[2] = s->flat.blas.size();
  out6[3] = s->flat.blas_items.size();
  out6[4] = s->flat.nodes.size();
  out6[5] = s->flat.items.size();
  return CC_OK;
}

int cc_scene_arrays(const cc_scene* s, uint32_t* ranges, void* blas, uint32_t* blas_items, void* nodes,
                    uint32_t* items) {
  if (!s) return fail(CC_ERR_INVALID, "null scene");
  const cc::FlatScene& f = s->flat;
  if (ranges) std::memcpy(ranges, f.ranges.data(), f.ranges.size() * 4);
  if (blas) std::memcpy(blas, f.blas.data(), f.blas.size() * sizeof(cc::NodeGpu));
  if (blas_items) std::memcpy(blas_items, f.blas_items.data(), f.blas_items.size() * 4);
  if (nodes) std::memcpy(nodes, f.nodes.data(), f.nodes.size() * sizeof(cc::NodeGpu));
  if (items) std::memcpy(items, f.items.data(), f.items.size() * 4);
  return CC_OK;
}

uint64_t cc_scene_device_bytes(const cc_scene* s) { return s ? s->bytes : 0; }

int cc_context_kernel_times(cc_context* ctx, float* out2, int max_calls) {
  if (!ctx || (max_calls > 0 && !out2)) return fail(CC_ERR_INVALID, "null argument");
  int rc = set_device(ctx);
  if (rc) return -rc;
  const int ring = cc_context::kTimingRing;
  int n = 0;
  while (ctx->timed_count > 0) {
    cudaEvent_t* m = &ctx->marks[3 * ctx->timed_first];
    cudaError_t e = cudaEventSynchronize(m[2]);
    if (e != cudaSuccess) return -cuda_fail(e, "kernel timing");
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, m[0], m[1]);
    cudaEventElapsedTime(&b, m[1], m[2]);
    if (n < max_calls) {
      out2[2 * n] = a;
      out2[2 * n + 1] = b;
      ++n;
    }
    ctx->timed_first = (ctx->timed_first + 1) % ring;
    ctx->timed_count--;
  }
  return n;
}

int cc_scene_primary_hits(const cc_scene* s, const float camera[10], uint32_t width, uint32_t height, float* out8,
                          uint8_t* hit) {
  if (!s || !camera || !out8 || !hit) return fail(CC_ERR_INVALID, "null argument");
  if (s->flat.nodes.empty()) return fail(CC_ERR_INVALID, "scene has no hierarchy");
  cc::primary_hits(s->flat, camera, width, height, out8, hit, threads_for_build());
  return CC_OK;
}

}  // extern "C"

// cc_visibility's body; `sky` (kSkyCones and its flags) makes the cones the
// receivers' six sky faces (nlights = 6, no lights); `cones` (device, with
// its count in device memory) walks only the listed cones, in that order.
int cc_host::visibility_impl(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                             const float* lights, uint32_t nlights, const cc_options* opt_in, const cc_outputs* out,
                             void* stream_in, uint32_t sky, const uint32_t* cones, const uint32_t* cones_count) {
  if (!ctx || !scene || !out) return fail(CC_ERR_INVALID, "null argument");
  if (scene->ctx != ctx) return fail(CC_ERR_INVALID, "scene belongs to another context (or to none)");
  if ((npoints && !receivers) || (nlights && !lights && !sky)) return fail(CC_ERR_INVALID, "null inputs");
  cc_options opt;
  if (opt_in) opt = *opt_in; else cc_options_default(&opt);
  if (opt.hierarchy > 2) return fail(CC_ERR_INVALID, "hierarchy must be 0, 1 or 2");
  if (opt.points_per_warp < 1 || opt.points_per_warp > 32) return fail(CC_ERR_INVALID, "points_per_warp must be 1..32");
  if (!(opt.prefilter >= 0.0f)) return fail(CC_ERR_INVALID, "prefilter must be >= 0");
  if (opt.prefilter > 0.0f && opt.hierarchy != 2) return fail(CC_ERR_INVALID, "prefiltered cones need hierarchy 2");
  const bool back = (opt.flags & CC_BACK_FACING) != 0;
  if (back && (sky || opt.prefilter > 0.0f))
    return fail(CC_ERR_INVALID, "CC_BACK_FACING takes exact light cones only");
  if (back && !scene->flat.xforms.empty())
    return fail(CC_ERR_INVALID, "CC_BACK_FACING takes scenes without instancing");
  const uint64_t ncones = npoints * (uint64_t)nlights;
  if (ncones >= 0xffffffffull) return fail(CC_ERR_INVALID, "more than 2^32 - 1 cones in one call");
  if (npoints >= (1ull << 31)) return fail(CC_ERR_INVALID, "more than 2^31 - 1 points in one call");
  int rc = set_device(ctx);
  if (rc) return rc;
  cudaStream_t stream = stream_in ? (cudaStream_t)stream_in : ctx->stream;
  const bool device_ptrs = (opt.flags & CC_DEVICE_POINTERS) != 0;

  cc::DevQuery q;
  q.npoints = npoints;
  q.nlights = nlights;
  q.hierarchy = opt.hierarchy;
  q.wide_extent = opt.wide_extent;
  q.light_cone_cap = opt.light_cone_cap;
  q.wide_cone_cap = opt.wide_cone_cap;
  q.sky = sky;
  q.prefilter = opt.prefilter;
  q.cones = cones;
  q.cones_count = cones_count;
  if (back) {
    int rc2 = ensure_slots(const_cast<cc_scene*>(scene));
    if (rc2) return rc2;
    q.back = 1u;
    q.ntris = (uint32_t)(scene->flat.tris.size() / 12);
    q.tri_slot = scene->tri_slot;
  }
  cc::DevScene sd = scene->dev();
  if (opt.prefilter > 0.0f) {
    int rc2 = ensure_coverage(const_cast<cc_scene*>(scene));
    if (rc2) return rc2;
    sd = scene->dev();
    if (opt.flags & CC_NO_OBJECT_PREFILTER) sd.obj_cov = nullptr;
  }
  cc::DevOut o{};
  if (device_ptrs) {
    // The kernels read and write these with vector accesses.
    auto misaligned = [](const void* p, uintptr_t a) { return p && (reinterpret_cast<uintptr_t>(p) % a) != 0; };
    if (misaligned(receivers, 16) || misaligned(lights, 16) || misaligned(out->partial, 16) ||
        misaligned(out->work, 16) || misaligned(out->full, 8) || misaligned(out->any, 8) ||
        misaligned(out->irradiance, 4) || misaligned(out->fraction, 4))
      return fail(CC_ERR_INVALID, "device buffers must be aligned (receivers, lights, partial, work: 16 B; full, any: 8 B)");
    q.receivers = reinterpret_cast<const float4*>(receivers);
    q.lights = reinterpret_cast<const float4*>(lights);
    o.full = reinterpret_cast<uint2*>(out->full);
    o.any = reinterpret_cast<uint2*>(out->any);
    o.partial = out->partial;
    o.irradiance = out->irradiance;
    o.fraction = out->fraction;
    o.work = reinterpret_cast<uint4*>(out->work);
  } else {
    CC_CUDA(ctx->receivers.reserve(npoints * 32), "receivers buffer");
    CC_CUDA(cudaMemcpyAsync(ctx->receivers.ptr, receivers, npoints * 32, cudaMemcpyHostToDevice, stream), "receivers upload");
    q.receivers = static_cast<const float4*>(ctx->receivers.ptr);
    q.lights = nullptr;
    if (!sky) {
      CC_CUDA(ctx->lights.reserve((size_t)nlights * 64), "lights buffer");
      CC_CUDA(cudaMemcpyAsync(ctx->lights.ptr, lights, (size_t)nlights * 64, cudaMemcpyHostToDevice, stream),
              "lights upload");
      q.lights = static_cast<const float4*>(ctx->lights.ptr);
    }
    if (out->full) { CC_CUDA(ctx->full.reserve(ncones * 8), "output"); o.full = static_cast<uint2*>(ctx->full.ptr); }
    if (out->any) { CC_CUDA(ctx->any.reserve(ncones * 8), "output"); o.any = static_cast<uint2*>(ctx->any.ptr); }
    if (out->partial) { CC_CUDA(ctx->partial.reserve(ncones * 256), "output"); o.partial = static_cast<float*>(ctx->partial.ptr); }
    if (out->irradiance) { CC_CUDA(ctx->irradiance.reserve(ncones * 4), "output"); o.irradiance = static_cast<float*>(ctx->irradiance.ptr); }
    if (out->fraction) { CC_CUDA(ctx->fraction.reserve(ncones * 4), "output"); o.fraction = static_cast<float*>(ctx->fraction.ptr); }
    if (out->work) { CC_CUDA(ctx->work.reserve(ncones * 16), "output"); o.work = static_cast<uint4*>(ctx->work.ptr); }
  }
  uint32_t* counters = static_cast<uint32_t*>(ctx->counters.ptr);
  o.redo_count = counters;
  o.error = counters + 1;
  o.next_packet = counters + 2;
  o.next_solo = counters + 3;
  if (!(opt.flags & CC_NO_REDO)) {
    CC_CUDA(ctx->redo.reserve(std::max<uint64_t>(ncones, 1) * 4), "redo list");
    o.redo_list = static_cast<uint32_t*>(ctx->redo.ptr);
    o.redo_capacity = (uint32_t)std::max<uint64_t>(ncones, 1);
  }
  CC_CUDA(cudaMemsetAsync(counters, 0, cc::kCounterWords * sizeof(uint32_t), stream), "counter reset");
  if (!sky && opt.prefilter <= 0.0f) {
    // The split path's scratch: one chunk of cone records and masks.
    const uint64_t slots = std::max<uint64_t>(std::min<uint64_t>(ncones, ctx->split_chunk), 1);
    CC_CUDA(ctx->records.reserve(slots * sizeof(cc::ConeRecord)), "cone records");
    CC_CUDA(ctx->masks.reserve(slots * 256), "cone masks");
    q.records = static_cast<const cc::ConeRecord*>(ctx->records.ptr);
    o.cov_out = static_cast<float*>(ctx->masks.ptr);
  }
  // Walk the points in Morton order of their positions (coherent packets).
  q.order = nullptr;
  if (!(opt.flags & CC_KEEP_ORDER) && !cones && npoints > 64 && !scene->flat.nodes.empty()) {
    CC_CUDA(ctx->order.reserve(npoints * sizeof(uint32_t)), "walk order");
    const size_t need = cc::walk_order_scratch_bytes(npoints);
    CC_CUDA(ctx->sort_scratch.reserve(need), "walk order scratch");
    CC_CUDA(cc::walk_order(q.receivers, npoints, scene->flat.nodes[0].lo, scene->flat.nodes[0].hi,
                           ctx->sort_scratch.ptr, ctx->sort_scratch.size, static_cast<uint32_t*>(ctx->order.ptr),
                           stream),
            "walk order");
    q.order = static_cast<const uint32_t*>(ctx->order.ptr);
  }
  // Lights with wider cones first (the split path; results do not depend on
  // the order).
  if (!(opt.flags & CC_KEEP_ORDER) && !cones && q.records && nlights >= 2 && nlights <= cc::kMaxOrderedLights &&
      npoints > 0) {
    CC_CUDA(ctx->light_order.reserve(nlights * sizeof(uint32_t)), "light order");
    CC_CUDA(cc::launch_light_order(q, static_cast<uint32_t*>(ctx->light_order.ptr), stream), "light order");
    q.light_order = static_cast<const uint32_t*>(ctx->light_order.ptr);
  }
  // The call's slot in the timing ring (the oldest unread call is dropped
  // when the ring is full).
  const int ring = cc_context::kTimingRing;
  if (ctx->timed_count == ring) {
    ctx->timed_first = (ctx->timed_first + 1) % ring;
    ctx->timed_count--;
  }
  const int slot = (ctx->timed_first + ctx->timed_count) % ring;
  ctx->timed_count++;
  // Host buffers: FULL/ANY are final once the walk passes end, so they go
  // down on the copy stream while the integration runs.
  const bool early = !device_ptrs && (out->full || out->any) && o.cov_out != nullptr;
  CC_CUDA(cc::launch_visibility(sd, q, o, opt.points_per_warp, o.work != nullptr, ctx->split_chunk, ctx->sm_count,
                                stream, &ctx->marks[3 * slot], early ? ctx->walked : nullptr),
          "visibility launch");
  if (device_ptrs) return CC_OK;

  cudaStream_t words = stream;
  if (early) {
    CC_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->walked, 0), "download order");
    words = ctx->copy_stream;
  }
  if (out->full) CC_CUDA(cudaMemcpyAsync(out->full, o.full, ncones * 8, cudaMemcpyDeviceToHost, words), "download");
  if (out->any) CC_CUDA(cudaMemcpyAsync(out->any, o.any, ncones * 8, cudaMemcpyDeviceToHost, words), "download");
  if (early) {
    CC_CUDA(cudaEventRecord(ctx->copied, ctx->copy_stream), "download order");
    CC_CUDA(cudaStreamWaitEvent(stream, ctx->copied, 0), "download order");
  }
  if (out->partial) CC_CUDA(cudaMemcpyAsync(out->partial, o.partial, ncones * 256, cudaMemcpyDeviceToHost, stream), "download");
  if (out->irradiance) CC_CUDA(cudaMemcpyAsync(out->irradiance, o.irradiance, ncones * 4, cudaMemcpyDeviceToHost, stream), "download");
  if (out->fraction) CC_CUDA(cudaMemcpyAsync(out->fraction, o.fraction, ncones * 4, cudaMemcpyDeviceToHost, stream), "download");
  if (out->work) CC_CUDA(cudaMemcpyAsync(out->work, o.work, ncones * 16, cudaMemcpyDeviceToHost, stream), "download");
  uint32_t host_counters[2] = {0, 0};
  CC_CUDA(cudaMemcpyAsync(host_counters, counters, sizeof(host_counters), cudaMemcpyDeviceToHost, stream), "status download");
  CC_CUDA(cudaStreamSynchronize(stream), "visibility");
  if (host_counters[1] & 2u) return fail(CC_ERR_STACK, "a traversal stack overflowed");
  if (host_counters[1] & 1u) return fail(CC_ERR_INVALID, "solo re-walk list overflowed");
  return CC_OK;
}

namespace {
// sky_irradiance (:1411-1426): the six faces' light summed in face order.
__global__ void sum_sky_faces(const float* __restrict__ faces, uint64_t npoints, float* __restrict__ out) {
  const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (p >= npoints) return;
  float total = 0.0f;
#pragma unroll
  for (int f = 0; f < 6; ++f) total += faces[f * npoints + p];
  out[p] = total;
}
}  // namespace

extern "C" {

int cc_visibility(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                  const float* lights, uint32_t nlights, const cc_options* opt, const cc_outputs* out,
                  void* stream) {
  return cc_host::visibility_impl(ctx, scene, receivers, npoints, lights, nlights, opt, out, stream, 0u, nullptr,
                                  nullptr);
}

int cc_scene_set_clear(cc_scene* s, const float* clear, uint32_t nobjects) {
  if (!s || (nobjects && !clear)) return fail(CC_ERR_INVALID, "null argument");
  cc::FlatScene& f = s->flat;
  if (f.xforms.empty() || f.object_geometry.empty())
    return fail(CC_ERR_INVALID, "blended and transmissive objects are placed objects: the scene is not instanced");
  if (nobjects != f.object_geometry.size()) return fail(CC_ERR_INVALID, "one value per object, in their order");
  for (uint32_t m = 0; m < nobjects; ++m)
    if (!std::isfinite(clear[m]) || clear[m] >= 1.0f) return fail(CC_ERR_INVALID, "clear must be finite and below 1");
  for (uint32_t m = 0; m < nobjects; ++m) f.xforms[16 * (size_t)f.ranges[4 * m + 3] + 14] = clear[m];
  if (!s->ctx) return CC_OK;
  int rc = set_device(s->ctx);
  if (rc) return rc;
  CC_CUDA(cudaMemcpy(s->xforms, f.xforms.data(), f.xforms.size() * sizeof(float), cudaMemcpyHostToDevice),
          "object transforms");
  if (s->coverage_ready) {
    // The prefiltered cones' samples scale with the objects' opacity: the
    // same buffers, refilled.
    const std::vector<float> blas = cc::blas_coverage(f);
    if (!blas.empty())
      CC_CUDA(cudaMemcpy(s->blas_cov, blas.data(), blas.size() * sizeof(float), cudaMemcpyHostToDevice),
              "triangle-node coverage");
    const std::vector<float> obj = cc::object_coverage(f, blas);
    if (!obj.empty() && s->obj_cov)
      CC_CUDA(cudaMemcpy(s->obj_cov, obj.data(), obj.size() * sizeof(float), cudaMemcpyHostToDevice),
              "object-node coverage");
  }
  return CC_OK;
}

int64_t cc_scene_coverage(const cc_scene* scene, float* blas27, uint64_t max_blas, float* obj27, uint64_t max_obj) {
  if (!scene) return -(int64_t)fail(CC_ERR_INVALID, "null scene");
  const std::vector<float> blas = cc::blas_coverage(scene->flat);
  const uint64_t nb = blas.size() / cc::kCoverageSamples;
  if (blas27) std::copy(blas.begin(), blas.begin() + std::min(nb, max_blas) * cc::kCoverageSamples, blas27);
  if (obj27 && !scene->flat.xforms.empty()) {
    const std::vector<float> obj = cc::object_coverage(scene->flat, blas);
    const uint64_t no = obj.size() / cc::kCoverageSamples;
    std::copy(obj.begin(), obj.begin() + std::min(no, max_obj) * cc::kCoverageSamples, obj27);
  }
  return (int64_t)nb;
}

int cc_sky_visibility(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                      const cc_options* opt_in, uint32_t sky_flags, float* irradiance, const cc_outputs* faces,
                      void* stream_in) {
  if (!ctx || !scene || !irradiance) return fail(CC_ERR_INVALID, "null argument");
  if (scene->ctx != ctx) return fail(CC_ERR_INVALID, "scene belongs to another context (or to none)");
  if (npoints && !receivers) return fail(CC_ERR_INVALID, "null inputs");
  if (sky_flags & ~(CC_SKY_COMBINE_MAX | CC_SKY_NO_HORIZON_CULL | CC_SKY_OBJECT_FRAME))
    return fail(CC_ERR_INVALID, "unknown sky flags");
  if (npoints >= (0xffffffffull / 6)) return fail(CC_ERR_INVALID, "too many receivers in one call");
  cc_options opt;
  if (opt_in) opt = *opt_in; else cc_options_default(&opt);
  int rc = set_device(ctx);
  if (rc) return rc;
  cudaStream_t stream = stream_in ? (cudaStream_t)stream_in : ctx->stream;
  const bool device_ptrs = (opt.flags & CC_DEVICE_POINTERS) != 0;
  const uint64_t ncones = 6 * npoints;
  uint32_t sky = cc::kSkyCones;
  if (sky_flags & CC_SKY_COMBINE_MAX) sky |= cc::kSkyCombineMax;
  if (sky_flags & CC_SKY_NO_HORIZON_CULL) sky |= cc::kSkyNoHorizonCull;
  if (sky_flags & CC_SKY_OBJECT_FRAME) sky |= cc::kSkyObjectFrame;
  // The face cones run on device buffers: the caller's with device pointers,
  // else the context's.
  cc_outputs fo{};
  if (device_ptrs && faces) fo = *faces;
  const float* d_rec = receivers;
  if (!device_ptrs) {
    CC_CUDA(ctx->receivers.reserve(npoints * 32), "receivers buffer");
    CC_CUDA(cudaMemcpyAsync(ctx->receivers.ptr, receivers, npoints * 32, cudaMemcpyHostToDevice, stream),
            "receivers upload");
    d_rec = static_cast<const float*>(ctx->receivers.ptr);
    if (faces) {
      if (faces->full) { CC_CUDA(ctx->full.reserve(ncones * 8), "output"); fo.full = static_cast<uint32_t*>(ctx->full.ptr); }
      if (faces->any) { CC_CUDA(ctx->any.reserve(ncones * 8), "output"); fo.any = static_cast<uint32_t*>(ctx->any.ptr); }
      if (faces->partial) { CC_CUDA(ctx->partial.reserve(ncones * 256), "output"); fo.partial = static_cast<float*>(ctx->partial.ptr); }
      if (faces->fraction) { CC_CUDA(ctx->fraction.reserve(ncones * 4), "output"); fo.fraction = static_cast<float*>(ctx->fraction.ptr); }
      if (faces->work) { CC_CUDA(ctx->work.reserve(ncones * 16), "output"); fo.work = static_cast<uint32_t*>(ctx->work.ptr); }
    }
  }
  if (!fo.irradiance) {
    CC_CUDA(ctx->irradiance.reserve(std::max<uint64_t>(ncones, 1) * 4), "sky faces");
    fo.irradiance = static_cast<float*>(ctx->irradiance.ptr);
  }
  float* d_sum = irradiance;
  if (!device_ptrs) {
    CC_CUDA(ctx->sky_sum.reserve(std::max<uint64_t>(npoints, 1) * 4), "sky sum");
    d_sum = static_cast<float*>(ctx->sky_sum.ptr);
  }
  cc_options vo = opt;
  vo.flags |= CC_DEVICE_POINTERS;
  rc = cc_host::visibility_impl(ctx, scene, d_rec, npoints, nullptr, 6, &vo, &fo, stream, sky, nullptr, nullptr);
  if (rc) return rc;
  if (npoints) {
    sum_sky_faces<<<(unsigned)((npoints + 255) / 256), 256, 0, stream>>>(fo.irradiance, npoints, d_sum);
    CC_CUDA(cudaGetLastError(), "sky sum");
  }
  if (device_ptrs) return CC_OK;
  CC_CUDA(cudaMemcpyAsync(irradiance, d_sum, npoints * 4, cudaMemcpyDeviceToHost, stream), "download");
  if (faces) {
    if (faces->irradiance) CC_CUDA(cudaMemcpyAsync(faces->irradiance, fo.irradiance, ncones * 4, cudaMemcpyDeviceToHost, stream), "download");
    if (faces->full) CC_CUDA(cudaMemcpyAsync(faces->full, fo.full, ncones * 8, cudaMemcpyDeviceToHost, stream), "download");
    if (faces->any) CC_CUDA(cudaMemcpyAsync(faces->any, fo.any, ncones * 8, cudaMemcpyDeviceToHost, stream), "download");
    if (faces->partial) CC_CUDA(cudaMemcpyAsync(faces->partial, fo.partial, ncones * 256, cudaMemcpyDeviceToHost, stream), "download");
    if (faces->fraction) CC_CUDA(cudaMemcpyAsync(faces->fraction, fo.fraction, ncones * 4, cudaMemcpyDeviceToHost, stream), "download");
    if (faces->work) CC_CUDA(cudaMemcpyAsync(faces->work, fo.work, ncones * 16, cudaMemcpyDeviceToHost, stream), "download");
  }
  uint32_t host_counters[2] = {0, 0};
  CC_CUDA(cudaMemcpyAsync(host_counters, ctx->counters.ptr, sizeof(host_counters), cudaMemcpyDeviceToHost, stream),
          "status download");
  CC_CUDA(cudaStreamSynchronize(stream), "sky visibility");
  if (host_counters[1] & 2u) return fail(CC_ERR_STACK, "a traversal stack overflowed");
  if (host_counters[1] & 1u) return fail(CC_ERR_INVALID, "solo re-walk list overflowed");
  return CC_OK;
}

int cc_visibility_static(const cc_scene* scene, const float* receivers, uint64_t npoints, const float* lights,
                         uint32_t nlights, const cc_options* opt_in, const cc_outputs* out, void* stream_in) {
  static_assert(cc::kStaticMaxCones == CC_STATIC_MAX_CONES, "header and library disagree on the limit");
  if (!scene || !out) return fail(CC_ERR_INVALID, "null argument");
  if (!scene->ctx) return fail(CC_ERR_INVALID, "scene is not on a device");
  if ((npoints && !receivers) || (nlights && !lights)) return fail(CC_ERR_INVALID, "null inputs");
  cc_options opt;
  if (opt_in) opt = *opt_in; else cc_options_default(&opt);
  if (opt.hierarchy > 2) return fail(CC_ERR_INVALID, "hierarchy must be 0, 1 or 2");
  if (opt.points_per_warp < 1 || opt.points_per_warp > 32) return fail(CC_ERR_INVALID, "points_per_warp must be 1..32");
  if (opt.prefilter != 0.0f) return fail(CC_ERR_INVALID, "cc_visibility_static takes exact cones only (prefilter 0)");
  if (opt.flags & CC_BACK_FACING) return fail(CC_ERR_INVALID, "CC_BACK_FACING is cc_visibility's");
  if (npoints > CC_STATIC_MAX_CONES || npoints * (uint64_t)nlights > CC_STATIC_MAX_CONES)
    return fail(CC_ERR_INVALID, "more than CC_STATIC_MAX_CONES cones (or points) in one cc_visibility_static call");
  const uint64_t ncones = npoints * (uint64_t)nlights;
  auto misaligned = [](const void* p, uintptr_t a) { return p && (reinterpret_cast<uintptr_t>(p) % a) != 0; };
  if (misaligned(receivers, 16) || misaligned(lights, 16) || misaligned(out->partial, 16) ||
      misaligned(out->work, 16) || misaligned(out->full, 8) || misaligned(out->any, 8) ||
      misaligned(out->irradiance, 4) || misaligned(out->fraction, 4))
    return fail(CC_ERR_INVALID, "device buffers must be aligned (receivers, lights, partial, work: 16 B; full, any: 8 B)");
  cc_context* ctx = scene->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  cudaStream_t stream = stream_in ? (cudaStream_t)stream_in : ctx->stream;
  void* base = nullptr;
  CC_CUDA(cc::static_scratch(ctx->device, &base), "static scratch address");
  uint8_t* scratch = static_cast<uint8_t*>(base);

  cc::DevQuery q;
  q.receivers = reinterpret_cast<const float4*>(receivers);
  q.lights = reinterpret_cast<const float4*>(lights);
  q.npoints = npoints;
  q.nlights = nlights;
  q.hierarchy = opt.hierarchy;
  q.wide_extent = opt.wide_extent;
  q.light_cone_cap = opt.light_cone_cap;
  q.wide_cone_cap = opt.wide_cone_cap;
  q.order = nullptr;
  cc::DevOut o{};
  o.full = reinterpret_cast<uint2*>(out->full);
  o.any = reinterpret_cast<uint2*>(out->any);
  o.partial = out->partial;
  o.irradiance = out->irradiance;
  o.fraction = out->fraction;
  o.work = reinterpret_cast<uint4*>(out->work);
  uint32_t* counters = reinterpret_cast<uint32_t*>(scratch);
  o.redo_count = counters;
  o.error = counters + 1;
  o.next_packet = counters + 2;
  o.next_solo = counters + 3;
  if (!(opt.flags & CC_NO_REDO)) {
    o.redo_list = reinterpret_cast<uint32_t*>(scratch + cc::kStaticRedoOffset);
    o.redo_capacity = (uint32_t)std::max<uint64_t>(ncones, 1);
  }
  // The counters are the only scratch that must start at zero.
  CC_CUDA(cudaMemsetAsync(counters, 0, cc::kCounterWords * sizeof(uint32_t), stream), "counter reset");
  if (!(opt.flags & CC_KEEP_ORDER) && npoints > 64 && !scene->flat.nodes.empty()) {
    const size_t sort_bytes = cc::kStaticScratchBytes - cc::kStaticSortOffset;
    if (cc::walk_order_scratch_bytes(npoints) > sort_bytes)
      return fail(CC_ERR_INVALID, "walk order scratch exceeds the static scratch");
    uint32_t* order = reinterpret_cast<uint32_t*>(scratch + cc::kStaticOrderOffset);
    CC_CUDA(cc::walk_order(q.receivers, npoints, scene->flat.nodes[0].lo, scene->flat.nodes[0].hi,
                           scratch + cc::kStaticSortOffset, sort_bytes, order, stream),
            "walk order");
    q.order = order;
  }
  // The split path's records and masks, over the sort scratch (used up by now).
  q.records = reinterpret_cast<const cc::ConeRecord*>(scratch + cc::kStaticRecordsOffset);
  o.cov_out = reinterpret_cast<float*>(scratch + cc::kStaticMasksOffset);
  CC_CUDA(cc::launch_visibility(scene->dev(), q, o, opt.points_per_warp, o.work != nullptr, cc::kStaticMaxCones,
                                ctx->sm_count, stream, nullptr, nullptr),
          "visibility launch");
  return CC_OK;
}

static void receivers_from6(const float* r6, uint64_t n, std::vector<float>& out) {
  out.assign(n * 8, 0.0f);
  for (uint64_t i = 0; i < n; ++i) {
    out[8 * i + 0] = r6[6 * i + 0];
    out[8 * i + 1] = r6[6 * i + 1];
    out[8 * i + 2] = r6[6 * i + 2];
    out[8 * i + 4] = r6[6 * i + 3];
    out[8 * i + 5] = r6[6 * i + 4];
    out[8 * i + 6] = r6[6 * i + 5];
  }
}

// RectLight -> LightGpu (lib.rs:722-728).
static void light_from9(const float* l9, int one_sided, float* out16) {
  std::memset(out16, 0, 16 * sizeof(float));
  for (int k = 0; k < 3; ++k) {
    out16[k] = l9[k];
    out16[4 + k] = l9[3 + k];
    out16[8 + k] = l9[6 + k];
  }
  out16[3] = one_sided ? 1.0f : 0.0f;
  out16[12] = out16[13] = out16[14] = 1.0f;
}

int cc_irradiance(cc_context* ctx, const float* receivers6, uint64_t npoints, const float* light9, int one_sided,
                  const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes, uint32_t hierarchy,
                  uint32_t runs, float* out, double* best_seconds) {
  if (!ctx || !light9 || !out || (npoints && !receivers6)) return fail(CC_ERR_INVALID, "null argument");
  if (hierarchy > 2) return fail(CC_ERR_INVALID, "hierarchy must be 0, 1 or 2");
  cc_scene* scene = nullptr;
  int rc = cc_scene_build(ctx, tri9, mesh_counts, nmeshes, &scene);
  if (rc) return rc;
  std::vector<float> rec;
  receivers_from6(receivers6, npoints, rec);
  float light[16];
  light_from9(light9, one_sided, light);
  cc_options opt;
  cc_options_default(&opt);
  opt.hierarchy = hierarchy;
  opt.flags = CC_DEVICE_POINTERS;
  // Inputs and the output on the device, then `runs` timed executions.
  float4* d_rec = nullptr;
  float4* d_light = nullptr;
  float* d_out = nullptr;
  auto cleanup = [&] {
    cudaFree(d_rec);
    cudaFree(d_light);
    cudaFree(d_out);
    cc_scene_destroy(scene);
  };
  cudaError_t e = cudaMalloc(&d_rec, std::max<uint64_t>(npoints, 1) * 32);
  if (e == cudaSuccess) e = cudaMalloc(&d_light, 64);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, std::max<uint64_t>(npoints, 1) * 4);
  if (e == cudaSuccess && npoints) e = cudaMemcpy(d_rec, rec.data(), npoints * 32, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_light, light, 64, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cleanup();
    return cuda_fail(e, "irradiance inputs");
  }
  cc_outputs o{};
  o.irradiance = d_out;
  double best = INFINITY;
  for (uint32_t r = 0; r < std::max(runs, 1u); ++r) {
    cudaEventRecord(ctx->ev0, ctx->stream);
    rc = cc_visibility(ctx, scene, reinterpret_cast<const float*>(d_rec), npoints, reinterpret_cast<const float*>(d_light),
                       1, &opt, &o, ctx->stream);
    if (rc) {
      cleanup();
      return rc;
    }
    cudaEventRecord(ctx->ev1, ctx->stream);
    e = cudaEventSynchronize(ctx->ev1);
    if (e != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "irradiance");
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    best = std::min(best, ms * 1e-3);
  }
  uint32_t host_counters[2] = {0, 0};
  e = cudaMemcpy(host_counters, ctx->counters.ptr, sizeof(host_counters), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && npoints) e = cudaMemcpy(out, d_out, npoints * 4, cudaMemcpyDeviceToHost);
  cleanup();
  if (e != cudaSuccess) return cuda_fail(e, "irradiance download");
  if (host_counters[1] & 2u) return fail(CC_ERR_STACK, "a traversal stack overflowed");
  if (best_seconds) *best_seconds = best;
  return CC_OK;
}

int cc_coverage(cc_context* ctx, const float* receivers6, uint64_t npoints, const float* light9, int one_sided,
                const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes, float* out64) {
  if (!ctx || !light9 || !out64 || (npoints && !receivers6)) return fail(CC_ERR_INVALID, "null argument");
  cc_scene* scene = nullptr;
  int rc = cc_scene_build(ctx, tri9, mesh_counts, nmeshes, &scene);
  if (rc) return rc;
  std::vector<float> rec;
  receivers_from6(receivers6, npoints, rec);
  float light[16];
  light_from9(light9, one_sided, light);
  cc_options opt;
  cc_options_default(&opt);
  opt.hierarchy = 0;
  cc_outputs o{};
  o.partial = out64;
  rc = cc_visibility(ctx, scene, rec.data(), npoints, light, 1, &opt, &o, nullptr);
  cc_scene_destroy(scene);
  return rc;
}

}  // extern "C"
