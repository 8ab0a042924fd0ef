// Movers in instanced scenes: the cones a moved object may have changed, and
// their recomputation.
//
// A cone from point p toward light l may have changed when a moved object's
// box, at its old or its new place, meets the convex hull of p and the
// light's box (hull_meets, mask_cones.wgsl:3903-3917; may_be_shadowed,
// :3961-3974, for a point instead of a page's box). Per light, the boxes'
// shadow regions (shadow_region, crates/continuum-gpu/src/hierarchy.rs:
// 418-457) are gathered in a small hierarchy on the host; on the device each
// (light, point) walks its light's hierarchy and runs the exact hull test on
// the boxes whose regions hold the point.
#include <cub/device/device_select.cuh>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "capi_internal.h"

using namespace cc_host;

namespace cc {
namespace {

struct Box3 {
  float lo[3], hi[3];
};

// light_box (mask_cones.wgsl:3887-3898): a box around the light.
Box3 light_box(const float* L) {
  const bool sphere = L[3] > 1.5f;
  float c[3], radius;
  if (sphere) {
    for (int k = 0; k < 3; ++k) c[k] = L[k];
    radius = 1.5f * L[4];
  } else {
    for (int k = 0; k < 3; ++k) c[k] = L[k] + (L[4 + k] + L[8 + k]) * 0.5f;
    const float lu = std::sqrt(L[4] * L[4] + L[5] * L[5] + L[6] * L[6]);
    const float lv = std::sqrt(L[8] * L[8] + L[9] * L[9] + L[10] * L[10]);
    radius = 0.5f * (lu + lv);
  }
  const float far = std::max(std::max(std::max(std::fabs(c[0]), 1.0f), std::max(std::fabs(c[1]), 1.0f)),
                             std::max(std::fabs(c[2]), 1.0f));
  radius = radius * 1.001f + 1e-5f * far + 1e-4f;
  Box3 b;
  for (int k = 0; k < 3; ++k) {
    b.lo[k] = c[k] - radius;
    b.hi[k] = c[k] + radius;
  }
  return b;
}

// shadow_region (hierarchy.rs:418-457): a box around where a cone from a
// point to the light box `l` can meet box `m`, clipped to `s`; false if none.
bool shadow_region(const Box3& m, const Box3& l, const Box3& s, Box3& out) {
  float d_lo[3], d_hi[3];
  for (int a = 0; a < 3; ++a) {
    d_lo[a] = m.lo[a] - l.hi[a];
    d_hi[a] = m.hi[a] - l.lo[a];
  }
  float t0 = 0.0f, t1 = INFINITY;
  for (int a = 0; a < 3; ++a) {
    float b = d_lo[a], c = s.hi[a] - m.lo[a];
    if (b > 0.0f) t1 = std::min(t1, c / b);
    else if (b < 0.0f) t0 = std::max(t0, c / b);
    else if (c < 0.0f) return false;
    b = d_hi[a];
    c = s.lo[a] - m.hi[a];
    if (b > 0.0f) t0 = std::max(t0, c / b);
    else if (b < 0.0f) t1 = std::min(t1, c / b);
    else if (c > 0.0f) return false;
  }
  if (t0 > t1 * (1.0f + 1e-6f) + 1e-6f) return false;
  if (!std::isfinite(t1)) {
    out = s;
    return true;
  }
  float lo[3], hi[3], mx = 1.0f;
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::max(std::min(m.lo[a] + d_lo[a] * t0, m.lo[a] + d_lo[a] * t1), s.lo[a]);
    hi[a] = std::min(std::max(m.hi[a] + d_hi[a] * t0, m.hi[a] + d_hi[a] * t1), s.hi[a]);
    mx = std::max(mx, std::max(std::fabs(lo[a]), std::fabs(hi[a])));
  }
  const float pad = 1e-4f * mx;
  for (int a = 0; a < 3; ++a) {
    out.lo[a] = lo[a] - pad;
    out.hi[a] = hi[a] + pad;
  }
  return true;
}

// hull_meets (mask_cones.wgsl:3903-3917) for a point p: whether box m meets
// the convex hull of p and the light box l.
__device__ __forceinline__ bool hull_meets_point(float3 p, const float* l, const float* m) {
  float s0 = 0.0f, s1 = 1.0f;
  const float pc[3] = {p.x, p.y, p.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float b0 = l[a] - pc[a];
    const float c0 = m[3 + a] - pc[a];
    if (b0 > 0.0f) s1 = fminf(s1, c0 / b0);
    else if (b0 < 0.0f) s0 = fmaxf(s0, c0 / b0);
    else if (c0 < 0.0f) return false;
    const float b1 = l[3 + a] - pc[a];
    const float c1 = m[a] - pc[a];
    if (b1 > 0.0f) s0 = fmaxf(s0, c1 / b1);
    else if (b1 < 0.0f) s1 = fminf(s1, c1 / b1);
    else if (c1 > 0.0f) return false;
  }
  return s0 <= s1 + 1e-6f;
}

struct StaleTables {
  const float4* nodes;     // per light's region hierarchy, 2 per node: (lo, first item or child), (hi, count)
  const uint32_t* roots;   // per light: its root node
  const uint32_t* items;   // region index per leaf slot
  const uint32_t* region_box;  // per region: its mover box (index into boxes)
  const float* regions;    // 6 per region: its box
  const float* boxes;      // 6 per box: lo, hi (2 per mover: old, new)
  const float* lboxes;     // 6 per light
};

constexpr int kStaleStack = 64;

__global__ void stale_kernel(const float4* __restrict__ receivers, uint64_t npoints, uint32_t nlights, StaleTables t,
                             uint8_t* __restrict__ stale, unsigned long long* __restrict__ count) {
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= npoints * (uint64_t)nlights) return;
  const uint32_t l = (uint32_t)(c / npoints);
  const uint64_t p = c - (uint64_t)l * npoints;
  const float4 q = __ldg(&receivers[2 * p]);
  const float3 pt = make_float3(q.x, q.y, q.z);
  bool hit = false;
  const uint32_t root = __ldg(&t.roots[l]);
  if (root != kNone) {
    uint32_t stack[kStaleStack];
    int sp = 0;
    stack[sp++] = root;
    while (sp > 0 && !hit) {
      const uint32_t n = stack[--sp];
      const float4 a = __ldg(&t.nodes[2 * n]), b = __ldg(&t.nodes[2 * n + 1]);
      // boxes_meet for the point's box (:3919-3921)
      if (pt.x < a.x || pt.y < a.y || pt.z < a.z || pt.x > b.x || pt.y > b.y || pt.z > b.z) continue;
      const uint32_t first = __float_as_uint(a.w), cnt = __float_as_uint(b.w);
      if (cnt > 0) {
        for (uint32_t k = first; k < first + cnt && !hit; ++k) {
          const uint32_t r = __ldg(&t.items[k]);
          const float* rb = t.regions + 6 * (size_t)r;
          // boxes_meet(p, the region) && hull_meets(p, light box, the moved box) (:3969-3972)
          if (pt.x < rb[0] || pt.y < rb[1] || pt.z < rb[2] || pt.x > rb[3] || pt.y > rb[4] || pt.z > rb[5]) continue;
          const uint32_t box = __ldg(&t.region_box[r]);
          if (hull_meets_point(pt, t.lboxes + 6 * l, t.boxes + 6 * box)) hit = true;
        }
      } else if (sp + 2 <= kStaleStack) {
        stack[sp++] = first;
        stack[sp++] = first + 1;
      }
    }
  }
  stale[c] = hit ? 1 : 0;
  if (hit) atomicAdd(count, 1ull);
}

// Moved objects' transforms into place: transform index in slot[i].x (its
// bits), the 4 rows at rows[4 i ..].
__global__ void scatter_xforms(const float4* __restrict__ slot, const float4* __restrict__ rows, uint64_t n,
                               float4* __restrict__ xforms) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = __float_as_uint(slot[i].x);
  for (int r = 0; r < 4; ++r) xforms[4 * (size_t)x + r] = rows[4 * i + r];
}

__global__ void iota_kernel(uint32_t* out, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (uint32_t)i;
}

// Slot k = l * npoints + i walks cone l * npoints + order[i] (the points'
// walk order within each light; no order: the points' own); its flag is that
// cone's staleness.
__global__ void stale_in_order(const uint32_t* __restrict__ order, const uint8_t* __restrict__ stale, uint64_t npoints,
                               uint64_t ncones, uint32_t* __restrict__ perm, uint8_t* __restrict__ flags) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncones) return;
  const uint64_t l = k / npoints;
  const uint64_t i = k - l * npoints;
  const uint32_t c = (uint32_t)(l * npoints + (order ? order[i] : i));
  perm[k] = c;
  flags[k] = stale[c];
}


// A hierarchy over boxes (two per leaf), for the region tables.
inline uint32_t float_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float bits_float(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

struct BoxTree {
  std::vector<float4> nodes;
  std::vector<uint32_t> items;
};

void box_tree(const std::vector<Box3>& boxes, uint32_t node_base, uint32_t item_base, BoxTree& out) {
  // Median split on the longest centroid axis, as the scene hierarchies.
  struct Rec {
    uint32_t self, first, count;
  };
  std::vector<uint32_t> order(boxes.size());
  for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
  std::vector<float4> nodes(2);
  std::vector<Rec> todo{{0, 0, (uint32_t)boxes.size()}};
  while (!todo.empty()) {
    Rec r = todo.back();
    todo.pop_back();
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = r.first; i < r.first + r.count; ++i) {
      const Box3& b = boxes[order[i]];
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], b.lo[k]);
        hi[k] = std::max(hi[k], b.hi[k]);
        const float c = 0.5f * (b.lo[k] + b.hi[k]);
        clo[k] = std::min(clo[k], c);
        chi[k] = std::max(chi[k], c);
      }
    }
    uint32_t a_w, b_w;
    if (r.count <= 2) {
      a_w = item_base + r.first;
      b_w = r.count;
    } else {
      const float e[3] = {chi[0] - clo[0], chi[1] - clo[1], chi[2] - clo[2]};
      const int axis = (e[0] >= e[1] && e[0] >= e[2]) ? 0 : (e[1] >= e[2] ? 1 : 2);
      const uint32_t mid = r.count / 2;
      std::nth_element(order.begin() + r.first, order.begin() + r.first + mid, order.begin() + r.first + r.count,
                       [&](uint32_t x, uint32_t y) {
                         const float kx = boxes[x].lo[axis] + boxes[x].hi[axis];
                         const float ky = boxes[y].lo[axis] + boxes[y].hi[axis];
                         return kx < ky || (kx == ky && x < y);
                       });
      const uint32_t left = (uint32_t)(nodes.size() / 2);
      nodes.resize(nodes.size() + 4);
      a_w = node_base + left;
      b_w = 0;
      todo.push_back({left + 1, r.first + mid, r.count - mid});
      todo.push_back({left, r.first, mid});
    }
    float aw, bw;
    std::memcpy(&aw, &a_w, 4);
    std::memcpy(&bw, &b_w, 4);
    nodes[2 * r.self] = make_float4(lo[0], lo[1], lo[2], aw);
    nodes[2 * r.self + 1] = make_float4(hi[0], hi[1], hi[2], bw);
  }
  out.nodes = std::move(nodes);
  out.items.assign(order.begin(), order.end());
}

}  // namespace

size_t stale_list_scratch_bytes(uint64_t ncones) {
  size_t sel_bytes = 0;
  cub::DeviceSelect::Flagged(nullptr, sel_bytes, (const uint32_t*)nullptr, (const uint8_t*)nullptr, (uint32_t*)nullptr,
                             (uint32_t*)nullptr, (int)ncones);
  return std::max<size_t>(sel_bytes, 256);
}

cudaError_t stale_list(const uint32_t* order, const uint8_t* stale, uint64_t npoints, uint32_t nlights, uint32_t* perm,
                       uint8_t* flags, uint32_t* list, uint32_t* count, void* temp, size_t temp_bytes,
                       cudaStream_t stream) {
  const uint64_t ncones = npoints * (uint64_t)nlights;
  if (ncones == 0) return cudaMemsetAsync(count, 0, sizeof(uint32_t), stream);
  const unsigned threads = 256;
  stale_in_order<<<(unsigned)((ncones + threads - 1) / threads), threads, 0, stream>>>(order, stale, npoints, ncones,
                                                                                       perm, flags);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(temp, temp_bytes, perm, flags, list, count, (int)ncones, stream);
  return e;
}

}  // namespace cc

int cc_scene_move(cc_scene* s, const cc_instance* placements, uint32_t n, float* boxes12) {
  if (!s || (n && !placements)) return fail(CC_ERR_INVALID, "null argument");
  cc::FlatScene& f = s->flat;
  if (f.movers.objects.empty()) return fail(CC_ERR_INVALID, "the scene was built without movable objects");
  if (n != f.movers.objects.size()) return fail(CC_ERR_INVALID, "one placement per movable object, in their order");
  for (uint32_t i = 0; i < n; ++i) {
    const cc_instance& o = placements[i];
    if (o.geometry != f.object_geometry[f.movers.objects[i]])
      return fail(CC_ERR_INVALID, "a moved object keeps its geometry");
    if (!(o.scale > 0.0f) || !std::isfinite(o.scale)) return fail(CC_ERR_INVALID, "instance scale must be positive");
  }
  cc::move_instances(f, reinterpret_cast<const cc::Instance*>(placements), boxes12);
  if (!s->ctx) return CC_OK;
  int rc = set_device(s->ctx);
  if (rc) return rc;
  // The movers' transforms (gathered, sent at once and scattered into place
  // on the device), the root, the movers' subtree and their items.
  const cc::MoverTree& t = f.movers;
  if (!t.objects.empty()) {
    const size_t nm = t.objects.size();
    std::vector<float4> packed(5 * nm);
    for (size_t i = 0; i < nm; ++i) {
      const uint32_t x = f.ranges[4 * t.objects[i] + 3];
      float xi;
      std::memcpy(&xi, &x, 4);
      packed[i] = make_float4(xi, 0.f, 0.f, 0.f);
      for (int r = 0; r < 4; ++r) {
        const float* row = &f.xforms[16 * (size_t)x + 4 * r];
        packed[nm + 4 * i + r] = make_float4(row[0], row[1], row[2], row[3]);
      }
    }
    CC_CUDA(s->ctx->move_xforms.reserve(packed.size() * sizeof(float4)), "move transforms");
    float4* d = static_cast<float4*>(s->ctx->move_xforms.ptr);
    cudaError_t e = cudaMemcpy(d, packed.data(), packed.size() * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      cc::scatter_xforms<<<(unsigned)((nm + 127) / 128), 128>>>(d, d + nm, nm, s->xforms);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "move transforms");
  }
  auto put_nodes = [&](uint32_t first, uint32_t count) -> int {
    std::vector<float4> packed(2 * (size_t)count);
    for (uint32_t i = 0; i < count; ++i) {
      const cc::NodeGpu& nd = f.nodes[first + i];
      float a, b;
      std::memcpy(&a, &nd.info[0], 4);
      std::memcpy(&b, &nd.info[1], 4);
      packed[2 * i] = make_float4(nd.lo[0], nd.lo[1], nd.lo[2], a);
      packed[2 * i + 1] = make_float4(nd.hi[0], nd.hi[1], nd.hi[2], b);
    }
    CC_CUDA(cudaMemcpy(s->nodes + 2 * (size_t)first, packed.data(), packed.size() * sizeof(float4), cudaMemcpyHostToDevice),
            "move nodes");
    return CC_OK;
  };
  if ((rc = put_nodes(0, 3))) return rc;
  if (t.nodes && (rc = put_nodes(t.first_node, t.nodes))) return rc;
  CC_CUDA(cudaMemcpy(s->items + t.first_item, &f.items[t.first_item], t.objects.size() * 4, cudaMemcpyHostToDevice),
          "move items");
  return CC_OK;
}

int cc_stale_cones(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                   const float* lights16, uint32_t nlights, const float* boxes12, uint32_t nmovers, uint8_t* stale,
                   uint64_t* count, void* stream_in) {
  if (!ctx || !scene || (npoints && !receivers) || (nlights && !lights16) || (nmovers && !boxes12) || !count)
    return fail(CC_ERR_INVALID, "null argument");
  if (npoints * (uint64_t)nlights && !stale) return fail(CC_ERR_INVALID, "null output");
  int rc = set_device(ctx);
  if (rc) return rc;
  cudaStream_t stream = stream_in ? (cudaStream_t)stream_in : ctx->stream;
  // The scene's box (the root's), which holds every point that matters.
  cc::Box3 sbox;
  for (int k = 0; k < 3; ++k) {
    sbox.lo[k] = scene->flat.nodes[0].lo[k];
    sbox.hi[k] = scene->flat.nodes[0].hi[k];
  }
  // Per light: the regions of every mover box, old and new, and their hierarchy.
  std::vector<float> boxes(12 * (size_t)nmovers);
  std::memcpy(boxes.data(), boxes12, boxes.size() * 4);
  std::vector<float> lboxes(6 * (size_t)nlights);
  std::vector<float4> nodes;
  std::vector<uint32_t> roots(nlights, cc::kNone), items, region_box;
  std::vector<float> region_boxes;
  // Each light's regions and their hierarchy on a host thread of its own
  // (numbered from 0), then joined in light order, renumbered.
  std::vector<std::vector<cc::Box3>> regions(nlights);
  std::vector<std::vector<uint32_t>> which(nlights);
  std::vector<cc::BoxTree> trees(nlights);
  auto per_light = [&](uint32_t l) {
    const cc::Box3 lb = cc::light_box(lights16 + 16 * (size_t)l);
    for (int k = 0; k < 3; ++k) {
      lboxes[6 * l + k] = lb.lo[k];
      lboxes[6 * l + 3 + k] = lb.hi[k];
    }
    for (uint32_t b = 0; b < 2 * nmovers; ++b) {
      cc::Box3 m, r;
      for (int k = 0; k < 3; ++k) {
        m.lo[k] = boxes[6 * b + k];
        m.hi[k] = boxes[6 * b + 3 + k];
      }
      if (cc::shadow_region(m, lb, sbox, r)) {
        regions[l].push_back(r);
        which[l].push_back(b);
      }
    }
    if (!regions[l].empty()) cc::box_tree(regions[l], 0, 0, trees[l]);
  };
  {
    std::vector<std::thread> pool;
    for (uint32_t l = 1; l < nlights; ++l) pool.emplace_back(per_light, l);
    if (nlights) per_light(0);
    for (std::thread& th : pool) th.join();
  }
  for (uint32_t l = 0; l < nlights; ++l) {
    if (regions[l].empty()) continue;
    const uint32_t node_base = (uint32_t)(nodes.size() / 2);
    const uint32_t item_base = (uint32_t)items.size();
    roots[l] = node_base;
    std::vector<float4>& tn = trees[l].nodes;
    for (size_t i = 0; i < tn.size(); i += 2) {
      uint32_t a = cc::float_bits(tn[i].w), b = cc::float_bits(tn[i + 1].w);
      a += b == 0 ? node_base : item_base;  // interior: left child; leaf: first item
      tn[i].w = cc::bits_float(a);
    }
    nodes.insert(nodes.end(), tn.begin(), tn.end());
    const uint32_t region_base = (uint32_t)region_box.size();
    for (uint32_t k : trees[l].items) items.push_back(region_base + k);
    region_box.insert(region_box.end(), which[l].begin(), which[l].end());
    for (const cc::Box3& r : regions[l])
      region_boxes.insert(region_boxes.end(), {r.lo[0], r.lo[1], r.lo[2], r.hi[0], r.hi[1], r.hi[2]});
  }
  // Tables to the device (one buffer, kept for the next frame).
  auto bytes_of = [](size_t n, size_t each) { return (n * each + 255) & ~size_t(255); };
  const size_t b_nodes = bytes_of(nodes.size(), sizeof(float4)), b_roots = bytes_of(roots.size(), 4),
               b_items = bytes_of(items.size(), 4), b_rbox = bytes_of(region_box.size(), 4),
               b_boxes = bytes_of(boxes.size(), 4), b_lbox = bytes_of(lboxes.size(), 4), b_count = 256,
               b_regions = bytes_of(region_boxes.size(), 4);
  CC_CUDA(ctx->stale_tables.reserve(b_nodes + b_roots + b_items + b_rbox + b_boxes + b_lbox + b_regions + b_count),
          "stale tables");
  uint8_t* at = static_cast<uint8_t*>(ctx->stale_tables.ptr);
  auto put = [&](const void* src, size_t n, size_t padded) {
    uint8_t* p = at;
    if (n) cudaMemcpyAsync(p, src, n, cudaMemcpyHostToDevice, stream);
    at += padded;
    return p;
  };
  cc::StaleTables t;
  t.nodes = reinterpret_cast<const float4*>(put(nodes.data(), nodes.size() * sizeof(float4), b_nodes));
  t.roots = reinterpret_cast<const uint32_t*>(put(roots.data(), roots.size() * 4, b_roots));
  t.items = reinterpret_cast<const uint32_t*>(put(items.data(), items.size() * 4, b_items));
  t.region_box = reinterpret_cast<const uint32_t*>(put(region_box.data(), region_box.size() * 4, b_rbox));
  t.boxes = reinterpret_cast<const float*>(put(boxes.data(), boxes.size() * 4, b_boxes));
  t.lboxes = reinterpret_cast<const float*>(put(lboxes.data(), lboxes.size() * 4, b_lbox));
  t.regions = reinterpret_cast<const float*>(put(region_boxes.data(), region_boxes.size() * 4, b_regions));
  unsigned long long* d_count = reinterpret_cast<unsigned long long*>(at);
  cudaMemsetAsync(d_count, 0, 8, stream);
  const uint64_t cones = npoints * (uint64_t)nlights;
  if (cones) {
    const unsigned threads = 256;
    cc::stale_kernel<<<(unsigned)((cones + threads - 1) / threads), threads, 0, stream>>>(
        reinterpret_cast<const float4*>(receivers), npoints, nlights, t, stale, d_count);
  }
  unsigned long long host_count = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&host_count, d_count, 8, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "stale cones");
  *count = host_count;
  return CC_OK;
}

int cc_visibility_update(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                         const float* lights, uint32_t nlights, const uint8_t* stale, const cc_options* opt_in,
                         const cc_outputs* out, uint64_t* recomputed, void* stream_in) {
  if (!ctx || !scene || !out || (npoints && !receivers) || (nlights && !lights) || !stale)
    return fail(CC_ERR_INVALID, "null argument");
  if (out->partial || out->work) return fail(CC_ERR_INVALID, "an update writes full, any, irradiance and fraction only");
  if (scene->ctx != ctx) return fail(CC_ERR_INVALID, "scene belongs to another context (or to none)");
  cc_options opt;
  if (opt_in) opt = *opt_in; else cc_options_default(&opt);
  int rc = set_device(ctx);
  if (rc) return rc;
  cudaStream_t stream = stream_in ? (cudaStream_t)stream_in : ctx->stream;
  const uint64_t ncones = npoints * (uint64_t)nlights;
  if (ncones >= 0xffffffffull) return fail(CC_ERR_INVALID, "more than 2^32 - 1 cones in one call");
  if (recomputed) *recomputed = 0;
  if (ncones == 0) return CC_OK;
  // The stale cones of every light as one list, each light's in the walk
  // order (Morton order of the points), so one launch walks them all in
  // coherent packets and writes each result at its own cone.
  size_t sel_bytes = 0;
  cub::DeviceSelect::Flagged(nullptr, sel_bytes, (const uint32_t*)nullptr, (const uint8_t*)nullptr, (uint32_t*)nullptr,
                             (uint32_t*)nullptr, (int)ncones);
  const size_t sort_bytes = cc::walk_order_scratch_bytes(npoints);
  // Scratch kept in the context between frames.
  cudaError_t e = ctx->upd_perm.reserve(ncones * 4);
  if (e == cudaSuccess) e = ctx->upd_flags.reserve(ncones);
  if (e == cudaSuccess) e = ctx->upd_list.reserve(ncones * 4);
  if (e == cudaSuccess) e = ctx->upd_count.reserve(4);
  if (e == cudaSuccess) e = ctx->upd_order.reserve(npoints * 4);
  if (e == cudaSuccess) e = ctx->upd_temp.reserve(std::max<size_t>(std::max(sel_bytes, sort_bytes), 256));
  if (e != cudaSuccess) return cuda_fail(e, "update scratch");
  uint32_t* perm = static_cast<uint32_t*>(ctx->upd_perm.ptr);
  uint8_t* flags = static_cast<uint8_t*>(ctx->upd_flags.ptr);
  uint32_t* list = static_cast<uint32_t*>(ctx->upd_list.ptr);
  uint32_t* count = static_cast<uint32_t*>(ctx->upd_count.ptr);
  uint32_t* order = static_cast<uint32_t*>(ctx->upd_order.ptr);
  void* temp = ctx->upd_temp.ptr;
  const unsigned threads = 256;
  if (e == cudaSuccess) {
    if (npoints > 64 && !scene->flat.nodes.empty()) {
      e = cc::walk_order(reinterpret_cast<const float4*>(receivers), npoints, scene->flat.nodes[0].lo,
                         scene->flat.nodes[0].hi, temp, std::max(sel_bytes, sort_bytes), order, stream);
    } else {
      cc::iota_kernel<<<(unsigned)((npoints + threads - 1) / threads), threads, 0, stream>>>(order, npoints);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess)
    e = cc::stale_list(order, stale, npoints, nlights, perm, flags, list, count, temp, std::max(sel_bytes, sort_bytes),
                       stream);
  if (e == cudaSuccess) {
    cc_options lo = opt;
    lo.flags |= CC_DEVICE_POINTERS;
    cc_outputs o{};
    o.full = out->full;
    o.any = out->any;
    o.irradiance = out->irradiance;
    o.fraction = out->fraction;
    rc = cc_host::visibility_impl(ctx, scene, receivers, npoints, lights, nlights, &lo, &o, stream, 0u, list, count);
  }
  uint32_t n = 0;
  if (e == cudaSuccess && rc == CC_OK) e = cudaMemcpyAsync(&n, count, 4, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess && rc == CC_OK) e = cudaStreamSynchronize(stream);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "visibility update");
  if (recomputed) *recomputed = n;
  return CC_OK;
}
