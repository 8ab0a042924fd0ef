// Primary hits of a pinhole camera through a host-side scene: the shading
// points of per-pixel visibility, as the reference's camera pass finds them
// (camera_dir :1724-1729, primary_hit :1732-1760, the lifted hit point
// surface_offset :2062-2064 and per_pixel_hit_color :2275-2277 of
// crates/continuum-gpu/src/mask_cones.wgsl). Input preparation only: it runs
// on host threads over the same hierarchies the device walks.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "bvh.h"

namespace cc {
namespace {

struct V {
  float x, y, z;
};
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V normalize(V a) {
  float l = std::sqrt(dot(a, a));
  return {a.x / l, a.y / l, a.z / l};
}

// Slab test of a ray against a box, nearer than `limit`.
inline bool ray_box(V o, V inv, const NodeGpu& n, float limit) {
  float t0 = 0.0f, t1 = limit;
  const float* lo = n.lo;
  const float* hi = n.hi;
  const float oc[3] = {o.x, o.y, o.z}, ic[3] = {inv.x, inv.y, inv.z};
  for (int k = 0; k < 3; ++k) {
    float a = (lo[k] - oc[k]) * ic[k], b = (hi[k] - oc[k]) * ic[k];
    if (a > b) std::swap(a, b);
    t0 = std::max(t0, a);
    t1 = std::min(t1, b);
    if (t0 > t1) return false;
  }
  return true;
}

// Moller-Trumbore intersection; distance or -1.
inline float ray_tri(V o, V d, V v0, V v1, V v2) {
  V e1 = v1 - v0, e2 = v2 - v0;
  V p = cross(d, e2);
  float det = dot(e1, p);
  if (std::fabs(det) < 1e-12f) return -1.0f;
  float inv = 1.0f / det;
  V s = o - v0;
  float u = dot(s, p) * inv;
  if (u < 0.0f || u > 1.0f) return -1.0f;
  V q = cross(s, e1);
  float v = dot(d, q) * inv;
  if (v < 0.0f || u + v > 1.0f) return -1.0f;
  float t = dot(e2, q) * inv;
  return t > 0.0f ? t : -1.0f;
}

struct Hit {
  float t = FLT_MAX;
  uint32_t tri = kNone;
  uint32_t xform = kNone;  // the hit object's transform (instanced scenes)
  uint32_t object = kNone; // the hit mesh (object)
};

void trace(const FlatScene& s, V o, V d, Hit& hit) {
  V inv{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  uint32_t stack[128];
  uint32_t bstack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const NodeGpu& n = s.nodes[stack[--sp]];
    if (!ray_box(o, inv, n, hit.t)) continue;
    if (n.info[1] > 0) {
      for (uint32_t k = n.info[0]; k < n.info[0] + n.info[1]; ++k) {
        const uint32_t* r = &s.ranges[4 * s.items[k]];
        if (r[2] == kNone) continue;
        // A placed object: the ray in its space, o' = R^T (o - t) / s and
        // d' = R^T d / s, so distances along it stay the world's.
        V ob = o, db = d, ib = inv;
        if (r[3] != kNone) {
          const float* x = &s.xforms[16 * (size_t)r[3]];
          const V a{x[0], x[1], x[2]}, b{x[4], x[5], x[6]}, c{x[8], x[9], x[10]}, t{x[3], x[7], x[11]};
          const float is = x[13];
          const V q = o - t;
          ob = (a * q.x + b * q.y + c * q.z) * is;
          db = (a * d.x + b * d.y + c * d.z) * is;
          ib = V{1.0f / db.x, 1.0f / db.y, 1.0f / db.z};
        }
        int bp = 0;
        bstack[bp++] = r[2];
        while (bp > 0) {
          const NodeGpu& b = s.blas[bstack[--bp]];
          if (!ray_box(ob, ib, b, hit.t)) continue;
          if (b.info[1] > 0) {
            for (uint32_t j = b.info[0]; j < b.info[0] + b.info[1]; ++j) {
              uint32_t t = s.blas_items[j];
              const float* p = &s.tris[12 * (size_t)t];
              float dist = ray_tri(ob, db, V{p[0], p[1], p[2]}, V{p[4], p[5], p[6]}, V{p[8], p[9], p[10]});
              if (dist > 0.0f && dist < hit.t) {
                hit.t = dist;
                hit.tri = t;
                hit.xform = r[3];
                hit.object = s.items[k];
              }
            }
          } else if (bp + 2 <= 128) {
            bstack[bp++] = b.info[0];
            bstack[bp++] = b.info[0] + 1;
          }
        }
      }
    } else if (sp + 2 <= 128) {
      stack[sp++] = n.info[0];
      stack[sp++] = n.info[0] + 1;
    }
  }
}

}  // namespace

// camera: eye.xyz, target.xyz, up.xyz, vertical fov (degrees). Writes per
// pixel (row-major) a receiver (8 floats: point, hit object's index as bits;
// normal, hit triangle's index + 1 as bits) and 1 if the ray hit.
void primary_hits(const FlatScene& s, const float* camera, uint32_t width, uint32_t height, float* out8,
                  uint8_t* hit_mask, int threads) {
  V eye{camera[0], camera[1], camera[2]}, target{camera[3], camera[4], camera[5]}, upw{camera[6], camera[7], camera[8]};
  float tan_half = std::tan(camera[9] * 3.14159265358979f / 360.0f);
  V fwd = normalize(target - eye);
  V right = normalize(cross(fwd, upw));
  V up = cross(right, fwd);
  float aspect = float(width) / float(height);
  std::atomic<uint32_t> next{0};
  auto work = [&] {
    for (;;) {
      uint32_t row = next.fetch_add(1);
      if (row >= height) break;
      for (uint32_t x = 0; x < width; ++x) {
        float sx = ((float(x) + 0.5f) / float(width) * 2.0f - 1.0f) * tan_half * aspect;
        float sy = (1.0f - (float(row) + 0.5f) / float(height) * 2.0f) * tan_half;
        V d = normalize(fwd + right * sx + up * sy);
        Hit h;
        trace(s, eye, d, h);
        size_t i = (size_t)row * width + x;
        float* o = out8 + 8 * i;
        if (h.tri == kNone) {
          for (int k = 0; k < 8; ++k) o[k] = 0.0f;
          hit_mask[i] = 0;
          continue;
        }
        const float* p = &s.tris[12 * (size_t)h.tri];
        V v0{p[0], p[1], p[2]}, v1{p[4], p[5], p[6]}, v2{p[8], p[9], p[10]};
        V n = normalize(cross(v1 - v0, v2 - v0));
        if (h.xform != kNone) {  // the object's normal in world space: R n
          const float* x = &s.xforms[16 * (size_t)h.xform];
          n = normalize(V{x[0] * n.x + x[1] * n.y + x[2] * n.z, x[4] * n.x + x[5] * n.y + x[6] * n.z,
                          x[8] * n.x + x[9] * n.y + x[10] * n.z});
        }
        if (dot(n, d) > 0.0f) n = n * -1.0f;
        V surface = eye + d * h.t;
        V point = surface + n * std::max(1e-4f, 2e-6f * h.t);
        // w: the hit object (point) and the hit triangle + 1 (normal), as
        // bits: CC_SKY_OBJECT_FRAME's object and CC_BACK_FACING's own triangle.
        const uint32_t own = h.tri + 1u;
        o[0] = point.x;
        o[1] = point.y;
        o[2] = point.z;
        std::memcpy(&o[3], &h.object, 4);
        o[4] = n.x;
        o[5] = n.y;
        o[6] = n.z;
        std::memcpy(&o[7], &own, 4);
        hit_mask[i] = 1;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < std::max(threads, 1); ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

}  // namespace cc
