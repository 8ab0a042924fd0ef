// Device-side cone geometry for the mask-cone visibility kernels (sm_100a).
//
// One lane owns one cone. The geometry follows the reference's WGSL light-cone
// path (crates/continuum-gpu/src/mask_cones.wgsl, cited per function); the
// per-cone state that the WGSL keeps in private arrays (64 coverages, the
// 68-cell accumulator) lives here in shared memory, lane-interleaved
// (cell * 32 + lane), so every access is bank-conflict-free whatever cell
// each lane touches.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cc {

constexpr int kGrid = 8;
constexpr int kBins = 64;
constexpr uint32_t kNoneU = 0xffffffffu;
constexpr float kNear = 1e-4f;  // NEAR, mask_cones.wgsl:213

// ---- small vector helpers -------------------------------------------------
struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float len(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 div(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
// Out of line (like the integration helpers below): the kernel is limited by
// instruction fetch, and inline copies of the division and square root at
// every call site cost more than the calls.
static __device__ __noinline__ f3 normalize(f3 a) { return div(a, len(a)); }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// ---- device scene and query -------------------------------------------------
// Nodes are two float4: (lo.xyz, a) and (hi.xyz, b) with a, b as bits:
// leaf: a = first item, b = item count; interior: a = left child, b = 0.
struct DevScene {
  const float4* tris;      // 3 per triangle (w unused), in triangle-hierarchy leaf order
  const uint4* meshes;     // first, count, blas root, transform
  const float4* nodes;     // object hierarchy, 2 per node
  const uint32_t* items;   // mesh per object leaf slot
  const float4* blas;      // triangle hierarchies, 2 per node; leaf items are triangle slots
  uint32_t nmeshes;
  // Instanced scenes: 4 per transform (rows 0-2 of the rotation with the
  // translation in w, then scale, 1 / scale); meshes[m].w names object m's.
  // Null when every object's triangles are in world space.
  const float4* xforms;
  // Prefiltered cones: 27 coverage samples per triangle-hierarchy node and
  // per object-hierarchy node (an object node's sample 13, unused as a
  // direction, is 1 where the node has no prefiltered coverage); null where
  // the scene has none on the device.
  const float* blas_cov;
  const float* obj_cov;
};

struct DevLight {
  f3 corner;
  float kind;  // corner.w: 0 two-sided rect, 1 one-sided rect, 2 sphere
  f3 eu;
  f3 ev;
  float evw;   // spot on (sphere)
};

__device__ __forceinline__ DevLight load_light(const float4* lights, uint32_t l) {
  float4 a = __ldg(&lights[4 * l + 0]);
  float4 b = __ldg(&lights[4 * l + 1]);
  float4 c = __ldg(&lights[4 * l + 2]);
  DevLight L;
  L.corner = xyz(a);
  L.kind = a.w;
  L.eu = xyz(b);
  L.ev = xyz(c);
  L.evw = c.w;
  return L;
}

__device__ __forceinline__ bool is_sphere(const DevLight& r) { return r.kind > 1.5f; }

// ---- the cone ----------------------------------------------------------------
// mask_cones.wgsl:136-155. The far plane's normal is the cone's forward axis
// for every light cone (:924, :1034), so only its offset is kept; light
// cones have no horizon.
struct Cone {
  f3 apex, right, up, fwd;
  float u0, v0, u1, v1;
  float far_offset;
  f3 baxis;
  float bcos, bsin;
};

// cone_to_object (:623-638): the cone in the space of the object placed by
// transform X (world = scale * rotation * p + translation): the apex moved and
// scaled, the frame and the bounding axis rotated (rotate_to_object, :61-63),
// the far plane moved; the window is a set of directions, which a rotation
// and a uniform scale keep.
__device__ __forceinline__ Cone cone_to_object(const Cone& c, const float4* __restrict__ X) {
  const float4 r0 = __ldg(X), r1 = __ldg(X + 1), r2 = __ldg(X + 2), r3 = __ldg(X + 3);
  const f3 a = {r0.x, r0.y, r0.z}, b = {r1.x, r1.y, r1.z}, d = {r2.x, r2.y, r2.z};
  auto rot = [&](f3 v) { return a * v.x + b * v.y + d * v.z; };
  const f3 t = {r0.w, r1.w, r2.w};
  Cone o;
  o.apex = rot(c.apex - t) * r3.y;
  o.right = rot(c.right);
  o.up = rot(c.up);
  o.fwd = rot(c.fwd);
  o.u0 = c.u0;
  o.v0 = c.v0;
  o.u1 = c.u1;
  o.v1 = c.v1;
  o.far_offset = (c.far_offset - dot(c.fwd, t)) * r3.y;  // the far plane's normal is the forward axis
  o.baxis = rot(c.baxis);
  o.bcos = c.bcos;
  o.bsin = c.bsin;
  return o;
}

__device__ __forceinline__ f3 direction(const Cone& c, float s, float t) {  // :203-206
  return c.fwd + c.right * (c.u0 + s * (c.u1 - c.u0)) + c.up * (c.v0 + t * (c.v1 - c.v0));
}

__device__ __forceinline__ f3 to_local(const Cone& c, f3 p) {  // :208-211
  f3 d = p - c.apex;
  return {dot(c.right, d), dot(c.up, d), dot(c.fwd, d)};
}

__device__ __forceinline__ bool in_bound(const Cone& c, f3 p, float r) {  // :159-168
  if (c.bcos < -1.0f) return true;
  f3 d = p - c.apex;
  float l = len(d);
  if (l <= r) return true;
  float s = r / l;
  float limit = c.bcos * sqrtf(1.0f - s * s) - c.bsin * s;
  return dot(c.baxis, d) >= limit * l;
}

__device__ __forceinline__ void bound_cone(Cone& c, f3 axis) {  // :174-186
  float cos_half = 1.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f3 d = normalize(direction(c, float(k & 1), float(k >> 1)));
    cos_half = fminf(cos_half, dot(axis, d));
  }
  float cb = clampf(cos_half - 1e-5f, -1.0f, 1.0f);
  c.baxis = axis;
  c.bcos = cb;
  c.bsin = sqrtf(fmaxf(1.0f - cb * cb, 0.0f));
}

struct LightConeInfo {
  bool ok;
  bool wide_clipped;
  bool wide_window;
};

// light_cone_sphere (:902-931)
__device__ __forceinline__ LightConeInfo light_cone_sphere(f3 apex, const DevLight& r, float wide_extent, Cone& c) {
  LightConeInfo info{false, false, false};
  f3 to_center = r.corner - apex;
  float d = len(to_center);
  float radius = r.eu.x;
  if (d <= radius * 1.0001f) return info;
  f3 fwd = div(to_center, d);
  float s = radius / d;
  float t = s / sqrtf(fmaxf(1.0f - s * s, 1e-12f));
  info.wide_clipped = 2.0f * t > wide_extent;
  info.wide_window = info.wide_clipped;
  t = fminf(t, 0.5f * wide_extent);
  f3 helper = fabsf(fwd.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
  f3 right = normalize(cross(helper, fwd));
  c.apex = apex;
  c.right = right;
  c.up = cross(fwd, right);
  c.fwd = fwd;
  c.u0 = -t;
  c.v0 = -t;
  c.u1 = t;
  c.v1 = t;
  c.far_offset = dot(fwd, apex) + (d - radius * s) * (1.0f - 1e-5f);
  bound_cone(c, fwd);
  info.ok = true;
  return info;
}

// light_cone_rect (:974-1042)
__device__ __forceinline__ LightConeInfo light_cone(f3 apex, const DevLight& r, float wide_extent, Cone& c) {
  if (is_sphere(r)) return light_cone_sphere(apex, r, wide_extent, c);
  LightConeInfo info{false, false, false};
  f3 fwd = normalize(cross(r.eu, r.ev));
  if (r.kind > 0.5f && dot(fwd, apex - r.corner) <= 0.0f) return info;
  if (dot(fwd, r.corner - apex) < 0.0f) fwd = -fwd;
  float dist = dot(fwd, r.corner - apex);
  if (dist <= 1e-6f) return info;
  f3 right = normalize(r.eu);
  f3 up = cross(fwd, right);
  f3 rel = r.corner - apex;
  float lo0 = 3.4e38f, lo1 = 3.4e38f, hi0 = -3.4e38f, hi1 = -3.4e38f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f3 corner = rel + r.eu * float(k & 1) + r.ev * float((k >> 1) & 1);
    float u = dot(right, corner) / dist, v = dot(up, corner) / dist;
    lo0 = fminf(lo0, u);
    lo1 = fminf(lo1, v);
    hi0 = fmaxf(hi0, u);
    hi1 = fmaxf(hi1, v);
  }
  float ext0 = hi0 - lo0, ext1 = hi1 - lo1;
  float foot0 = fminf(fmaxf(0.0f, lo0), hi0), foot1 = fminf(fmaxf(0.0f, lo1), hi1);
  f3 mid = normalize(mk(0.5f * (lo0 + hi0), 0.5f * (lo1 + hi1), 1.0f));
  float cos_wide = 1.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f3 q = mk((k & 1) ? hi0 : lo0, (k & 2) ? hi1 : lo1, 1.0f);
    cos_wide = fminf(cos_wide, dot(mid, normalize(q)));
  }
  const float size = wide_extent;
  info.wide_window = ext0 > size || ext1 > size;
  info.wide_clipped = info.wide_window && cos_wide < 0.8660254f;
  if (info.wide_clipped) {
    if (ext0 > size) {
      float keep = fminf(fmaxf(foot0 - 0.5f * size, lo0), hi0 - size);
      lo0 = keep;
      hi0 = keep + size;
    }
    if (ext1 > size) {
      float keep = fminf(fmaxf(foot1 - 0.5f * size, lo1), hi1 - size);
      lo1 = keep;
      hi1 = keep + size;
    }
  }
  c.apex = apex;
  c.right = right;
  c.up = up;
  c.fwd = fwd;
  c.u0 = lo0;
  c.v0 = lo1;
  c.u1 = hi0;
  c.v1 = hi1;
  c.far_offset = dot(fwd, apex) + dist * (1.0f - 1e-5f);
  f3 axis = normalize(rel + (r.eu + r.ev) * 0.5f);
  if (info.wide_clipped) axis = normalize(direction(c, 0.5f, 0.5f));
  bound_cone(c, axis);
  info.ok = true;
  return info;
}

// ---- culling ---------------------------------------------------------------
// rotate_to_object (:61-63): a direction in the space of the object placed by
// transform X.
__device__ __forceinline__ f3 rotate_to_object(f3 v, const float4* __restrict__ X) {
  const float4 r0 = __ldg(X), r1 = __ldg(X + 1), r2 = __ldg(X + 2);
  return mk(r0.x, r0.y, r0.z) * v.x + mk(r1.x, r1.y, r1.z) * v.y + mk(r2.x, r2.y, r2.z) * v.z;
}

// may_touch_box (:234-255), which is node_cone_test (:519-574) for exact cones.
// kHorizon: sky cones, whose horizon `horizon` (the receiver's normal, in the
// cone's space) also culls a box wholly below it (:245); a light cone's
// horizon is zero (:146-147), which culls nothing, so light cones skip it.
// kUnrolled: the eight corners side by side (the walk's hot test of a node's
// children); else one at a time, in a fifth of the code (the tests of a
// walk's root and of meshes' roots, which run far less often).
template <bool kHorizon = false, bool kUnrolled = true>
__device__ __forceinline__ bool may_touch_box(const Cone& c, f3 lo, f3 hi, f3 horizon = f3{0.f, 0.f, 0.f}) {
  bool far_out = true, near_out = true, out_u0 = true, out_u1 = true, out_v0 = true, out_v1 = true, below = kHorizon;
#pragma unroll (kUnrolled ? 8 : 1)
  for (int k = 0; k < 8; ++k) {
    f3 corner = mk((k & 1) ? hi.x : lo.x, (k & 2) ? hi.y : lo.y, (k & 4) ? hi.z : lo.z);
    if (c.far_offset - dot(c.fwd, corner) >= 0.0f) far_out = false;
    if constexpr (kHorizon) {
      if (dot(horizon, corner - c.apex) >= 0.0f) below = false;
    }
    f3 p = to_local(c, corner);
    if (p.z >= kNear) near_out = false;
    if (p.x - c.u0 * p.z >= 0.0f) out_u0 = false;
    if (c.u1 * p.z - p.x >= 0.0f) out_u1 = false;
    if (p.y - c.v0 * p.z >= 0.0f) out_v0 = false;
    if (c.v1 * p.z - p.y >= 0.0f) out_v1 = false;
  }
  if (far_out || near_out || out_u0 || out_u1 || out_v0 || out_v1 || below) return false;
  return in_bound(c, (lo + hi) * 0.5f, 0.5f * len(hi - lo));
}

// may_touch (:215-232); kHorizon as in may_touch_box (:220-221).
template <bool kHorizon = false>
__device__ __forceinline__ bool may_touch(const Cone& c, f3 v0, f3 v1, f3 v2, f3 horizon = f3{0.f, 0.f, 0.f}) {
  float f0 = c.far_offset - dot(c.fwd, v0);
  float f1 = c.far_offset - dot(c.fwd, v1);
  float f2 = c.far_offset - dot(c.fwd, v2);
  if (f0 < 0.0f && f1 < 0.0f && f2 < 0.0f) return false;
  if constexpr (kHorizon) {
    if (dot(horizon, v0 - c.apex) < 0.0f && dot(horizon, v1 - c.apex) < 0.0f && dot(horizon, v2 - c.apex) < 0.0f)
      return false;
  }
  f3 p0 = to_local(c, v0), p1 = to_local(c, v1), p2 = to_local(c, v2);
  if (p0.z < kNear && p1.z < kNear && p2.z < kNear) return false;
  if (p0.x - c.u0 * p0.z < 0.0f && p1.x - c.u0 * p1.z < 0.0f && p2.x - c.u0 * p2.z < 0.0f) return false;
  if (c.u1 * p0.z - p0.x < 0.0f && c.u1 * p1.z - p1.x < 0.0f && c.u1 * p2.z - p2.x < 0.0f) return false;
  if (p0.y - c.v0 * p0.z < 0.0f && p1.y - c.v0 * p1.z < 0.0f && p2.y - c.v0 * p2.z < 0.0f) return false;
  if (c.v1 * p0.z - p0.y < 0.0f && c.v1 * p1.z - p1.y < 0.0f && c.v1 * p2.z - p2.y < 0.0f) return false;
  return true;
}

// ---- the accumulation rasterizer ------------------------------------------------
// A cone's 68-cell accumulator (the WGSL's `acc`, :719-760) in shared
// memory, cell-major with the cone's lane innermost, in fixed point (units of
// 2^-24 of a bin: an f32's resolution at 1). Any lane may add to any cone's
// cells: integer addition is exact and order-free, so the sum — and every
// result — is the same whichever lanes draw which triangles in whatever
// order. (The reference sums in f32 in walk order; the exact sum differs from
// that by f32 rounding only.) The packet pass keeps 32-bit cells, so more
// warps fit an SM; an add that overflows one (a mesh piling 128 bins' worth
// of coverage into a cell) flags its cone, which the solo pass walks again
// with 64-bit cells of the same unit — the same result, never a wrapped one.
// Cells 64..65 receive writes "one past the last row" that no resolve ever
// reads, so they are dropped.
constexpr float kFixScale = 16777216.0f;        // 2^24
constexpr float kFixUnit = 1.0f / 16777216.0f;  // 2^-24

template <class Cell>
struct LaneAcc;

// 64-bit cells: no overflow is possible (each add is at most one bin).
template <>
struct LaneAcc<unsigned long long> {
  unsigned long long* base;  // &acc[cone]; cell k at base[32 * k]
  uint32_t span_lo, span_hi; // rows this triangle wrote (the WGSL's span, :758-760)
  uint32_t* overflow;        // unused
  uint32_t bit;
  __device__ __forceinline__ void add(uint32_t cell, float v) {
    if (cell < (uint32_t)kBins) atomicAdd(base + 32 * cell, (unsigned long long)__float2ll_rn(v * kFixScale));
  }
};

// 32-bit cells: a signed overflow of any add sets the cone's bit in *overflow.
template <>
struct LaneAcc<unsigned int> {
  unsigned int* base;
  uint32_t span_lo, span_hi;
  uint32_t* overflow;
  uint32_t bit;
  __device__ __forceinline__ void add(uint32_t cell, float v) {
    if (cell < (uint32_t)kBins) {
      const int a = __float2int_rn(v * kFixScale);
      const int old = (int)atomicAdd(base + 32 * cell, (unsigned int)a);
      const int sum = (int)((unsigned int)old + (unsigned int)a);
      if (((old ^ sum) & (a ^ sum)) < 0) atomicOr(overflow, bit);
    }
  }
};

// draw_edge (:297-348)
template <class Acc>
__device__ __forceinline__ void draw_edge(Acc& acc, float q0x, float q0y, float q1x, float q1y, float weight) {
  if (fabsf(q0y - q1y) <= 1.1920929e-7f) return;
  float dir = 1.0f;
  float p0x = q0x, p0y = q0y, p1x = q1x, p1y = q1y;
  if (q0y > q1y) {
    dir = -1.0f;
    p0x = q1x;
    p0y = q1y;
    p1x = q0x;
    p1y = q0y;
  }
  const float dxdy = (p1x - p0x) / (p1y - p0y);
  float x = p0x;
  const uint32_t y_end = min((uint32_t)ceilf(p1y), (uint32_t)kGrid);
#pragma unroll 1
  for (uint32_t y = (uint32_t)p0y; y < y_end; ++y) {
    const uint32_t row = y * kGrid;
    acc.span_lo = min(acc.span_lo, row);
    acc.span_hi = max(acc.span_hi, row + kGrid + 1);
    float dy = fminf(float(y + 1), p1y) - fmaxf(float(y), p0y);
    float x_next = clampf(x + dxdy * dy, 0.0f, float(kGrid));
    float d = dy * dir * weight;
    float x0 = fminf(x, x_next), x1 = fmaxf(x, x_next);
    float x0_floor = floorf(x0);
    uint32_t x0i = (uint32_t)x0_floor;
    float x1_ceil = ceilf(x1);
    uint32_t x1i = (uint32_t)x1_ceil;
    // The row's cells x0i .. last and their shares (the WGSL's cases), all
    // added from one site.
    const bool narrow = x1i <= x0i + 1;
    const float xmf = 0.5f * (x + x_next) - x0_floor;
    float s = 0.f, a0 = 0.f, am = 0.f, a1 = 0.f, a2 = 0.f;
    if (!narrow) {
      s = 1.0f / (x1 - x0);
      const float x0f = x0 - x0_floor;
      a0 = 0.5f * s * (1.0f - x0f) * (1.0f - x0f);
      const float x1f = x1 - x1_ceil + 1.0f;
      am = 0.5f * s * x1f * x1f;
      a1 = s * (1.5f - x0f);
      a2 = a1 + float(x1i - x0i - 3) * s;
    }
    const uint32_t last = narrow ? x0i + 1 : x1i;
#pragma unroll 1
    for (uint32_t xi = x0i; xi <= last; ++xi) {
      float v;
      if (narrow) v = xi == x0i ? d - d * xmf : d * xmf;
      else if (xi == x0i) v = d * a0;
      else if (xi == x1i) v = d * am;
      else if (x1i == x0i + 2) v = d * (1.0f - a0 - am);
      else if (xi == x0i + 1) v = d * (a1 - a0);
      else if (xi == x1i - 1) v = d * (1.0f - a2 - am);
      else v = d * s;
      acc.add(row + xi, v);
    }
    x = x_next;
  }
}

// Polygons of the general clip path. The WGSL holds 10 vertices
// (mask_cones.wgsl:11); a triangle clipped by the far and near planes has
// at most 5, the window square clipped by 5 edge planes at most 9, and four
// rounding-dust clips at the square's sides can add one each, so 16 holds
// every case.
constexpr int kPolyCap = 16;

// clip_plane3 (:264-277), in place through a scratch copy.
__device__ __forceinline__ int clip_plane3(const f3* in, int n, f3* out, f3 normal, float offset) {
  int m = 0;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    f3 a = in[i], b = in[i + 1 == n ? 0 : i + 1];
    float da = offset - dot(normal, a), db = offset - dot(normal, b);
    if (da >= 0.0f && m < kPolyCap) out[m++] = a;
    // The crossing, from the vertex inside (a, leaving) or outside (b,
    // entering): one division site for both.
    const bool leaves = da >= 0.0f && db < 0.0f, enters = da < 0.0f && db >= 0.0f;
    if ((leaves || enters) && m < kPolyCap) {
      const f3 from = leaves ? a : b, to = leaves ? b : a;
      const float d_from = leaves ? da : db, d_to = leaves ? db : da;
      out[m++] = from + (to - from) * (d_from / (d_from - d_to));
    }
  }
  return m;
}

// clip_line2 (:280-294)
__device__ __forceinline__ int clip_line2(const float2* in, int n, float2* out, float nx, float ny, float offset) {
  int m = 0;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    float2 a = in[i], b = in[i + 1 == n ? 0 : i + 1];
    float da = offset - (nx * a.x + ny * a.y);
    float db = offset - (nx * b.x + ny * b.y);
    if (da >= 0.0f && m < kPolyCap) out[m++] = a;
    const bool leaves = da >= 0.0f && db < 0.0f, enters = da < 0.0f && db >= 0.0f;
    if ((leaves || enters) && m < kPolyCap) {
      const float2 from = leaves ? a : b, to = leaves ? b : a;
      const float d_from = leaves ? da : db, d_to = leaves ? db : da;
      const float f = d_from / (d_from - d_to);
      out[m++] = make_float2(from.x + (to.x - from.x) * f, from.y + (to.y - from.y) * f);
    }
  }
  return m;
}

template <class Acc>
__device__ __forceinline__ void draw_polygon(Acc& acc, const float2* q, int n, float weight) {
  const float g = float(kGrid);
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    float2 a = q[i], b = q[i + 1 == n ? 0 : i + 1];
    draw_edge(acc, clampf(a.x, 0.f, g), clampf(a.y, 0.f, g), clampf(b.x, 0.f, g), clampf(b.y, 0.f, g), weight);
  }
}

// The clipped polygon in bin space, drawn (general path of rasterize,
// :350-451): far and near clips, then either the projected corners or, for a
// polygon reaching outside the window, the window square clipped to the
// planes through the apex and each edge; finally the square's sides.
// Every loop here stays rolled and each clip has one call site: the walk
// kernel is bound by instruction fetch, and the unrolled path (1,832
// instructions against 1,069) made the packet pass 13 % slower.
// kWeighted: the triangle is drawn with `weight` (tri_weight: a blended or
// transmissive object's); else whole.
template <class Acc, bool kWeighted = false>
static __device__ __noinline__ bool rasterize_general(const Cone& c, Acc& acc, f3 v0, f3 v1, f3 v2, bool far_clip,
                                                      float weight = 1.0f) {
  f3 pa[kPolyCap], pb[kPolyCap];
  pa[0] = v0;
  pa[1] = v1;
  pa[2] = v2;
  int n = 3;
  f3* p = pa;
  f3* other = pb;
  // Pass 0: the far clip (world space), then the corners in the cone's
  // frame; pass 1: the near clip there. One clip call site for both.
  bool all_near_ok = true, all_in_window = true;
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 0 ? far_clip : !all_near_ok) {
      n = clip_plane3(p, n, other, pass == 0 ? c.fwd : mk(0.f, 0.f, -1.f), pass == 0 ? c.far_offset : -kNear);
      f3* t = p;
      p = other;
      other = t;
    }
    if (pass == 1) break;
#pragma unroll 1
    for (int i = 0; i < n; ++i) {
      f3 v = to_local(c, p[i]);
      p[i] = v;
      if (v.z < kNear) all_near_ok = false;
      if (v.x < c.u0 * v.z || v.x > c.u1 * v.z || v.y < c.v0 * v.z || v.y > c.v1 * v.z) all_in_window = false;
    }
  }
  if (n < 3) return false;
  const float su = float(kGrid) / (c.u1 - c.u0);
  const float sv = float(kGrid) / (c.v1 - c.v0);
  const float g = float(kGrid);
  float2 qa[kPolyCap], qb[kPolyCap];
  float2* q = qa;
  float2* q2 = qb;
  int m;
  const bool projected = all_near_ok && all_in_window;
  float side = 1.0f;
  if (projected) {
    m = n;
#pragma unroll 1
    for (int i = 0; i < n; ++i) q[i] = make_float2((p[i].x / p[i].z - c.u0) * su, (p[i].y / p[i].z - c.v0) * sv);
  } else {
    f3 l0 = to_local(c, v0), l1 = to_local(c, v1), l2 = to_local(c, v2);
    float d = dot(l0, cross(l1, l2));
    if (d == 0.0f) return false;
    side = d > 0.0f ? 1.0f : -1.0f;
    m = 4;
    q[0] = make_float2(0.f, 0.f);
    q[2] = make_float2(g, g);
    if (side > 0.0f) {
      q[1] = make_float2(g, 0.f);
      q[3] = make_float2(0.f, g);
    } else {
      q[1] = make_float2(0.f, g);
      q[3] = make_float2(g, 0.f);
    }
  }
  // Every 2D clip from one call site: first the planes through the apex and
  // each edge (the apex-plane case), then, if some vertex lies outside the
  // grid, the square's four sides — the reference's sequence of clips.
  int stage = projected ? 1 : 0;  // 0: edge planes, 1: the inside check, 2: the square's sides
  int i = 0;
#pragma unroll 1
  for (;;) {
    float nx, ny, off;
    if (stage == 0) {
      if (i == n) {
        stage = 1;
        continue;
      }
      const f3 e = cross(p[i], p[i + 1 == n ? 0 : i + 1]);
      ++i;
      const float l = len(e);
      if (l == 0.0f) continue;
      const f3 k = e * (side / l);
      nx = -k.x / su;
      ny = -k.y / sv;
      off = k.x * c.u0 + k.y * c.v0 + k.z;
    } else if (stage == 1) {
      bool inside = true;
#pragma unroll 1
      for (int j = 0; j < m; ++j)
        if (q[j].x < 0.f || q[j].y < 0.f || q[j].x > g || q[j].y > g) inside = false;
      if (inside) break;
      stage = 2;
      i = 0;
      continue;
    } else {
      if (i == 4) break;
      nx = i == 0 ? -1.f : (i == 1 ? 1.f : 0.f);
      ny = i == 2 ? -1.f : (i == 3 ? 1.f : 0.f);
      off = (i & 1) ? g : 0.f;
      ++i;
    }
    m = clip_line2(q, m, q2, nx, ny, off);
    float2* t = q;
    q = q2;
    q2 = t;
  }
  if (m < 3) return false;
  draw_polygon(acc, q, m, kWeighted ? weight : 1.0f);
  return true;
}

// Whether the triangle reaches past the far plane (rasterize's far clip, :356-362).
__device__ __forceinline__ bool crosses_far(const Cone& c, f3 v0, f3 v1, f3 v2) {
  const float f0 = c.far_offset - dot(c.fwd, v0);
  const float f1 = c.far_offset - dot(c.fwd, v1);
  const float f2 = c.far_offset - dot(c.fwd, v2);
  return f0 < 0.0f || f1 < 0.0f || f2 < 0.0f;
}

// rasterize (:350-451), its common case: a triangle wholly inside the window
// between the near and far planes projects its three corners and draws them
// from registers. Returns false, having drawn nothing, for every other
// triangle: those take rasterize_general.
template <class Acc>
__device__ __forceinline__ bool rasterize_fast(const Cone& c, Acc& acc, f3 v0, f3 v1, f3 v2, float weight = 1.0f) {
  if (!crosses_far(c, v0, v1, v2)) {
    f3 p0 = to_local(c, v0), p1 = to_local(c, v1), p2 = to_local(c, v2);
    auto in_win = [&](f3 v) {
      return v.z >= kNear && !(v.x < c.u0 * v.z || v.x > c.u1 * v.z || v.y < c.v0 * v.z || v.y > c.v1 * v.z);
    };
    if (in_win(p0) && in_win(p1) && in_win(p2)) {
      const float su = float(kGrid) / (c.u1 - c.u0);
      const float sv = float(kGrid) / (c.v1 - c.v0);
      const float g = float(kGrid);
      // The corners projected in turn (one site for each division).
      float ax = 0.f, ay = 0.f, bx = 0.f, by = 0.f, cx = 0.f, cy = 0.f;
      f3 pk = p0;
#pragma unroll 1
      for (int k = 0; k < 3; ++k) {
        ax = bx;
        ay = by;
        bx = cx;
        by = cy;
        cx = (pk.x / pk.z - c.u0) * su;
        cy = (pk.y / pk.z - c.v0) * sv;
        pk = k == 0 ? p1 : p2;
      }
      bool inside = ax >= 0.f && ay >= 0.f && ax <= g && ay <= g && bx >= 0.f && by >= 0.f && bx <= g &&
                    by <= g && cx >= 0.f && cy >= 0.f && cx <= g && cy <= g;
      if (inside) {
        // The three edges from one call site (a rolled loop keeps the hot
        // code small enough for the instruction caches).
#pragma unroll 1
        for (int e = 0; e < 3; ++e) {
          const float sx = e == 0 ? ax : (e == 1 ? bx : cx), sy = e == 0 ? ay : (e == 1 ? by : cy);
          const float tx = e == 0 ? bx : (e == 1 ? cx : ax), ty = e == 0 ? by : (e == 1 ? cy : ay);
          draw_edge(acc, sx, sy, tx, ty, weight);
        }
        return true;
      }
    }
  }
  return false;
}

// rasterize (:350-451): the common case, else the general path.
template <class Acc>
__device__ __forceinline__ bool rasterize(const Cone& c, Acc& acc, f3 v0, f3 v1, f3 v2) {
  if (rasterize_fast(c, acc, v0, v1, v2)) return true;
  return rasterize_general(c, acc, v0, v1, v2, crosses_far(c, v0, v1, v2));
}

// ---- integration --------------------------------------------------------------
// lambert_edge_unit / lambert_edge (:188-201). Out of line: an inline copy
// of atan2f at each of its many call sites made up a quarter of the kernel.
static __device__ __noinline__ float lambert_edge_unit(f3 n, f3 an, f3 bn) {
  f3 g = cross(an, bn);
  float l = len(g);
  if (l > 1e-12f) return atan2f(l, dot(an, bn)) * dot(n, div(g, l));
  return 0.0f;
}
__device__ __forceinline__ float lambert_edge(f3 n, f3 a, f3 b) { return lambert_edge_unit(n, normalize(a), normalize(b)); }

// The quad d[0..4] clipped to dot(n, x) >= 0 and Lambert-integrated
// (clipped_bin_weight / clipped_window_weight, :1331-1403; rect_open :2177-2199).
static __device__ __noinline__ float clipped_quad_weight(f3 n, f3 d0, f3 d1, f3 d2, f3 d3) {
  f3 d[4] = {d0, d1, d2, d3};
  f3 poly[6];
  int k_n = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f3 a = d[k], e = d[(k + 1) & 3];
    float sa = dot(n, a), se = dot(n, e);
    if (sa >= 0.0f) poly[k_n++] = a;
    if ((sa >= 0.0f) != (se >= 0.0f)) poly[k_n++] = a + (e - a) * (sa / (sa - se));
  }
  if (k_n < 3) return 0.0f;
  float sum = 0.0f;
  for (int k = 0; k < k_n; ++k) sum += lambert_edge(n, poly[k], poly[(k + 1) % k_n]);
  return fabsf(0.5f * sum);
}

// bin_weight (:1232-1242)
__device__ __forceinline__ float bin_weight(const Cone& c, f3 n, int b) {
  const float g = float(kGrid);
  float col = float(b % kGrid), row = float(b / kGrid);
  f3 d0 = direction(c, col / g, row / g);
  f3 d1 = direction(c, (col + 1.f) / g, row / g);
  f3 d2 = direction(c, (col + 1.f) / g, (row + 1.f) / g);
  f3 d3 = direction(c, col / g, (row + 1.f) / g);
  return fabsf(0.5f * (lambert_edge(n, d0, d1) + lambert_edge(n, d1, d2) + lambert_edge(n, d2, d3) +
                       lambert_edge(n, d3, d0)));
}

__device__ __forceinline__ float clipped_bin_weight(const Cone& c, f3 n, int b) {  // :1331-1369
  const float g = float(kGrid);
  float col = float(b % kGrid), row = float(b / kGrid);
  f3 d0 = direction(c, col / g, row / g);
  f3 d1 = direction(c, (col + 1.f) / g, row / g);
  f3 d2 = direction(c, (col + 1.f) / g, (row + 1.f) / g);
  f3 d3 = direction(c, col / g, (row + 1.f) / g);
  int above = (dot(n, d0) > 0.f) + (dot(n, d1) > 0.f) + (dot(n, d2) > 0.f) + (dot(n, d3) > 0.f);
  if (above == 4) return bin_weight(c, n, b);
  if (above == 0) return 0.0f;
  return clipped_quad_weight(n, d0, d1, d2, d3);
}

__device__ __forceinline__ float window_weight(const Cone& c, f3 n, bool* all_above) {
  f3 d00 = direction(c, 0.f, 0.f), d10 = direction(c, 1.f, 0.f);
  f3 d11 = direction(c, 1.f, 1.f), d01 = direction(c, 0.f, 1.f);
  *all_above = dot(n, d00) > 0.f && dot(n, d10) > 0.f && dot(n, d11) > 0.f && dot(n, d01) > 0.f;
  if (*all_above)
    return fabsf(0.5f * (lambert_edge(n, d00, d10) + lambert_edge(n, d10, d11) + lambert_edge(n, d11, d01) +
                         lambert_edge(n, d01, d00)));
  return clipped_quad_weight(n, d00, d10, d11, d01);
}

// ---- sky cones (:1323-1511) --------------------------------------------------------
// Far enough that every scene lies inside a sky cone (SKY_FAR, :1326).
constexpr float kSkyFar = 1e7f;

// clipped_window_weight (:1375-1403): the window's quad of directions clipped
// to the horizon of `n`, Lambert-integrated.
__device__ __forceinline__ float clipped_window_weight(const Cone& c, f3 n) {
  return clipped_quad_weight(n, direction(c, 0.f, 0.f), direction(c, 1.f, 0.f), direction(c, 1.f, 1.f),
                             direction(c, 0.f, 1.f));
}

// rotate_to_world (:65-67): a direction of the space of the object placed by
// transform X, in world space.
__device__ __forceinline__ f3 rotate_to_world(f3 d, const float4* __restrict__ X) {
  const float4 r0 = __ldg(X), r1 = __ldg(X + 1), r2 = __ldg(X + 2);
  return mk(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z,
            r2.x * d.x + r2.y * d.y + r2.z * d.z);
}

// sky_face (:1444-1478): cube face f (axis f / 2, negative for odd f) around
// `apex`, reaching kSkyFar past it (its horizon, the receiver's normal or
// zero, is the caller's), in world axes or, with `frame` (the transform of
// the object the receiver lies on: the reference's sky_frame, :1432-1456),
// in that object's axes turned to world space. Returns whether any of its
// directions lies above the horizon of `normal`.
__device__ __forceinline__ bool sky_face(uint32_t f, f3 apex, f3 normal, Cone& c,
                                         const float4* __restrict__ frame = nullptr) {
  const uint32_t axis = f / 2u;
  const float sign = (f & 1u) ? -1.0f : 1.0f;
  f3 forward = mk(0.f, 0.f, 0.f), right = mk(0.f, 0.f, 0.f);
  if (axis == 0u) forward.x = sign; else if (axis == 1u) forward.y = sign; else forward.z = sign;
  const uint32_t r = (axis + 1u) % 3u;
  if (r == 0u) right.x = 1.0f; else if (r == 1u) right.y = 1.0f; else right.z = 1.0f;
  if (frame) {
    forward = rotate_to_world(forward, frame);
    right = rotate_to_world(right, frame);
  }
  c.apex = apex;
  c.right = right;
  c.up = cross(forward, right);
  c.fwd = forward;
  c.u0 = -1.0f;
  c.v0 = -1.0f;
  c.u1 = 1.0f;
  c.v1 = 1.0f;
  c.far_offset = dot(forward, apex) + kSkyFar;
  bound_cone(c, forward);
  bool above = false;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (dot(normal, direction(c, float(k & 1), float(k >> 1))) > 0.0f) above = true;
  return above;
}

// ---- lights: gating and the unshadowed denominator -------------------------------
__device__ __forceinline__ f3 light_center(const DevLight& r) {  // :866-869
  if (is_sphere(r)) return r.corner;
  return r.corner + (r.eu + r.ev) * 0.5f;
}

__device__ __forceinline__ float spot_falloff(const DevLight& r, f3 w) {  // :872-876
  if (!is_sphere(r) || r.evw < 0.5f) return 1.0f;
  float a = clampf(dot(r.ev, w) * r.eu.y + r.eu.z, 0.0f, 1.0f);
  return a * a;
}

__device__ __forceinline__ bool faces_light(const DevLight& r, f3 point, f3 normal) {  // :880-884
  f3 to_light = light_center(r) - point;
  if (is_sphere(r)) return dot(normal, to_light) > -r.eu.x;
  return dot(normal, to_light) > 0.0f;
}

static __device__ __noinline__ float rect_open(f3 point, f3 normal, const DevLight& r) {  // :2148-2199
  f3 c0 = r.corner - point;
  float facing = dot(normalize(cross(r.eu, r.ev)), c0);
  if ((r.kind > 0.5f && facing >= 0.0f) || fabsf(facing) <= 1e-6f) return 0.0f;
  f3 d1 = c0 + r.eu, d2 = c0 + r.eu + r.ev, d3 = c0 + r.ev;
  if (dot(normal, c0) >= 0.f && dot(normal, d1) >= 0.f && dot(normal, d2) >= 0.f && dot(normal, d3) >= 0.f) {
    f3 a0 = normalize(c0), a1 = normalize(d1), a2 = normalize(d2), a3 = normalize(d3);
    float sum = 0.0f;
    sum += lambert_edge_unit(normal, a0, a1);
    sum += lambert_edge_unit(normal, a1, a2);
    sum += lambert_edge_unit(normal, a2, a3);
    sum += lambert_edge_unit(normal, a3, a0);
    return fabsf(0.5f * sum);
  }
  return clipped_quad_weight(normal, c0, d1, d2, d3);
}

__device__ __forceinline__ float sphere_unshadowed(f3 point, f3 normal, const DevLight& r) {  // :937-952
  f3 to_center = r.corner - point;
  float d2 = dot(to_center, to_center);
  float radius = r.eu.x;
  if (d2 <= radius * radius) return 0.0f;
  float sin2 = radius * radius / d2;
  float cos_t = clampf(dot(normal, to_center) * (1.0f / sqrtf(d2)), -1.0f, 1.0f);
  if (cos_t * cos_t > sin2) return 3.14159265f * sin2 * fmaxf(cos_t, 0.0f);
  float sin_t = sqrtf(1.0f - cos_t * cos_t);
  float x = sqrtf(1.0f / sin2 - 1.0f);
  float y = clampf(-x * cos_t / sin_t, -1.0f, 1.0f);
  float q = sin_t * sqrtf(1.0f - y * y);
  return fmaxf((cos_t * acosf(y) - x * q) * sin2 + atanf(q / x), 0.0f);
}

// unshadowed_rect (:2135-2141)
__device__ __forceinline__ float unshadowed(f3 point, f3 normal, const DevLight& r) {
  if (!faces_light(r, point, normal)) return 0.0f;
  if (is_sphere(r)) return spot_falloff(r, normalize(point - r.corner)) * sphere_unshadowed(point, normal, r);
  return rect_open(point, normal, r);
}

}  // namespace cc
