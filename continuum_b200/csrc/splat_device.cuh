// Prefiltered cones (mask_cones.wgsl:453-574, :1090-1150): a hierarchy node
// that projects to at most `prefilter` bins, wholly between the cone's near
// and far planes, is splatted as the convex hull of its projected corners,
// drawn with the node's opacity from its directional coverage samples,
// instead of being descended into.
#pragma once
#include "cone_device.cuh"

namespace cc {

constexpr int kCoverageSamples = 27;

// node_front_area (:462-486): the projected area of a node's front-facing
// triangles seen from unit direction v (toward the viewer), bilinear on the
// face of the cube of sample directions v points through; `cov` holds the
// node's 27 samples. mix as WGSL defines it: a (1 - t) + b t.
__device__ __forceinline__ float node_front_area(const float* __restrict__ cov, f3 v) {
  const f3 a = mk(fabsf(v.x), fabsf(v.y), fabsf(v.z));
  int axis = 0;
  if (a.y > a.x && a.y >= a.z) axis = 1;
  else if (a.z > a.x && a.z > a.y) axis = 2;
  float main, s, t;
  if (axis == 0) { main = v.x; s = v.y / a.x; t = v.z / a.x; }
  else if (axis == 1) { main = v.y; s = v.x / a.y; t = v.z / a.y; }
  else { main = v.z; s = v.x / a.z; t = v.y / a.z; }
  const int m = main >= 0.0f ? 1 : -1;
  const int s0 = s < 0.0f ? -1 : 0, t0 = t < 0.0f ? -1 : 0;
  const float fs = s - float(s0), ft = t - float(t0);
  float f[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int gs = s0 + (c & 1), gt = t0 + (c >> 1);
    int i, j, k;
    if (axis == 0) { i = m; j = gs; k = gt; }
    else if (axis == 1) { i = gs; j = m; k = gt; }
    else { i = gs; j = gt; k = m; }
    f[c] = __ldg(&cov[9 * (i + 1) + 3 * (j + 1) + (k + 1)]);
  }
  auto mix = [](float x, float y, float u) { return x * (1.0f - u) + y * u; };
  return mix(mix(f[0], f[1], fs), mix(f[2], f[3], fs), ft);
}

// hull8 (:488-511): the clockwise convex hull of 8 points (gift wrapping
// from the lowest-x point), the winding front-facing triangles have in bin
// space, so splats add to them. Returns its vertex count (at most 8).
__device__ __forceinline__ int hull8(const float2* pts, float2* out) {
  int start = 0;
#pragma unroll 1
  for (int k = 1; k < 8; ++k)
    if (pts[k].x < pts[start].x || (pts[k].x == pts[start].x && pts[k].y < pts[start].y)) start = k;
  int n = 0, cur = start;
#pragma unroll 1
  for (;;) {
    out[n++] = pts[cur];
    int next = (cur + 1) & 7;
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
      const float ex = pts[next].x - pts[cur].x, ey = pts[next].y - pts[cur].y;
      const float fx = pts[k].x - pts[cur].x, fy = pts[k].y - pts[cur].y;
      const float cr = ex * fy - ey * fx;
      if (cr > 0.0f || (cr == 0.0f && fx * fx + fy * fy > ex * ex + ey * ey)) next = k;
    }
    cur = next;
    if (cur == start || n >= 8) break;
  }
  return n;
}

// The hull of 8 projected corners clipped to the window's square and drawn
// with weight `alpha` (:564-573, :1123-1133). Returns whether anything was
// drawn. Out of line, with the square's four clips from one call site and
// rolled loops: the prefiltering walk, like the exact one, is bound by
// instruction fetch.
template <class Acc>
static __device__ __noinline__ bool draw_hull(Acc& acc, const float2* pts, float alpha) {
  const float g = float(kGrid);
  float2 qa[kPolyCap], qb[kPolyCap];
  int n = hull8(pts, qa);
  float2* q = qa;
  float2* q2 = qb;
#pragma unroll 1
  for (int side = 0; side < 4; ++side) {
    const float nx = side == 0 ? -1.0f : (side == 1 ? 1.0f : 0.0f);
    const float ny = side == 2 ? -1.0f : (side == 3 ? 1.0f : 0.0f);
    n = clip_line2(q, n, q2, nx, ny, (side & 1) ? g : 0.0f);
    float2* t = q;
    q = q2;
    q2 = t;
  }
  if (n < 3) return false;
  draw_polygon(acc, q, n, alpha);
  return true;
}

// A box's opacity terms (:555-560, :1114-1119): its silhouette area seen
// from the apex and the view direction toward the apex.
__device__ __forceinline__ float box_silhouette(const Cone& c, f3 lo, f3 hi, f3* v) {
  const f3 e = hi - lo;
  *v = normalize(c.apex - (lo + hi) * 0.5f);
  return fabsf(v->x) * e.y * e.z + fabsf(v->y) * e.x * e.z + fabsf(v->z) * e.x * e.y;
}

// node_cone_test (:519-574) for a triangle-hierarchy node (box lo..hi, its
// 27 coverage samples `cov`) and a cone prefiltering at `prefilter` bins:
// 0 if the box cannot touch the cone, 1 if it was splatted with nothing to
// draw, 2 if splatted and drawn into `acc`, 3 if the cone must descend.
// kHorizon: sky cones (their horizon culls a box wholly below it).
template <bool kHorizon, class Acc>
__device__ __noinline__ int node_cone_test(const Cone& c, f3 horizon, Acc& acc, const float* __restrict__ cov, f3 lo,
                                           f3 hi, float prefilter) {
  const float g = float(kGrid);
  float2 pts[8];
  float mnx = 3.4e38f, mny = 3.4e38f, mxx = -3.4e38f, mxy = -3.4e38f;
  bool far_out = true, near_out = true, out_u0 = true, out_u1 = true, out_v0 = true, out_v1 = true;
  bool below = kHorizon;
  bool inside = prefilter > 0.0f;  // splattable: every corner between the near and far planes
#pragma unroll 1
  for (int k = 0; k < 8; ++k) {
    const f3 corner = mk((k & 1) ? hi.x : lo.x, (k & 2) ? hi.y : lo.y, (k & 4) ? hi.z : lo.z);
    if constexpr (kHorizon) {
      if (dot(horizon, corner - c.apex) >= 0.0f) below = false;
    }
    const bool in_far = c.far_offset - dot(c.fwd, corner) >= 0.0f;
    if (in_far) far_out = false; else inside = false;
    const f3 p = to_local(c, corner);
    if (p.z >= kNear) near_out = false; else inside = false;
    if (p.x - c.u0 * p.z >= 0.0f) out_u0 = false;
    if (c.u1 * p.z - p.x >= 0.0f) out_u1 = false;
    if (p.y - c.v0 * p.z >= 0.0f) out_v0 = false;
    if (c.v1 * p.z - p.y >= 0.0f) out_v1 = false;
    if (inside) {
      const float qx = (p.x / p.z - c.u0) / (c.u1 - c.u0) * g;
      const float qy = (p.y / p.z - c.v0) / (c.v1 - c.v0) * g;
      pts[k] = make_float2(qx, qy);
      mnx = fminf(mnx, qx);
      mny = fminf(mny, qy);
      mxx = fmaxf(mxx, qx);
      mxy = fmaxf(mxy, qy);
    }
  }
  if (far_out || near_out || out_u0 || out_u1 || out_v0 || out_v1 || below) return 0;
  if (!in_bound(c, (lo + hi) * 0.5f, 0.5f * len(hi - lo))) return 0;
  if (!inside || fmaxf(mxx - mnx, mxy - mny) > prefilter) return 3;
  if (mxx <= 0.0f || mxy <= 0.0f || mnx >= g || mny >= g) return 1;
  f3 v;
  const float silhouette = box_silhouette(c, lo, hi, &v);
  if (silhouette <= 1e-30f) return 1;
  const float alpha = node_front_area(cov, v) / silhouette;
  if (alpha <= 0.0f) return 1;
  return draw_hull(acc, pts, alpha) ? 2 : 1;
}

// splat_object_node (:1096-1150) up to the drawing: whether object node lo..hi
// (its 27 coverage samples `cov`) is small enough in the cone to splat; if so,
// its hull is drawn into `acc` with opacity 1 - exp(-front area / silhouette)
// (its objects as independent occluders), to be combined into the mask as
// one more mesh without the whole-bin snap.
template <class Acc>
__device__ __noinline__ bool splat_object_node(const Cone& c, Acc& acc, const float* __restrict__ cov, f3 lo, f3 hi,
                                               float prefilter) {
  if (prefilter <= 0.0f) return false;
  const float g = float(kGrid);
  float2 pts[8];
  float mnx = 3.4e38f, mny = 3.4e38f, mxx = -3.4e38f, mxy = -3.4e38f;
#pragma unroll 1
  for (int k = 0; k < 8; ++k) {
    const f3 corner = mk((k & 1) ? hi.x : lo.x, (k & 2) ? hi.y : lo.y, (k & 4) ? hi.z : lo.z);
    if (c.far_offset - dot(c.fwd, corner) < 0.0f) return false;
    const f3 p = to_local(c, corner);
    if (p.z < kNear) return false;
    const float qx = (p.x / p.z - c.u0) / (c.u1 - c.u0) * g;
    const float qy = (p.y / p.z - c.v0) / (c.v1 - c.v0) * g;
    pts[k] = make_float2(qx, qy);
    mnx = fminf(mnx, qx);
    mny = fminf(mny, qy);
    mxx = fmaxf(mxx, qx);
    mxy = fmaxf(mxy, qy);
  }
  if (fmaxf(mxx - mnx, mxy - mny) > prefilter) return false;
  if (mxx <= 0.0f || mxy <= 0.0f || mnx >= g || mny >= g) return true;
  f3 v;
  const float silhouette = box_silhouette(c, lo, hi, &v);
  if (silhouette <= 1e-30f) return true;
  const float alpha = 1.0f - expf(-node_front_area(cov, v) / silhouette);
  if (alpha <= 0.0f) return true;
  draw_hull(acc, pts, alpha);
  return true;
}

}  // namespace cc
