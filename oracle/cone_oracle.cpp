// ORACLE — test infrastructure only. Nothing in the product links or calls this
// file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do,
// as the checker.
//
// A plain CPU restatement of Continuum's mask-cone area-light visibility path
// (reference v0.3.2), templated on the scalar type so the same code runs in
// FP32 (parity) and FP64 (error report). It follows, function by function:
//   crates/continuum-gpu/src/mask_cones.wgsl   (the GPU path the CUDA kernels replace)
//   crates/continuum-gpu/src/hierarchy.rs      (host BVH layouts)
//   crates/continuum/src/cone3.rs, coverage.rs, bvh.rs (the reference CPU path,
//                                               used to pin the restatement)
// Parity pins: the reference's own known-answer tests (cones_match_the_cpu,
// the large-wall test, cone3/coverage/bvh unit tests) are re-run against this
// file in tests/test_oracle_kat.py. Per-bin coverage has no golden vector in the
// reference; beyond the 1e-4-of-light-weight KAT bound it is pinned only by
// this restatement.
//
// Deliberate simplifications (all outside the exact light-cone path):
//   * prefilter threshold 0 (exact cones): node_cone_test reduces to
//     may_touch_box, splat_object_node never splats;
//   * light cones carry no horizon (the WGSL zero-initialises it), so the
//     horizon tests never cull and are left out;
//   * meshes are in world space (no instancing transforms), tri_weight 1.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

namespace oracle {

constexpr uint32_t GRID = 8;
constexpr uint32_t BINS = 64;
constexpr uint32_t NONE = 0xffffffffu;
constexpr int POLY_CAP = 16;  // the WGSL's is 10 (mask_cones.wgsl:11); see clip counts

template <class R> struct V3 {
  R x, y, z;
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> normalize(V3<R> a) { return a / length(a); }
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) {
  return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)};
}
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) {
  return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)};
}
template <class R> inline R clampv(R x, R lo, R hi) { return std::min(std::max(x, lo), hi); }

template <class R> struct V2 {
  R x, y;
};

// ---------------------------------------------------------------------------
// Host hierarchy (hierarchy.rs). Built in FP32 as the reference builds it.
// ---------------------------------------------------------------------------

struct Node {  // NodeGpu (hierarchy.rs:68-76): lo, hi, info = [first/left, count, 0, 0]
  float lo[4];
  float hi[4];
  uint32_t info[4];
};

using F3 = V3<float>;

// padded (hierarchy.rs:762-765)
static void padded(F3& lo, F3& hi) {
  float m = std::max(std::max(std::fabs(lo.x), std::fabs(hi.x)),
                     std::max(std::max(std::fabs(lo.y), std::fabs(hi.y)),
                              std::max(std::fabs(lo.z), std::fabs(hi.z))));
  float pad = 1e-5f * std::max(m, 1.0f);
  lo = lo - F3{pad, pad, pad};
  hi = hi + F3{pad, pad, pad};
}

// split (hierarchy.rs:128-179). The median partition puts the `mid` smallest
// keys on the left (ties broken by item id), and each leaf lists its items in
// increasing id, so the tree is fully determined by its inputs.
static void split(std::vector<Node>& nodes, size_t node, uint32_t* items, size_t count,
                  size_t start, const std::vector<std::pair<F3, F3>>& bounds, size_t leaf,
                  uint32_t node_base, uint32_t item_base) {
  F3 lo{FLT_MAX, FLT_MAX, FLT_MAX}, hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
  F3 clo = lo, chi = hi;
  for (size_t i = 0; i < count; ++i) {
    const auto& b = bounds[items[i]];
    lo = vmin(lo, b.first);
    hi = vmax(hi, b.second);
    F3 c = (b.first + b.second) * 0.5f;
    clo = vmin(clo, c);
    chi = vmax(chi, c);
  }
  Node& n = nodes[node];
  n.lo[0] = lo.x; n.lo[1] = lo.y; n.lo[2] = lo.z; n.lo[3] = 0;
  n.hi[0] = hi.x; n.hi[1] = hi.y; n.hi[2] = hi.z; n.hi[3] = 0;
  if (count <= leaf) {
    std::sort(items, items + count);
    n.info[0] = item_base + (uint32_t)start;
    n.info[1] = (uint32_t)count;
    n.info[2] = n.info[3] = 0;
    return;
  }
  F3 e = chi - clo;
  int axis = (e.x >= e.y && e.x >= e.z) ? 0 : (e.y >= e.z ? 1 : 2);
  auto key = [&](uint32_t m) {
    const auto& b = bounds[m];
    const float* a = &b.first.x;
    const float* c = &b.second.x;
    return a[axis] + c[axis];
  };
  size_t mid = count / 2;
  std::nth_element(items, items + mid, items + count, [&](uint32_t a, uint32_t b) {
    float ka = key(a), kb = key(b);
    return ka < kb || (ka == kb && a < b);
  });
  size_t left = nodes.size();
  nodes.push_back(Node{});
  nodes.push_back(Node{});
  nodes[node].info[0] = node_base + (uint32_t)left;
  nodes[node].info[1] = nodes[node].info[2] = nodes[node].info[3] = 0;
  split(nodes, left, items, mid, start, bounds, leaf, node_base, item_base);
  split(nodes, left + 1, items + mid, count - mid, start + mid, bounds, leaf, node_base, item_base);
}

struct Scene {
  std::vector<float> tris;       // 12 floats per triangle: three vec4 (hierarchy.rs:12-13)
  std::vector<uint32_t> ranges;  // 4 per mesh: first, count, blas root, xform (NONE)
  std::vector<Node> blas;
  std::vector<uint32_t> blas_items;
  std::vector<Node> nodes;       // object hierarchy (mesh_hierarchy)
  std::vector<uint32_t> items;
  uint32_t nmeshes = 0;
  // Instanced scenes: per transform, rows 0-2 of the rotation with the
  // translation in w, then (scale, 1 / scale, 0, 0) (Placement::rows,
  // hierarchy.rs:272-285); ranges[4 * m + 3] names object m's.
  std::vector<float> xforms;
  std::vector<uint32_t> object_geometry;  // instanced scenes: each object's geometry
  std::vector<uint32_t> geometry_root;    // instanced scenes: each geometry's triangle-hierarchy root (NONE: none)
  std::vector<std::pair<F3, F3>> geometry_box;  // instanced scenes: each geometry's object-space box
  // The movers' subtree (MoverTree, hierarchy.rs:309-327): root node 2, other
  // nodes from first_node, items from first_item, in `movers` order.
  uint32_t first_node = 0, mover_nodes = 0, first_item = 0;
  std::vector<uint32_t> movers;
  // Prefiltered cones: 27 coverage samples per triangle-hierarchy node and
  // (instanced scenes) per object-hierarchy node, built on first use.
  std::vector<float> blas_cov, obj_cov;
  bool coverage_built = false;
};

// COVERAGE_SAMPLES and coverage_directions (hierarchy.rs:710-723): directions
// (i, j, k) in {-1, 0, 1}^3 at index 9(i+1) + 3(j+1) + (k+1), normalized as
// glam's normalize_or_zero (times 1 / length; zero stays zero).
constexpr uint32_t COV = 27;
static void cov_directions(float d[COV][3]) {
  for (uint32_t n = 0; n < COV; ++n) {
    const float v[3] = {float(n / 9) - 1.0f, float(n / 3 % 3) - 1.0f, float(n % 3) - 1.0f};
    const float r = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int k = 0; k < 3; ++k) d[n][k] = (std::isfinite(r) && r > 0.0f) ? v[k] * r : 0.0f;
  }
}

// front_area (hierarchy.rs:625-652): bilinear on the sample cube's face,
// with Rust's lerp (a + (b - a) t).
static float host_front_area(const float* cov, const float v[3]) {
  const float ax = std::fabs(v[0]), ay = std::fabs(v[1]), az = std::fabs(v[2]);
  const int axis = (ay > ax && ay >= az) ? 1 : ((az > ax && az > ay) ? 2 : 0);
  const float main = axis == 0 ? v[0] : (axis == 1 ? v[1] : v[2]);
  const float div = axis == 0 ? ax : (axis == 1 ? ay : az);
  const float s = (axis == 0 ? v[1] : v[0]) / div;
  const float t = (axis == 2 ? v[1] : v[2]) / div;
  const int m = main >= 0.0f ? 1 : -1, s0 = s < 0.0f ? -1 : 0, t0 = t < 0.0f ? -1 : 0;
  const float fs = s - float(s0), ft = t - float(t0);
  float f[4];
  for (int c = 0; c < 4; ++c) {
    const int gs = s0 + (c & 1), gt = t0 + (c >> 1);
    int i = gs, j = gt, k = m;
    if (axis == 0) i = m, j = gs, k = gt;
    else if (axis == 1) i = gs, j = m, k = gt;
    f[c] = cov[9 * (i + 1) + 3 * (j + 1) + (k + 1)];
  }
  auto lerp = [](float a, float b, float u) { return a + (b - a) * u; };
  return lerp(lerp(f[0], f[1], fs), lerp(f[2], f[3], fs), ft);
}

// triangle_hierarchy's coverage (hierarchy.rs:546-569) over every mesh's
// triangle hierarchy, and object_coverage (:661-707) for instanced scenes.
static void build_coverage(Scene& sc) {
  if (sc.coverage_built) return;
  float d[COV][3];
  cov_directions(d);
  sc.blas_cov.assign(sc.blas.size() * COV, 0.0f);
  for (size_t n = sc.blas.size(); n-- > 0;) {
    float* out = &sc.blas_cov[n * COV];
    const uint32_t x = sc.blas[n].info[0], count = sc.blas[n].info[1];
    if (count > 0) {
      for (uint32_t k = x; k < x + count; ++k) {
        const float* t = &sc.tris[12 * (size_t)sc.blas_items[k]];
        const F3 a{t[0], t[1], t[2]}, b{t[4], t[5], t[6]}, c{t[8], t[9], t[10]};
        const F3 an = cross(b - a, c - a) * 0.5f;
        for (uint32_t i = 0; i < COV; ++i) out[i] += std::max(an.x * d[i][0] + an.y * d[i][1] + an.z * d[i][2], 0.0f);
      }
    } else {
      for (uint32_t i = 0; i < COV; ++i) out[i] = sc.blas_cov[(size_t)x * COV + i] + sc.blas_cov[((size_t)x + 1) * COV + i];
    }
  }
  // flatten_instanced (hierarchy.rs:469-503): a geometry's node samples
  // (from its root up to the next geometry's root, in root order) scale by
  // the opacity of the first object placing it, if that object is blended
  // or transmissive.
  if (!sc.geometry_root.empty()) {
    std::vector<std::pair<uint32_t, uint32_t>> roots;
    for (uint32_t g = 0; g < sc.geometry_root.size(); ++g)
      if (sc.geometry_root[g] != NONE) roots.push_back({sc.geometry_root[g], g});
    std::sort(roots.begin(), roots.end());
    for (size_t k = 0; k < roots.size(); ++k) {
      uint32_t first = NONE;
      for (uint32_t m = 0; m < sc.object_geometry.size(); ++m)
        if (sc.object_geometry[m] == roots[k].second) {
          first = m;
          break;
        }
      if (first == NONE) continue;
      const float clear = sc.xforms[16 * (size_t)sc.ranges[4 * first + 3] + 14];
      if (clear == 0.0f) continue;
      float opacity;
      if (clear > 0.0f) {
        opacity = 1.0f - clear;
      } else if (clear <= -2.0f) {
        const float t = 0.96f * (-2.0f - clear);
        opacity = 1.0f - t * t;
      } else {
        opacity = 1.0f - 0.96f * -clear;
      }
      const size_t end = k + 1 < roots.size() ? roots[k + 1].first : sc.blas.size();
      for (size_t i = (size_t)roots[k].first * COV; i < end * COV; ++i) sc.blas_cov[i] *= opacity;
    }
  }
  if (!sc.xforms.empty()) {
    std::vector<float> per((size_t)sc.nmeshes * COV, 0.0f);
    for (uint32_t m = 0; m < sc.nmeshes; ++m) {
      const uint32_t root = sc.ranges[4 * m + 2], xi = sc.ranges[4 * m + 3];
      if (root == NONE || xi == NONE) continue;
      const float* X = &sc.xforms[16 * (size_t)xi];
      for (uint32_t i = 0; i < COV; ++i) {
        if (d[i][0] == 0.0f && d[i][1] == 0.0f && d[i][2] == 0.0f) continue;
        // rotation^T d (glam: columns of the transpose, the rotation's rows, summed in order)
        const float v[3] = {X[0] * d[i][0] + X[4] * d[i][1] + X[8] * d[i][2],
                            X[1] * d[i][0] + X[5] * d[i][1] + X[9] * d[i][2],
                            X[2] * d[i][0] + X[6] * d[i][1] + X[10] * d[i][2]};
        per[(size_t)m * COV + i] = X[12] * X[12] * host_front_area(&sc.blas_cov[(size_t)root * COV], v);
      }
    }
    sc.obj_cov.assign(sc.nodes.size() * COV, 0.0f);
    for (size_t n = sc.nodes.size(); n-- > 0;) {
      float* out = &sc.obj_cov[n * COV];
      const uint32_t x = sc.nodes[n].info[0], count = sc.nodes[n].info[1];
      if (count > 0) {
        for (uint32_t k = x; k < x + count; ++k)
          for (uint32_t i = 0; i < COV; ++i) out[i] += per[(size_t)sc.items[k] * COV + i];
      } else {
        for (uint32_t i = 0; i < COV; ++i) out[i] = sc.obj_cov[(size_t)x * COV + i] + sc.obj_cov[((size_t)x + 1) * COV + i];
      }
    }
  }
  sc.coverage_built = true;
}

static void mesh_bounds(const float* tris, uint32_t first, uint32_t count, F3& lo, F3& hi) {
  lo = {FLT_MAX, FLT_MAX, FLT_MAX};
  hi = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t t = first; t < first + count; ++t)
    for (int k = 0; k < 3; ++k) {
      const float* v = tris + 12 * t + 4 * k;
      F3 p{v[0], v[1], v[2]};
      lo = vmin(lo, p);
      hi = vmax(hi, p);
    }
}

// object_hierarchy (hierarchy.rs:198-253): at most two objects per leaf,
// oversized objects (diagonal > 64 x median) in their own subtree.
static void object_hierarchy(Scene* s, const std::vector<std::pair<F3, F3>>& mesh_box,
                             const std::vector<uint32_t>* keep = nullptr) {
  std::vector<uint32_t> items;
  if (keep) {
    items = *keep;
  } else {
    items.resize(mesh_box.size());
    std::iota(items.begin(), items.end(), 0u);
  }
  const size_t nmeshes = items.size();
  s->nodes.assign(1, Node{});
  if (items.empty()) {
    s->items = {0};
    s->nodes[0].info[1] = 1;
    return;
  }
  auto diagonal = [&](uint32_t m) { return length(mesh_box[m].second - mesh_box[m].first); };
  std::vector<float> sizes(nmeshes);
  for (size_t i = 0; i < nmeshes; ++i) sizes[i] = diagonal(items[i]);
  size_t mid = sizes.size() / 2;
  std::nth_element(sizes.begin(), sizes.begin() + mid, sizes.end());
  float median = sizes[mid];
  std::vector<uint32_t> big, small;
  for (uint32_t m : items) (diagonal(m) > 64.0f * median ? big : small).push_back(m);
  if (big.empty() || small.empty()) {
    split(s->nodes, 0, items.data(), items.size(), 0, mesh_box, 2, 0, 0);
  } else {
    size_t nb = big.size();
    items = big;
    items.insert(items.end(), small.begin(), small.end());
    s->nodes.push_back(Node{});
    s->nodes.push_back(Node{});
    split(s->nodes, 1, items.data(), nb, 0, mesh_box, 2, 0, 0);
    split(s->nodes, 2, items.data() + nb, items.size() - nb, nb, mesh_box, 2, 0, 0);
    Node& r = s->nodes[0];
    const Node &a = s->nodes[1], &b = s->nodes[2];
    for (int k = 0; k < 3; ++k) {
      r.lo[k] = std::min(a.lo[k], b.lo[k]);
      r.hi[k] = std::max(a.hi[k], b.hi[k]);
    }
    r.info[0] = 1;
  }
  s->items = items;
}

// flatten + triangle_hierarchy + mesh_hierarchy/object_hierarchy
// (hierarchy.rs:29-66, 527-545, 183-253). Coverage samples (prefiltering) are
// not built: exact cones never read them.
static Scene* build_scene(const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes) {
  Scene* s = new Scene;
  s->nmeshes = nmeshes;
  uint64_t total = 0;
  for (uint32_t m = 0; m < nmeshes; ++m) total += mesh_counts[m];
  s->tris.resize(total * 12);
  for (uint64_t t = 0; t < total; ++t)
    for (int k = 0; k < 3; ++k) {
      s->tris[12 * t + 4 * k + 0] = tri9[9 * t + 3 * k + 0];
      s->tris[12 * t + 4 * k + 1] = tri9[9 * t + 3 * k + 1];
      s->tris[12 * t + 4 * k + 2] = tri9[9 * t + 3 * k + 2];
      s->tris[12 * t + 4 * k + 3] = 0.0f;
    }
  uint32_t first = 0;
  std::vector<std::pair<F3, F3>> mesh_box(nmeshes);
  for (uint32_t m = 0; m < nmeshes; ++m) {
    uint32_t count = mesh_counts[m];
    uint32_t root = NONE;
    if (count > 0) {
      root = (uint32_t)s->blas.size();
      std::vector<std::pair<F3, F3>> bounds(count);
      for (uint32_t t = 0; t < count; ++t) {
        F3 lo, hi;
        mesh_bounds(s->tris.data(), first + t, 1, lo, hi);
        padded(lo, hi);
        bounds[t] = {lo, hi};
      }
      std::vector<uint32_t> items(count);
      std::iota(items.begin(), items.end(), 0u);
      std::vector<Node> nodes(1);
      split(nodes, 0, items.data(), count, 0, bounds, 8, root, first);
      s->blas.insert(s->blas.end(), nodes.begin(), nodes.end());
      for (uint32_t t : items) s->blas_items.push_back(first + t);
    }
    s->ranges.insert(s->ranges.end(), {first, count, root, NONE});
    F3 lo, hi;
    mesh_bounds(s->tris.data(), first, count, lo, hi);
    padded(lo, hi);
    mesh_box[m] = {lo, hi};
    first += count;
  }
  object_hierarchy(s, mesh_box);
  return s;
}

// One object placing a geometry (cc_instance's layout): world = scale *
// rotation * p + translation, rotation row-major.
struct Instance {
  uint32_t geometry;
  float rotation[9];
  float scale;
  float translation[3];
};

// flatten_instanced (hierarchy.rs:464-522) + object_hierarchy over the
// objects' padded world bounds (Placement::world_bounds, :287-303).
// Placement::world_bounds (hierarchy.rs:287-303): the padded world bounds of
// an object-space box placed by `o`.
static std::pair<F3, F3> world_bounds(const std::pair<F3, F3>& box, const Instance& o) {
  const float* R = o.rotation;
  const float* t = o.translation;
  F3 lo{FLT_MAX, FLT_MAX, FLT_MAX}, hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
  const F3 a = box.first, b = box.second;
  for (int c = 0; c < 8; ++c) {
    const F3 p{(c & 1) ? b.x : a.x, (c & 2) ? b.y : a.y, (c & 4) ? b.z : a.z};
    const F3 w{(R[0] * p.x + R[1] * p.y + R[2] * p.z) * o.scale + t[0],
               (R[3] * p.x + R[4] * p.y + R[5] * p.z) * o.scale + t[1],
               (R[6] * p.x + R[7] * p.y + R[8] * p.z) * o.scale + t[2]};
    lo = vmin(lo, w);
    hi = vmax(hi, w);
  }
  padded(lo, hi);
  return {lo, hi};
}

// mover_subtree (hierarchy.rs:383-410): the movers' subtree over their
// current bounds (root at node 2, the rest from first_node, items from
// first_item), marked NO_SPLAT (1), and the root over both subtrees
// (union_root, :372-381).
static void mover_subtree(Scene* s, const std::vector<std::pair<F3, F3>>& bounds) {
  std::vector<Node> local(1);
  std::vector<uint32_t> order(bounds.size());
  std::iota(order.begin(), order.end(), 0u);
  split(local, 0, order.data(), order.size(), 0, bounds, 2, s->first_node - 1, s->first_item);
  for (Node& n : local) n.info[2] = 1;
  s->nodes[2] = local[0];
  for (size_t i = 1; i < local.size(); ++i) s->nodes[s->first_node + i - 1] = local[i];
  for (size_t k = 0; k < order.size(); ++k) s->items[s->first_item + k] = s->movers[order[k]];
  Node& r = s->nodes[0];
  r = Node{};
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = std::min(s->nodes[1].lo[k], s->nodes[2].lo[k]);
    r.hi[k] = std::max(s->nodes[1].hi[k], s->nodes[2].hi[k]);
  }
  r.info[0] = 1;
  r.info[2] = 1;
}

static uint32_t tree_nodes(uint32_t n, uint32_t leaf) {
  return n <= leaf ? 1 : 1 + tree_nodes(n / 2, leaf) + tree_nodes(n - n / 2, leaf);
}

static Scene* build_instanced(const float* tri9, const uint32_t* geometry_counts, uint32_t ngeometries,
                              const Instance* inst, uint32_t ninstances, const uint32_t* movable = nullptr,
                              uint32_t nmovable = 0) {
  Scene* s = build_scene(tri9, geometry_counts, ngeometries);
  const std::vector<uint32_t> geometry = s->ranges;
  std::vector<std::pair<F3, F3>> local(ngeometries);
  for (uint32_t g = 0; g < ngeometries; ++g) mesh_bounds(s->tris.data(), geometry[4 * g], geometry[4 * g + 1], local[g].first, local[g].second);
  s->ranges.clear();
  s->geometry_box = local;
  s->geometry_root.assign(ngeometries, NONE);
  for (uint32_t g = 0; g < ngeometries; ++g) s->geometry_root[g] = geometry[4 * g + 2];
  s->object_geometry.assign(ninstances, 0);
  std::vector<std::pair<F3, F3>> box(ninstances);
  for (uint32_t k = 0; k < ninstances; ++k) {
    const Instance& o = inst[k];
    s->object_geometry[k] = o.geometry;
    const uint32_t* r = &geometry[4 * o.geometry];
    s->ranges.insert(s->ranges.end(), {r[0], r[1], r[2], k});
    const float* R = o.rotation;
    const float* t = o.translation;
    s->xforms.insert(s->xforms.end(), {R[0], R[1], R[2], t[0], R[3], R[4], R[5], t[1], R[6], R[7], R[8], t[2],
                                       o.scale, 1.0f / o.scale, 0.0f, 0.0f});
    box[k] = world_bounds(local[o.geometry], o);
  }
  if (s->ranges.empty()) s->ranges.insert(s->ranges.end(), {0u, 0u, NONE, NONE});
  if (s->xforms.empty()) s->xforms.assign(16, 0.0f);
  s->nmeshes = (uint32_t)(s->ranges.size() / 4);
  s->nodes.clear();
  s->items.clear();
  if (nmovable == 0) {
    object_hierarchy(s, box);
    return s;
  }
  // object_hierarchy_with_movers (hierarchy.rs:331-369).
  std::vector<uint8_t> is_movable(ninstances, 0);
  for (uint32_t i = 0; i < nmovable; ++i) is_movable[movable[i]] = 1;
  std::vector<uint32_t> keep;
  for (uint32_t m = 0; m < ninstances; ++m)
    if (!is_movable[m]) keep.push_back(m);
  object_hierarchy(s, box, &keep);
  std::vector<Node> fixed = s->nodes;
  std::vector<uint32_t> items = s->items;
  auto place = [](uint32_t i) { return i == 0 ? 1u : i + 2u; };
  s->first_node = (uint32_t)fixed.size() + 2;
  s->first_item = (uint32_t)items.size();
  s->movers.assign(movable, movable + nmovable);
  s->mover_nodes = tree_nodes(nmovable, 2) - 1;
  s->nodes.assign(s->first_node + s->mover_nodes, Node{});
  for (size_t i = 0; i < fixed.size(); ++i) {
    Node n = fixed[i];
    if (n.info[1] == 0) n.info[0] = place(n.info[0]);
    s->nodes[place((uint32_t)i)] = n;
  }
  s->items = items;
  s->items.resize(items.size() + nmovable);
  std::vector<std::pair<F3, F3>> mb(nmovable);
  for (uint32_t i = 0; i < nmovable; ++i) mb[i] = box[movable[i]];
  mover_subtree(s, mb);
  return s;
}

// The movers placed anew (in `movers` order): transforms replaced, their
// subtree rebuilt; boxes12 (nullable) receives the bounds before and after.
static void move_objects(Scene* s, const Instance* placements, float* boxes12) {
  std::vector<std::pair<F3, F3>> mb(s->movers.size());
  for (size_t i = 0; i < s->movers.size(); ++i) {
    const uint32_t m = s->movers[i];
    const uint32_t x = s->ranges[4 * m + 3];
    float* X = &s->xforms[16 * (size_t)x];
    Instance old{};
    old.geometry = s->object_geometry[m];
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) old.rotation[3 * r + c] = X[4 * r + c];
      old.translation[r] = X[4 * r + 3];
    }
    old.scale = X[12];
    const auto before = world_bounds(s->geometry_box[old.geometry], old);
    const Instance& o = placements[i];
    const float* R = o.rotation;
    const float* t = o.translation;
    const float row[16] = {R[0], R[1], R[2], t[0], R[3], R[4], R[5], t[1], R[6], R[7], R[8], t[2],
                           o.scale, 1.0f / o.scale, X[14], 0.0f};  // the object keeps its clear
    std::memcpy(X, row, sizeof(row));
    mb[i] = world_bounds(s->geometry_box[old.geometry], o);
    if (boxes12) {
      const float v[12] = {before.first.x, before.first.y, before.first.z, before.second.x, before.second.y,
                           before.second.z, mb[i].first.x, mb[i].first.y, mb[i].first.z, mb[i].second.x,
                           mb[i].second.y, mb[i].second.z};
      std::memcpy(boxes12 + 12 * i, v, sizeof(v));
    }
  }
  mover_subtree(s, mb);
}

// ---------------------------------------------------------------------------
// The light cone (mask_cones.wgsl:136-1042).
// ---------------------------------------------------------------------------

template <class R> struct Cone {  // mask_cones.wgsl:136-155
  V3<R> apex, right, up, forward;
  R window[4];  // u0, v0, u1, v1
  V3<R> far_normal;
  R far_offset;
  V3<R> bound_axis;
  R bound_cos;
  R bound_sin;
  // Geometry wholly below the plane through the apex with this normal is
  // skipped: sky cones' receiver normal; zero (nothing skipped) for light
  // cones (:146-147).
  V3<R> horizon{R(0), R(0), R(0)};
};

template <class R> struct Light {  // LightRect (mask_cones.wgsl:843-848), LightGpu (lib.rs:710-749)
  V3<R> corner;
  R corner_w;  // 0 two-sided rect, 1 one-sided rect, 2 sphere
  V3<R> edge_u;
  R edge_u_w;
  V3<R> edge_v;
  R edge_v_w;
};

// How a mesh's cells are summed. kSumWalkOrder is the reference's: each
// add rounded into the scalar type in walk order (mask_cones.wgsl:297-348,
// 809-812). kSumFixed adds each value rounded to a multiple of 2^-24 of a bin
// into exact integer cells (the CUDA library's accumulator: its sums do not
// depend on the order of the adds). kSumExact sums the same values in double.
// Only the summation differs: every value added is the same.
enum AccumulateMode : uint32_t { kSumWalkOrder = 0, kSumFixed = 1, kSumExact = 2 };

template <class R> struct Params {
  uint32_t hierarchy;  // 0 every triangle, 1 mesh hierarchy, 2 + triangle hierarchies
  R wide_extent;
  uint32_t light_cone_cap;
  uint32_t wide_cone_cap;
  R prefilter = 0;               // prefilter_bins (0: exact cones)
  bool object_prefilter = true;  // object-level splats in instanced scenes
  uint32_t accumulate = kSumWalkOrder;  // AccumulateMode
  bool back_facing = false;  // vc_bake's estimator for a light below the horizon (:3476-3494)
};

template <class R> constexpr R NEAR = R(1e-4);

template <class R> inline V3<R> direction(const Cone<R>& c, R s, R t) {  // :203-206
  return c.forward + c.right * (c.window[0] + s * (c.window[2] - c.window[0])) +
         c.up * (c.window[1] + t * (c.window[3] - c.window[1]));
}

template <class R> inline V3<R> to_local(const Cone<R>& c, V3<R> p) {  // :208-211
  V3<R> d = p - c.apex;
  return {dot(c.right, d), dot(c.up, d), dot(c.forward, d)};
}

template <class R> bool in_bound(const Cone<R>& c, V3<R> p, R r) {  // :159-168
  if (c.bound_cos < R(-1)) return true;
  V3<R> d = p - c.apex;
  R len = length(d);
  if (len <= r) return true;
  R s = r / len;
  R limit = c.bound_cos * std::sqrt(R(1) - s * s) - c.bound_sin * s;
  return dot(c.bound_axis, d) >= limit * len;
}

template <class R> void bound_cone(Cone<R>& c, V3<R> axis) {  // :174-186
  R cos_half = 1;
  for (uint32_t k = 0; k < 4; ++k) {
    V3<R> d = normalize(direction(c, R(k & 1u), R(k >> 1u)));
    cos_half = std::min(cos_half, dot(axis, d));
  }
  R cos_b = clampv(cos_half - R(1e-5), R(-1), R(1));
  c.bound_axis = axis;
  c.bound_cos = cos_b;
  c.bound_sin = std::sqrt(std::max(R(1) - cos_b * cos_b, R(0)));
}

template <class R> R lambert_edge_unit(V3<R> n, V3<R> an, V3<R> bn) {  // :193-201
  V3<R> g = cross(an, bn);
  R len = length(g);
  if (len > R(1e-12)) return std::atan2(len, dot(an, bn)) * dot(n, g / len);
  return 0;
}

template <class R> R lambert_edge(V3<R> n, V3<R> a, V3<R> b) {  // :188-190
  return lambert_edge_unit(n, normalize(a), normalize(b));
}

template <class R> bool may_touch(const Cone<R>& c, V3<R> v0, V3<R> v1, V3<R> v2) {  // :215-232
  R f0 = c.far_offset - dot(c.far_normal, v0);
  R f1 = c.far_offset - dot(c.far_normal, v1);
  R f2 = c.far_offset - dot(c.far_normal, v2);
  if (f0 < 0 && f1 < 0 && f2 < 0) return false;
  if (dot(c.horizon, v0 - c.apex) < 0 && dot(c.horizon, v1 - c.apex) < 0 && dot(c.horizon, v2 - c.apex) < 0)
    return false;
  V3<R> p0 = to_local(c, v0), p1 = to_local(c, v1), p2 = to_local(c, v2);
  const R NR = NEAR<R>;
  if (p0.z < NR && p1.z < NR && p2.z < NR) return false;
  const R* w = c.window;
  if (p0.x - w[0] * p0.z < 0 && p1.x - w[0] * p1.z < 0 && p2.x - w[0] * p2.z < 0) return false;
  if (w[2] * p0.z - p0.x < 0 && w[2] * p1.z - p1.x < 0 && w[2] * p2.z - p2.x < 0) return false;
  if (p0.y - w[1] * p0.z < 0 && p1.y - w[1] * p1.z < 0 && p2.y - w[1] * p2.z < 0) return false;
  if (w[3] * p0.z - p0.y < 0 && w[3] * p1.z - p1.y < 0 && w[3] * p2.z - p2.y < 0) return false;
  return true;
}

template <class R> bool may_touch_box(const Cone<R>& c, V3<R> lo, V3<R> hi) {  // :234-255
  bool far_out = true, near_out = true, out_u0 = true, out_u1 = true, out_v0 = true, out_v1 = true, below = true;
  for (uint32_t k = 0; k < 8; ++k) {
    V3<R> corner{(k & 1u) ? hi.x : lo.x, (k & 2u) ? hi.y : lo.y, (k & 4u) ? hi.z : lo.z};
    if (c.far_offset - dot(c.far_normal, corner) >= 0) far_out = false;
    if (dot(c.horizon, corner - c.apex) >= 0) below = false;
    V3<R> p = to_local(c, corner);
    if (p.z >= NEAR<R>) near_out = false;
    if (p.x - c.window[0] * p.z >= 0) out_u0 = false;
    if (c.window[2] * p.z - p.x >= 0) out_u1 = false;
    if (p.y - c.window[1] * p.z >= 0) out_v0 = false;
    if (c.window[3] * p.z - p.y >= 0) out_v1 = false;
  }
  if (far_out || near_out || out_u0 || out_u1 || out_v0 || out_v1 || below) return false;
  return in_bound(c, (lo + hi) * R(0.5), R(0.5) * length(hi - lo));
}

template <class R> struct Poly3 {
  V3<R> v[POLY_CAP];
  int n = 0;
};
template <class R> struct Poly2 {
  V2<R> v[POLY_CAP];
  int n = 0;
};

// Diagnostic: polygons that would have exceeded the WGSL's 10-vertex arrays.
static std::atomic<uint64_t> g_poly_overflow{0};

template <class P, class T> inline void poly_push(P& out, const T& x) {
  if (out.n >= 10) g_poly_overflow.fetch_add(1, std::memory_order_relaxed);
  if (out.n < POLY_CAP) out.v[out.n++] = x;
}

// clip_plane3 (:264-277): keeps dot(normal, x) <= offset; crossings found from
// the kept end.
template <class R> Poly3<R> clip_plane3(const Poly3<R>& p, V3<R> normal, R offset) {
  Poly3<R> out;
  for (int i = 0; i < p.n; ++i) {
    V3<R> a = p.v[i], b = p.v[(i + 1) % p.n];
    R da = offset - dot(normal, a), db = offset - dot(normal, b);
    if (da >= 0) poly_push(out, a);
    if (da >= 0 && db < 0) poly_push(out, a + (b - a) * (da / (da - db)));
    if (da < 0 && db >= 0) poly_push(out, b + (a - b) * (db / (db - da)));
  }
  return out;
}

// clip_line2 (:280-294)
template <class R> Poly2<R> clip_line2(const Poly2<R>& p, V2<R> normal, R offset) {
  Poly2<R> out;
  for (int i = 0; i < p.n; ++i) {
    V2<R> a = p.v[i], b = p.v[(i + 1) % p.n];
    R da = offset - (normal.x * a.x + normal.y * a.y);
    R db = offset - (normal.x * b.x + normal.y * b.y);
    if (da >= 0) poly_push(out, a);
    if (da >= 0 && db < 0) {
      R f = da / (da - db);
      poly_push(out, V2<R>{a.x + (b.x - a.x) * f, a.y + (b.y - a.y) * f});
    }
    if (da < 0 && db >= 0) {
      R f = db / (db - da);
      poly_push(out, V2<R>{b.x + (a.x - b.x) * f, b.y + (a.y - b.y) * f});
    }
  }
  return out;
}

template <class R> struct Acc {
  R cell[68];
  int64_t fix[68];
  double wide[68];
  uint32_t mode = kSumWalkOrder;
  uint32_t span_lo, span_hi;
  void reset() {
    std::fill(cell, cell + 68, R(0));
    std::fill(fix, fix + 68, int64_t(0));
    std::fill(wide, wide + 68, 0.0);
    span_lo = 68;
    span_hi = 0;
  }
  void add(uint32_t i, R v) {
    if (mode == kSumFixed)
      fix[i] += (int64_t)std::nearbyint(float(v) * 16777216.0f);
    else if (mode == kSumExact)
      wide[i] += double(v);
    else
      cell[i] += v;
  }
};

// The running sum of a mesh's cells (:809-812) in the accumulator's mode.
template <class R> struct Running {
  R r = 0;
  int64_t f = 0;
  double w = 0;
  R next(const Acc<R>& a, uint32_t b) {
    if (a.mode == kSumFixed) {
      f += a.fix[b];
      return R(std::fabs(float(f) * (1.0f / 16777216.0f)));
    }
    if (a.mode == kSumExact) {
      w += a.wide[b];
      return R(std::fabs(w));
    }
    r += a.cell[b];
    return std::fabs(r);
  }
};

// draw_edge (:297-348): an edge's signed swept area added to the cells it
// crosses (accumulation rasterizer).
template <class R> void draw_edge(Acc<R>& acc, V2<R> q0, V2<R> q1, R weight) {
  if (std::fabs(q0.y - q1.y) <= R(1.1920929e-7)) return;
  R dir = 1;
  V2<R> p0 = q0, p1 = q1;
  if (q0.y > q1.y) {
    dir = -1;
    p0 = q1;
    p1 = q0;
  }
  R dxdy = (p1.x - p0.x) / (p1.y - p0.y);
  R x = p0.x;
  uint32_t y_end = std::min((uint32_t)std::ceil(p1.y), GRID);
  for (uint32_t y = (uint32_t)p0.y; y < y_end; ++y) {
    uint32_t row = y * GRID;
    acc.span_lo = std::min(acc.span_lo, row);
    acc.span_hi = std::max(acc.span_hi, row + GRID + 1);
    R dy = std::min(R(y + 1), p1.y) - std::max(R(y), p0.y);
    R x_next = clampv(x + dxdy * dy, R(0), R(GRID));
    R d = dy * dir * weight;
    R x0 = std::min(x, x_next), x1 = std::max(x, x_next);
    R x0_floor = std::floor(x0);
    uint32_t x0i = (uint32_t)x0_floor;
    R x1_ceil = std::ceil(x1);
    uint32_t x1i = (uint32_t)x1_ceil;
    if (x1i <= x0i + 1) {
      R xmf = R(0.5) * (x + x_next) - x0_floor;
      acc.add(row + x0i, d - d * xmf);
      acc.add(row + x0i + 1, d * xmf);
    } else {
      R s = R(1) / (x1 - x0);
      R x0f = x0 - x0_floor;
      R a0 = R(0.5) * s * (R(1) - x0f) * (R(1) - x0f);
      R x1f = x1 - x1_ceil + R(1);
      R am = R(0.5) * s * x1f * x1f;
      acc.add(row + x0i, d * a0);
      if (x1i == x0i + 2) {
        acc.add(row + x0i + 1, d * (R(1) - a0 - am));
      } else {
        R a1 = s * (R(1.5) - x0f);
        acc.add(row + x0i + 1, d * (a1 - a0));
        for (uint32_t xi = x0i + 2; xi < x1i - 1; ++xi) acc.add(row + xi, d * s);
        R a2 = a1 + R(x1i - x0i - 3) * s;
        acc.add(row + x1i - 1, d * (R(1) - a2 - am));
      }
      acc.add(row + x1i, d * am);
    }
    x = x_next;
  }
}

// rasterize (:350-451)
template <class R> bool rasterize(const Cone<R>& c, Acc<R>& acc, V3<R> v0, V3<R> v1, V3<R> v2, R weight = R(1)) {
  Poly3<R> p;
  p.v[0] = v0;
  p.v[1] = v1;
  p.v[2] = v2;
  p.n = 3;
  R f0 = c.far_offset - dot(c.far_normal, v0);
  R f1 = c.far_offset - dot(c.far_normal, v1);
  R f2 = c.far_offset - dot(c.far_normal, v2);
  if (f0 < 0 || f1 < 0 || f2 < 0) p = clip_plane3(p, c.far_normal, c.far_offset);
  bool all_near_ok = true, all_in_window = true;
  const R* w = c.window;
  for (int i = 0; i < p.n; ++i) {
    p.v[i] = to_local(c, p.v[i]);
    V3<R> v = p.v[i];
    if (v.z < NEAR<R>) all_near_ok = false;
    if (v.x < w[0] * v.z || v.x > w[2] * v.z || v.y < w[1] * v.z || v.y > w[3] * v.z) all_in_window = false;
  }
  if (!all_near_ok) p = clip_plane3(p, V3<R>{0, 0, -1}, -NEAR<R>);
  if (p.n < 3) return false;
  R su = R(GRID) / (w[2] - w[0]);
  R sv = R(GRID) / (w[3] - w[1]);
  R g = R(GRID);
  Poly2<R> q;
  if (all_near_ok && all_in_window) {
    q.n = p.n;
    for (int i = 0; i < p.n; ++i)
      q.v[i] = V2<R>{(p.v[i].x / p.v[i].z - w[0]) * su, (p.v[i].y / p.v[i].z - w[1]) * sv};
  } else {
    // The window's square clipped to the directions through the polygon
    // (the apex-plane clip, :376-425).
    R d = dot(to_local(c, v0), cross(to_local(c, v1), to_local(c, v2)));
    if (d == 0) return false;
    R side = d > 0 ? R(1) : R(-1);
    q.n = 4;
    q.v[0] = {0, 0};
    q.v[2] = {g, g};
    if (side > 0) {
      q.v[1] = {g, 0};
      q.v[3] = {0, g};
    } else {
      q.v[1] = {0, g};
      q.v[3] = {g, 0};
    }
    for (int i = 0; i < p.n; ++i) {
      V3<R> e = cross(p.v[i], p.v[(i + 1) % p.n]);
      R len = length(e);
      if (len == 0) continue;
      V3<R> k = e * (side / len);
      q = clip_line2(q, V2<R>{-k.x / su, -k.y / sv}, k.x * w[0] + k.y * w[1] + k.z);
    }
  }
  bool inside = true;
  for (int i = 0; i < q.n; ++i)
    if (q.v[i].x < 0 || q.v[i].y < 0 || q.v[i].x > g || q.v[i].y > g) inside = false;
  if (!inside) {
    q = clip_line2(q, V2<R>{-1, 0}, R(0));
    q = clip_line2(q, V2<R>{1, 0}, g);
    q = clip_line2(q, V2<R>{0, -1}, R(0));
    q = clip_line2(q, V2<R>{0, 1}, g);
  }
  if (q.n < 3) return false;
  for (int i = 0; i < q.n; ++i) {
    V2<R> a = q.v[i], b = q.v[(i + 1) % q.n];
    a = {clampv(a.x, R(0), g), clampv(a.y, R(0), g)};
    b = {clampv(b.x, R(0), g), clampv(b.y, R(0), g)};
    draw_edge(acc, a, b, weight);
  }
  return true;
}

template <class R> inline V3<R> tri_vertex(const Scene& s, uint32_t t, int k) {
  const float* v = s.tris.data() + 12 * (size_t)t + 4 * k;
  return {R(v[0]), R(v[1]), R(v[2])};
}

struct Work {  // the reference's work counters (mask_cones.wgsl:655-665), per cone
  uint32_t object_nodes = 0;  // object-hierarchy nodes tested
  uint32_t blas_nodes = 0;    // triangle-hierarchy nodes tested
  uint32_t tris = 0;          // triangles tested
  uint32_t flags = 0;         // bit 0: walk capped; bit 1: stack overflow
  uint32_t skip = NONE;       // a triangle not drawn (cover_skip, :588-595): the receiver's own
};

// cover_triangle (:594-616)
// The placed object a mesh's triangles belong to: its triangles' weight and
// its transmission, from its transform's `clear` (row 3's z;
// add_mesh_coverage_if, :725-741). World-space meshes: weight 1.
template <class R> struct ObjectLight {
  R weight = R(1);
  R transmit = R(0);
  bool volume = false;
};
template <class R> ObjectLight<R> object_light(const Scene& s, uint32_t x) {
  ObjectLight<R> o;
  if (x == NONE || s.xforms.empty()) return o;
  const R clear = R(s.xforms[16 * (size_t)x + 14]);
  o.weight = R(1) - std::max(clear, R(0));
  o.transmit = std::max(-clear, R(0));
  if (clear <= R(-2)) {  // a volume: two surfaces
    o.transmit = R(-2) - clear;
    o.volume = true;
  }
  return o;
}

// cover_triangle (:594-616): the culls, then the triangle drawn with its
// object's weight, or for a transmissive object one less what passes through
// it at the cone's central direction (Schlick's Fresnel, F0 0.04; twice for
// a volume; the fifth power by multiplications).
template <class R> bool cover_triangle(const Scene& s, const Cone<R>& c, Acc<R>& acc, uint32_t t, Work& wk,
                                       const ObjectLight<R>& ol = ObjectLight<R>{}) {
  wk.tris++;
  if (t == wk.skip) return false;
  V3<R> v0 = tri_vertex<R>(s, t, 0), v1 = tri_vertex<R>(s, t, 1), v2 = tri_vertex<R>(s, t, 2);
  V3<R> n = cross(v1 - v0, v2 - v0);
  if (dot(n, c.apex - v0) <= 0) return false;
  if (dot(n, direction(c, R(0), R(0))) >= 0 && dot(n, direction(c, R(1), R(0))) >= 0 &&
      dot(n, direction(c, R(0), R(1))) >= 0 && dot(n, direction(c, R(1), R(1))) >= 0)
    return false;
  if (!may_touch(c, v0, v1, v2)) return false;
  R weight = ol.weight;
  if (ol.transmit > R(0)) {
    const R cos_t = std::fabs(dot(normalize(n), normalize(direction(c, R(0.5), R(0.5)))));
    const R x = R(1) - cos_t;
    const R x2 = x * x;
    const R f = R(0.04) + R(0.96) * (x2 * x2 * x);
    R passes = ol.transmit * (R(1) - f);
    if (ol.volume) passes *= R(1) - f;
    weight = R(1) - passes;
  }
  return rasterize(c, acc, v0, v1, v2, weight);
}

// --- Prefiltered cones (:453-574, :1090-1150) ---

// node_front_area (:462-486) over a node's 27 samples, with WGSL's mix
// (a (1 - t) + b t).
template <class R> R node_front_area(const float* cov, V3<R> v) {
  const R ax = std::fabs(v.x), ay = std::fabs(v.y), az = std::fabs(v.z);
  uint32_t axis = 0;
  if (ay > ax && ay >= az) axis = 1;
  else if (az > ax && az > ay) axis = 2;
  R main, s, t;
  if (axis == 0) { main = v.x; s = v.y / ax; t = v.z / ax; }
  else if (axis == 1) { main = v.y; s = v.x / ay; t = v.z / ay; }
  else { main = v.z; s = v.x / az; t = v.y / az; }
  const int m = main >= 0 ? 1 : -1, s0 = s < 0 ? -1 : 0, t0 = t < 0 ? -1 : 0;
  const R fs = s - R(s0), ft = t - R(t0);
  R f[4];
  for (int c = 0; c < 4; ++c) {
    const int gs = s0 + (c & 1), gt = t0 + (c >> 1);
    int i, j, k;
    if (axis == 0) { i = m; j = gs; k = gt; }
    else if (axis == 1) { i = gs; j = m; k = gt; }
    else { i = gs; j = gt; k = m; }
    f[c] = R(cov[9 * (i + 1) + 3 * (j + 1) + (k + 1)]);
  }
  auto mix = [](R a, R b, R u) { return a * (R(1) - u) + b * u; };
  return mix(mix(f[0], f[1], fs), mix(f[2], f[3], fs), ft);
}

// hull8 (:488-511): clockwise convex hull of 8 points by gift wrapping.
template <class R> Poly2<R> hull8(const V2<R> (&pts)[8]) {
  int start = 0;
  for (int k = 1; k < 8; ++k)
    if (pts[k].x < pts[start].x || (pts[k].x == pts[start].x && pts[k].y < pts[start].y)) start = k;
  Poly2<R> out;
  int cur = start;
  for (;;) {
    out.v[out.n++] = pts[cur];
    int next = (cur + 1) % 8;
    for (int k = 0; k < 8; ++k) {
      const R ex = pts[next].x - pts[cur].x, ey = pts[next].y - pts[cur].y;
      const R fx = pts[k].x - pts[cur].x, fy = pts[k].y - pts[cur].y;
      const R cr = ex * fy - ey * fx;
      if (cr > 0 || (cr == 0 && fx * fx + fy * fy > ex * ex + ey * ey)) next = k;
    }
    cur = next;
    if (cur == start || out.n >= 8) break;
  }
  return out;
}

// The hull clipped to the square and drawn with weight alpha (:564-573).
template <class R> bool draw_hull(Acc<R>& acc, const V2<R> (&pts)[8], R alpha) {
  const R g = R(GRID);
  Poly2<R> q = hull8(pts);
  q = clip_line2(q, V2<R>{-1, 0}, R(0));
  q = clip_line2(q, V2<R>{1, 0}, g);
  q = clip_line2(q, V2<R>{0, -1}, R(0));
  q = clip_line2(q, V2<R>{0, 1}, g);
  if (q.n < 3) return false;
  for (int i = 0; i < q.n; ++i) {
    V2<R> a = q.v[i], b = q.v[(i + 1) % q.n];
    a = {clampv(a.x, R(0), g), clampv(a.y, R(0), g)};
    b = {clampv(b.x, R(0), g), clampv(b.y, R(0), g)};
    draw_edge(acc, a, b, alpha);
  }
  return true;
}

// node_cone_test (:519-574): 0 cannot touch, 1 splatted with nothing drawn,
// 2 splatted and drawn, 3 descend. With prefilter 0 it is may_touch_box.
template <class R> int node_cone_test(const Cone<R>& c, Acc<R>& acc, const float* cov, V3<R> lo, V3<R> hi,
                                      R prefilter) {
  const R g = R(GRID);
  V2<R> pts[8];
  R mnx = R(3.4e38), mny = R(3.4e38), mxx = R(-3.4e38), mxy = R(-3.4e38);
  bool far_out = true, near_out = true, out_u0 = true, out_u1 = true, out_v0 = true, out_v1 = true, below = true;
  bool inside = prefilter > 0;
  const R* w = c.window;
  for (uint32_t k = 0; k < 8; ++k) {
    V3<R> corner{(k & 1u) ? hi.x : lo.x, (k & 2u) ? hi.y : lo.y, (k & 4u) ? hi.z : lo.z};
    if (dot(c.horizon, corner - c.apex) >= 0) below = false;
    const bool in_far = c.far_offset - dot(c.far_normal, corner) >= 0;
    if (in_far) far_out = false; else inside = false;
    V3<R> p = to_local(c, corner);
    if (p.z >= NEAR<R>) near_out = false; else inside = false;
    if (p.x - w[0] * p.z >= 0) out_u0 = false;
    if (w[2] * p.z - p.x >= 0) out_u1 = false;
    if (p.y - w[1] * p.z >= 0) out_v0 = false;
    if (w[3] * p.z - p.y >= 0) out_v1 = false;
    if (inside) {
      const V2<R> q{(p.x / p.z - w[0]) / (w[2] - w[0]) * g, (p.y / p.z - w[1]) / (w[3] - w[1]) * g};
      pts[k] = q;
      mnx = std::min(mnx, q.x);
      mny = std::min(mny, q.y);
      mxx = std::max(mxx, q.x);
      mxy = std::max(mxy, q.y);
    }
  }
  if (far_out || near_out || out_u0 || out_u1 || out_v0 || out_v1 || below) return 0;
  if (!in_bound(c, (lo + hi) * R(0.5), R(0.5) * length(hi - lo))) return 0;
  if (!inside || std::max(mxx - mnx, mxy - mny) > prefilter) return 3;
  if (mxx <= 0 || mxy <= 0 || mnx >= g || mny >= g) return 1;
  const V3<R> e = hi - lo;
  const V3<R> v = normalize(c.apex - (lo + hi) * R(0.5));
  const R silhouette = std::fabs(v.x) * e.y * e.z + std::fabs(v.y) * e.x * e.z + std::fabs(v.z) * e.x * e.y;
  if (silhouette <= R(1e-30)) return 1;
  const R alpha = node_front_area(cov, v) / silhouette;
  if (alpha <= 0) return 1;
  return draw_hull(acc, pts, alpha) ? 2 : 1;
}

template <class R> inline V3<R> node_lo(const Node& n) { return {R(n.lo[0]), R(n.lo[1]), R(n.lo[2])}; }
template <class R> inline V3<R> node_hi(const Node& n) { return {R(n.hi[0]), R(n.hi[1]), R(n.hi[2])}; }

template <class R> struct Walk {
  R cov[BINS];
  uint32_t full = 0;
  uint32_t cone_work = 0;
  uint32_t cone_cap = NONE;
  bool independent = false;  // sky cones: meshes combine as independent occluders (:819-821)
  R prefilter = 0;           // prefilter_bins (0: exact cones)
  bool object_prefilter = false;
  uint32_t accumulate = kSumWalkOrder;  // how each mesh's cells are summed (AccumulateMode)
  Work work;
};

// splat_object_node (:1096-1150): an object node small in the cone splatted
// into the mask as one more mesh (opacity 1 - exp(-front area / silhouette),
// no whole-bin snap). Returns whether it was splatted (or found empty).
template <class R> bool splat_object_node(const Scene& s, const Cone<R>& c, uint32_t n, V3<R> lo, V3<R> hi,
                                          Walk<R>& wk) {
  if (!wk.object_prefilter || s.obj_cov.empty() || wk.prefilter <= 0) return false;
  const R g = R(GRID);
  const R* w = c.window;
  V2<R> pts[8];
  R mnx = R(3.4e38), mny = R(3.4e38), mxx = R(-3.4e38), mxy = R(-3.4e38);
  for (uint32_t k = 0; k < 8; ++k) {
    V3<R> corner{(k & 1u) ? hi.x : lo.x, (k & 2u) ? hi.y : lo.y, (k & 4u) ? hi.z : lo.z};
    if (c.far_offset - dot(c.far_normal, corner) < 0) return false;
    V3<R> p = to_local(c, corner);
    if (p.z < NEAR<R>) return false;
    const V2<R> q{(p.x / p.z - w[0]) / (w[2] - w[0]) * g, (p.y / p.z - w[1]) / (w[3] - w[1]) * g};
    pts[k] = q;
    mnx = std::min(mnx, q.x);
    mny = std::min(mny, q.y);
    mxx = std::max(mxx, q.x);
    mxy = std::max(mxy, q.y);
  }
  if (std::max(mxx - mnx, mxy - mny) > wk.prefilter) return false;
  if (mxx <= 0 || mxy <= 0 || mnx >= g || mny >= g) return true;
  const V3<R> e = hi - lo;
  const V3<R> v = normalize(c.apex - (lo + hi) * R(0.5));
  const R silhouette = std::fabs(v.x) * e.y * e.z + std::fabs(v.y) * e.x * e.z + std::fabs(v.z) * e.x * e.y;
  if (silhouette <= R(1e-30)) return true;
  const R alpha = R(1) - std::exp(-node_front_area(&s.obj_cov[(size_t)n * COV], v) / silhouette);
  if (alpha <= 0) return true;
  Acc<R> acc;
  acc.reset();
  acc.mode = wk.accumulate;
  if (!draw_hull(acc, pts, alpha)) return true;
  Running<R> running;
  for (uint32_t b = acc.span_lo; b < std::min(acc.span_hi, BINS); ++b) {
    const R covered = std::min(running.next(acc, b), R(1));
    if (covered > R(1e-6)) {
      const R before = wk.cov[b];
      wk.cov[b] = wk.independent ? R(1) - (R(1) - before) * (R(1) - covered) : std::max(before, covered);
      if (before < R(1) && wk.cov[b] >= R(1)) wk.full++;
    }
  }
  return true;
}

constexpr int STACK = 64;

// cone_to_object (:623-638) with rotate_to_object, translation and
// point_to_object (:61-78): the cone in the space of the object placed by
// transform x.
template <class R> Cone<R> cone_to_object(const Scene& s, const Cone<R>& c, uint32_t x) {
  const float* X = s.xforms.data() + 16 * (size_t)x;
  const V3<R> r0{R(X[0]), R(X[1]), R(X[2])}, r1{R(X[4]), R(X[5]), R(X[6])}, r2{R(X[8]), R(X[9]), R(X[10])};
  const V3<R> t{R(X[3]), R(X[7]), R(X[11])};
  const R inv_scale = R(X[13]);
  auto rot = [&](V3<R> d) { return r0 * d.x + r1 * d.y + r2 * d.z; };
  Cone<R> o = c;
  o.apex = rot(c.apex - t) * inv_scale;
  o.right = rot(c.right);
  o.up = rot(c.up);
  o.forward = rot(c.forward);
  o.far_normal = rot(c.far_normal);
  o.far_offset = (c.far_offset - dot(c.far_normal, t)) * inv_scale;
  o.bound_axis = rot(c.bound_axis);
  o.horizon = rot(c.horizon);
  return o;
}

// add_mesh_coverage_if for one cone walking alone (:713-829).
template <class R> void add_mesh_coverage(const Scene& s, const Cone<R>& world, uint32_t m, Walk<R>& wk,
                                          uint32_t hierarchy) {
  Acc<R> acc;
  acc.reset();
  acc.mode = wk.accumulate;
  bool touched = false;
  const uint32_t* range = s.ranges.data() + 4 * m;
  const Cone<R> c = range[3] != NONE ? cone_to_object(s, world, range[3]) : world;
  const ObjectLight<R> ol = object_light<R>(s, range[3]);
  if (hierarchy == 2) {
    if (range[2] != NONE) {
      uint32_t stack[STACK];
      int sp = 0;
      stack[sp++] = range[2];
      while (sp > 0) {
        uint32_t n = stack[--sp];
        if (!(wk.cone_work < wk.cone_cap)) continue;
        wk.cone_work++;
        const Node& node = s.blas[n];
        wk.work.blas_nodes++;
        const float* cov = s.blas_cov.empty() ? nullptr : &s.blas_cov[(size_t)n * COV];
        const int test = node_cone_test(c, acc, cov, node_lo<R>(node), node_hi<R>(node), wk.prefilter);
        if (test == 2) touched = true;
        if (test != 3) continue;
        if (node.info[1] > 0) {
          wk.cone_work += node.info[1];
          for (uint32_t k = node.info[0]; k < node.info[0] + node.info[1]; ++k)
            if (cover_triangle(s, c, acc, s.blas_items[k], wk.work, ol)) touched = true;
        } else {
          if (sp + 2 > STACK) {
            wk.work.flags |= 2;
            continue;
          }
          stack[sp++] = node.info[0];
          stack[sp++] = node.info[0] + 1;
        }
      }
    }
  } else {
    for (uint32_t t = range[0]; t < range[0] + range[1]; ++t)
      if (cover_triangle(s, c, acc, t, wk.work, ol)) touched = true;
  }
  if (touched) {
    Running<R> running;
    for (uint32_t b = acc.span_lo; b < std::min(acc.span_hi, BINS); ++b) {
      R covered = running.next(acc, b);
      if (covered >= R(1) - R(1e-5)) covered = 1;
      if (covered > R(1e-6)) {
        R before = wk.cov[b];
        if (wk.independent)
          wk.cov[b] = R(1) - (R(1) - before) * (R(1) - std::min(covered, R(1)));
        else
          wk.cov[b] = std::max(before, std::min(covered, R(1)));
        if (before < R(1) && wk.cov[b] >= R(1)) wk.full++;
      }
    }
  }
}

// scene_coverage_if for one cone walking alone (:1160-1227): nearest child
// first along the bounding cone's axis, stop once every bin is full or at
// the walk cap.
template <class R> void scene_coverage(const Scene& s, const Cone<R>& c, Walk<R>& wk, uint32_t hierarchy) {
  wk.cone_work = 0;
  if (hierarchy >= 1) {
    uint32_t stack[STACK];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      uint32_t n = stack[--sp];
      if (!(wk.full < BINS && wk.cone_work < wk.cone_cap)) continue;
      wk.cone_work++;
      const Node& node = s.nodes[n];
      wk.work.object_nodes++;
      if (!may_touch_box(c, node_lo<R>(node), node_hi<R>(node))) continue;
      // info.z 1: no prefiltered coverage (the root over movers and the
      // movers' subtree, whose boxes change).
      if (node.info[2] == 0 && splat_object_node(s, c, n, node_lo<R>(node), node_hi<R>(node), wk)) continue;
      if (node.info[1] > 0) {
        for (uint32_t k = node.info[0]; k < node.info[0] + node.info[1]; ++k)
          add_mesh_coverage(s, c, s.items[k], wk, hierarchy);
      } else {
        uint32_t near_ = node.info[0], far_ = node.info[0] + 1;
        const Node& a = s.nodes[near_];
        const Node& b = s.nodes[far_];
        // Nearest child first where meshes combine by the maximum; independent
        // occluders (sky cones) keep the left child first (:1188-1207).
        if (!wk.independent) {
          V3<R> axis = c.bound_axis;  // a light cone's bound is always set
          R da = dot(axis, (node_lo<R>(a) + node_hi<R>(a)) * R(0.5) - c.apex);
          R db = dot(axis, (node_lo<R>(b) + node_hi<R>(b)) * R(0.5) - c.apex);
          if (db < da) std::swap(near_, far_);
        }
        if (sp + 2 > STACK) {
          wk.work.flags |= 2;
          continue;
        }
        stack[sp++] = far_;
        stack[sp++] = near_;
      }
    }
  } else {
    for (uint32_t m = 0; m < s.nmeshes; ++m)
      if (wk.full < BINS) add_mesh_coverage(s, c, m, wk, hierarchy);
  }
}

// bin_weight (:1232-1242)
template <class R> R bin_weight(const Cone<R>& c, V3<R> n, uint32_t b) {
  R col = R(b % GRID), row = R(b / GRID), g = R(GRID);
  V3<R> d0 = direction(c, col / g, row / g);
  V3<R> d1 = direction(c, (col + 1) / g, row / g);
  V3<R> d2 = direction(c, (col + 1) / g, (row + 1) / g);
  V3<R> d3 = direction(c, col / g, (row + 1) / g);
  return std::fabs(R(0.5) * (lambert_edge(n, d0, d1) + lambert_edge(n, d1, d2) + lambert_edge(n, d2, d3) +
                             lambert_edge(n, d3, d0)));
}

// The quad d[0..4] clipped to dot(n, x) >= 0, Lambert-integrated (:1331-1403).
template <class R> R clipped_quad_weight(V3<R> n, const V3<R> d[4]) {
  V3<R> poly[6];
  int k_n = 0;
  for (int k = 0; k < 4; ++k) {
    V3<R> a = d[k], e = d[(k + 1) % 4];
    R sa = dot(n, a), se = dot(n, e);
    if (sa >= 0) poly[k_n++] = a;
    if ((sa >= 0) != (se >= 0)) poly[k_n++] = a + (e - a) * (sa / (sa - se));
  }
  if (k_n < 3) return 0;
  R sum = 0;
  for (int k = 0; k < k_n; ++k) sum += lambert_edge(n, poly[k], poly[(k + 1) % k_n]);
  return std::fabs(R(0.5) * sum);
}

template <class R> R clipped_bin_weight(const Cone<R>& c, V3<R> n, uint32_t b) {  // :1331-1369
  R col = R(b % GRID), row = R(b / GRID), g = R(GRID);
  V3<R> d[4] = {direction(c, col / g, row / g), direction(c, (col + 1) / g, row / g),
                direction(c, (col + 1) / g, (row + 1) / g), direction(c, col / g, (row + 1) / g)};
  int above = 0;
  for (int k = 0; k < 4; ++k)
    if (dot(n, d[k]) > 0) above++;
  if (above == 4) return bin_weight(c, n, b);
  if (above == 0) return 0;
  return clipped_quad_weight(n, d);
}

template <class R> R clipped_window_weight(const Cone<R>& c, V3<R> n) {  // :1375-1403
  V3<R> d[4] = {direction(c, R(0), R(0)), direction(c, R(1), R(0)), direction(c, R(1), R(1)),
                direction(c, R(0), R(1))};
  return clipped_quad_weight(n, d);
}

// cone_visible (:1244-1272)
template <class R> R cone_visible(const Cone<R>& c, V3<R> n, const R* cov) {
  V3<R> d00 = direction(c, R(0), R(0)), d10 = direction(c, R(1), R(0));
  V3<R> d11 = direction(c, R(1), R(1)), d01 = direction(c, R(0), R(1));
  if (dot(n, d00) > 0 && dot(n, d10) > 0 && dot(n, d11) > 0 && dot(n, d01) > 0) {
    R blocked = 0;
    for (uint32_t b = 0; b < BINS; ++b)
      if (cov[b] > 0) blocked += cov[b] * bin_weight(c, n, b);
    R total = std::fabs(R(0.5) * (lambert_edge(n, d00, d10) + lambert_edge(n, d10, d11) +
                                  lambert_edge(n, d11, d01) + lambert_edge(n, d01, d00)));
    return std::max(total - blocked, R(0));
  }
  R blocked = 0;
  for (uint32_t b = 0; b < BINS; ++b)
    if (cov[b] > 0) blocked += cov[b] * clipped_bin_weight(c, n, b);
  return std::max(clipped_window_weight(c, n) - blocked, R(0));
}

template <class R> R window_open(const Cone<R>& c, V3<R> n) {  // :1074-1085
  V3<R> d00 = direction(c, R(0), R(0)), d10 = direction(c, R(1), R(0));
  V3<R> d11 = direction(c, R(1), R(1)), d01 = direction(c, R(0), R(1));
  if (dot(n, d00) > 0 && dot(n, d10) > 0 && dot(n, d11) > 0 && dot(n, d01) > 0)
    return std::fabs(R(0.5) * (lambert_edge(n, d00, d10) + lambert_edge(n, d10, d11) +
                               lambert_edge(n, d11, d01) + lambert_edge(n, d01, d00)));
  return clipped_window_weight(c, n);
}

template <class R> inline bool is_sphere(const Light<R>& r) { return r.corner_w > R(1.5); }

template <class R> V3<R> light_center(const Light<R>& r) {  // :866-869
  if (is_sphere(r)) return r.corner;
  return r.corner + (r.edge_u + r.edge_v) * R(0.5);
}

template <class R> R spot_falloff(const Light<R>& r, V3<R> w) {  // :872-876
  if (!is_sphere(r) || r.edge_v_w < R(0.5)) return 1;
  R a = clampv(dot(r.edge_v, w) * r.edge_u.y + r.edge_u.z, R(0), R(1));
  return a * a;
}

template <class R> bool faces_light(const Light<R>& r, V3<R> point, V3<R> normal) {  // :880-884
  V3<R> to_light = light_center(r) - point;
  if (is_sphere(r)) return dot(normal, to_light) > -r.edge_u.x;
  return dot(normal, to_light) > 0;
}

// rect_open (:2148-2199)
template <class R> R rect_open(V3<R> point, V3<R> normal, const Light<R>& r) {
  V3<R> u = r.edge_u, v = r.edge_v, c0 = r.corner - point;
  R facing = dot(normalize(cross(u, v)), c0);
  if ((r.corner_w > R(0.5) && facing >= 0) || std::fabs(facing) <= R(1e-6)) return 0;
  V3<R> d1 = c0 + u, d2 = c0 + u + v, d3 = c0 + v;
  if (dot(normal, c0) >= 0 && dot(normal, d1) >= 0 && dot(normal, d2) >= 0 && dot(normal, d3) >= 0) {
    V3<R> a0 = normalize(c0), a1 = normalize(d1), a2 = normalize(d2), a3 = normalize(d3);
    R sum = 0;
    sum += lambert_edge_unit(normal, a0, a1);
    sum += lambert_edge_unit(normal, a1, a2);
    sum += lambert_edge_unit(normal, a2, a3);
    sum += lambert_edge_unit(normal, a3, a0);
    return std::fabs(R(0.5) * sum);
  }
  V3<R> d[4] = {c0, c0 + u, c0 + u + v, c0 + v};
  return clipped_quad_weight(normal, d);
}

// sphere_unshadowed (:937-952)
template <class R> R sphere_unshadowed(V3<R> point, V3<R> normal, const Light<R>& r) {
  V3<R> to_center = r.corner - point;
  R d2 = dot(to_center, to_center);
  R radius = r.edge_u.x;
  if (d2 <= radius * radius) return 0;
  R sin2 = radius * radius / d2;
  R cos_t = clampv(dot(normal, to_center) * (R(1) / std::sqrt(d2)), R(-1), R(1));
  const R PI = R(3.14159265);
  if (cos_t * cos_t > sin2) return PI * sin2 * std::max(cos_t, R(0));
  R sin_t = std::sqrt(R(1) - cos_t * cos_t);
  R x = std::sqrt(R(1) / sin2 - R(1));
  R y = clampv(-x * cos_t / sin_t, R(-1), R(1));
  R q = sin_t * std::sqrt(R(1) - y * y);
  return std::max((cos_t * std::acos(y) - x * q) * sin2 + std::atan(q / x), R(0));
}

// unshadowed_rect (:2135-2141): the fraction's denominator.
template <class R> R unshadowed_rect(V3<R> point, V3<R> normal, const Light<R>& r) {
  if (!faces_light(r, point, normal)) return 0;
  if (is_sphere(r)) return spot_falloff(r, normalize(point - r.corner)) * sphere_unshadowed(point, normal, r);
  return rect_open(point, normal, r);
}

// The fraction of each bin inside the disk inscribed in a sphere light's
// window (the WGSL's DISK table, mask_cones.wgsl:888-897): computed here
// from the geometry (circle of radius 4 bins centred on the 8x8 grid, each
// cell's covered area by fine quadrature) and rounded to the table's six
// decimals.
static const double* disk_table() {
  static double table[BINS];
  static bool init = false;
  if (!init) {
    const int S = 2000;  // samples per cell side (midpoint rule on the circle's chord)
    for (uint32_t b = 0; b < BINS; ++b) {
      int col = b % 8, row = b / 8;
      double area = 0;
      for (int i = 0; i < S; ++i) {
        // Exact chord length in y at this x: the integral over x of the
        // vertical overlap of [row, row+1] with the circle at x.
        double x = col + (i + 0.5) / S - 4.0;
        double h2 = 16.0 - x * x;
        if (h2 <= 0) continue;
        double h = std::sqrt(h2);
        double y0 = std::max((double)row - 4.0, -h), y1 = std::min((double)row + 1 - 4.0, h);
        if (y1 > y0) area += (y1 - y0) / S;
      }
      table[b] = std::round(area * 1e6) / 1e6;
    }
    init = true;
  }
  return table;
}

// sphere_open_share (:957-972)
template <class R> R sphere_open_share(const Cone<R>& c, V3<R> normal, const R* cov, bool wide_clipped) {
  const double* disk = disk_table();
  R total = 0, open = 0, g = R(GRID);
  for (uint32_t b = 0; b < BINS; ++b) {
    R m = wide_clipped ? R(1) : R(float(disk[b]));
    if (m <= 0) continue;
    V3<R> d = direction(c, (R(b % GRID) + R(0.5)) / g, (R(b / GRID) + R(0.5)) / g);
    R l2 = dot(d, d);
    R w = m * std::max(dot(normal, d), R(0)) / (l2 * l2);
    total += w;
    open += w * (R(1) - cov[b]);
  }
  if (total <= 0) return 1;
  return open / total;
}

template <class R> struct LightCone {
  Cone<R> c;
  bool ok = false;
  bool wide_clipped = false;
  bool wide_window = false;
};

// light_cone_sphere (:902-931)
template <class R> LightCone<R> light_cone_sphere(V3<R> apex, const Light<R>& r, R wide_extent) {
  LightCone<R> out;
  V3<R> to_center = r.corner - apex;
  R d = length(to_center);
  R radius = r.edge_u.x;
  if (d <= radius * R(1.0001)) return out;
  V3<R> forward = to_center / d;
  R s = radius / d;
  R t = s / std::sqrt(std::max(R(1) - s * s, R(1e-12)));
  out.wide_clipped = R(2) * t > wide_extent;
  out.wide_window = out.wide_clipped;
  t = std::min(t, R(0.5) * wide_extent);
  V3<R> helper = std::fabs(forward.x) > R(0.9) ? V3<R>{0, 1, 0} : V3<R>{1, 0, 0};
  V3<R> right = normalize(cross(helper, forward));
  Cone<R>& c = out.c;
  c.apex = apex;
  c.right = right;
  c.up = cross(forward, right);
  c.forward = forward;
  c.window[0] = -t;
  c.window[1] = -t;
  c.window[2] = t;
  c.window[3] = t;
  c.far_normal = forward;
  c.far_offset = dot(forward, apex) + (d - radius * s) * (R(1) - R(1e-5));
  bound_cone(c, forward);
  out.ok = true;
  return out;
}

// light_cone_rect (:974-1042)
template <class R> LightCone<R> light_cone_rect(V3<R> apex, const Light<R>& r, R wide_extent) {
  if (is_sphere(r)) return light_cone_sphere(apex, r, wide_extent);
  LightCone<R> out;
  V3<R> corner0 = r.corner, edge_u = r.edge_u, edge_v = r.edge_v;
  V3<R> forward = normalize(cross(edge_u, edge_v));
  if (r.corner_w > R(0.5) && dot(forward, apex - corner0) <= 0) return out;
  if (dot(forward, corner0 - apex) < 0) forward = -forward;
  R dist = dot(forward, corner0 - apex);
  if (dist <= R(1e-6)) return out;
  V3<R> right = normalize(edge_u);
  V3<R> up = cross(forward, right);
  V3<R> rel = corner0 - apex;
  R lo[2] = {R(3.4e38), R(3.4e38)}, hi[2] = {R(-3.4e38), R(-3.4e38)};
  for (uint32_t k = 0; k < 4; ++k) {
    V3<R> corner = rel + edge_u * R(k & 1u) + edge_v * R((k >> 1u) & 1u);
    R u = dot(right, corner) / dist, v = dot(up, corner) / dist;
    lo[0] = std::min(lo[0], u);
    lo[1] = std::min(lo[1], v);
    hi[0] = std::max(hi[0], u);
    hi[1] = std::max(hi[1], v);
  }
  R extent[2] = {hi[0] - lo[0], hi[1] - lo[1]};
  R foot[2] = {std::min(std::max(R(0), lo[0]), hi[0]), std::min(std::max(R(0), lo[1]), hi[1])};
  V3<R> mid = normalize(V3<R>{R(0.5) * (lo[0] + hi[0]), R(0.5) * (lo[1] + hi[1]), R(1)});
  R cos_wide = 1;
  for (uint32_t k = 0; k < 4; ++k) {
    V3<R> q{(k & 1u) ? hi[0] : lo[0], (k & 2u) ? hi[1] : lo[1], R(1)};
    cos_wide = std::min(cos_wide, dot(mid, normalize(q)));
  }
  R size = wide_extent;
  out.wide_window = extent[0] > size || extent[1] > size;
  out.wide_clipped = out.wide_window && cos_wide < R(0.8660254);
  if (out.wide_clipped) {
    for (int i = 0; i < 2; ++i) {
      if (extent[i] > size) {
        R keep = std::min(std::max(foot[i] - R(0.5) * size, lo[i]), hi[i] - size);
        lo[i] = keep;
        hi[i] = keep + size;
      }
    }
  }
  Cone<R>& c = out.c;
  c.apex = apex;
  c.right = right;
  c.up = up;
  c.forward = forward;
  c.window[0] = lo[0];
  c.window[1] = lo[1];
  c.window[2] = hi[0];
  c.window[3] = hi[1];
  c.far_normal = forward;
  c.far_offset = dot(forward, apex) + dist * (R(1) - R(1e-5));
  V3<R> axis = normalize(rel + (edge_u + edge_v) * R(0.5));
  if (out.wide_clipped) axis = normalize(direction(c, R(0.5), R(0.5)));
  bound_cone(c, axis);
  out.ok = true;
  return out;
}

template <class R> struct ConeResult {
  R cov[BINS];
  R irradiance;
  R fraction;
  R unshadowed;
  Work work;
};

// hit_irradiance_rect (:2125-2128) through cone_irradiance_rect (:1286-1321),
// plus the lighting cache's ratio (vc_bake, :3453-3510, static light): the
// visible fraction of the unshadowed light, exactly 1 for an empty cone and 0
// for a full one.
// `own`: the receiver's own triangle + 1 (0: none). With prm.back_facing, a
// light that gives the receiver no unshadowed light but lies in front of a
// horizon facing it is traced with that horizon (the normal replaced by the
// direction to the light's centre) past the receiver's own triangle; the
// ratio is then the share seen past it and the light 0 (vc_bake :3476-3531).
template <class R> void visibility_cone(const Scene& s, V3<R> point, V3<R> normal, const Light<R>& r,
                                        const Params<R>& prm, ConeResult<R>& out, uint32_t own = 0) {
  bool back = false;
  uint32_t skip = NONE;
  if (prm.back_facing && own != 0) {
    const V3<R> toward = normalize(light_center(r) - point);
    if (unshadowed_rect(point, normal, r) <= 0 && faces_light(r, point, toward)) {
      back = true;
      normal = toward;
      skip = own - 1;
    }
  }
  R spot = spot_falloff(r, normalize(point - light_center(r)));
  bool on = spot > 0 && faces_light(r, point, normal);
  LightCone<R> lc = light_cone_rect(point, r, prm.wide_extent);
  bool traced = on && lc.ok;
  Walk<R> wk;
  std::fill(wk.cov, wk.cov + BINS, R(0));
  wk.cone_cap = lc.wide_window ? prm.wide_cone_cap : prm.light_cone_cap;
  wk.prefilter = prm.prefilter;
  wk.object_prefilter = prm.object_prefilter;
  wk.accumulate = prm.accumulate;
  wk.work.skip = skip;
  if (traced) scene_coverage(s, lc.c, wk, prm.hierarchy);
  if (wk.cone_work >= wk.cone_cap && traced) wk.work.flags |= 1;
  if (traced && wk.cone_work >= wk.cone_cap && lc.wide_window && !lc.wide_clipped) {
    std::fill(wk.cov, wk.cov + BINS, R(1));
    wk.full = BINS;
  }
  bool last_empty = true, last_full = true;
  for (uint32_t b = 0; b < BINS; ++b) {
    if (wk.cov[b] > 0) last_empty = false;
    if (wk.cov[b] < 1) last_full = false;
  }
  R value = 0;
  if (traced) {
    if (is_sphere(r)) {
      value = sphere_unshadowed(point, normal, r) * sphere_open_share(lc.c, normal, wk.cov, lc.wide_clipped);
    } else {
      R visible = cone_visible(lc.c, normal, wk.cov);
      if (lc.wide_clipped) {  // wide_visible (:1070-1073)
        R kept = window_open(lc.c, normal);
        visible = (kept > R(1e-9) ? visible / kept : R(1)) * rect_open(point, normal, r);
      }
      value = visible;
    }
  }
  value *= spot;
  R open = unshadowed_rect(point, normal, r);
  R ratio = open > 0 ? clampv(value / open, R(0), R(1)) : R(1);
  if (open > 0 && last_empty) ratio = 1;
  if (open > 0 && last_full) ratio = 0;
  std::copy(wk.cov, wk.cov + BINS, out.cov);
  out.irradiance = back ? R(0) : value;
  out.fraction = ratio;
  out.unshadowed = open;
  out.work = wk.work;
}

// Sky light (:1323-1511), a uniform sky in world axes without prefiltering.
constexpr float SKY_FAR = 1e7f;  // :1326

// sky_face (:1444-1478): cube face f around `apex`; returns whether any of its
// window's corner directions lies above the horizon of `normal`.
// `frame` (nullable): the rotation rows of the transform of the object the
// receiver lies on (sky_frame, :1432-1456): the face's axes are turned to
// world space by rotate_to_world (:65-67).
template <class R> bool sky_face(uint32_t f, V3<R> apex, V3<R> normal, bool horizon_cull, Cone<R>& c,
                                 const float* frame = nullptr) {
  const uint32_t axis = f / 2;
  const R sign = (f & 1u) ? R(-1) : R(1);
  R fw[3] = {0, 0, 0}, rt[3] = {0, 0, 0};
  fw[axis] = sign;
  rt[(axis + 1) % 3] = 1;
  V3<R> forward{fw[0], fw[1], fw[2]}, right{rt[0], rt[1], rt[2]};
  if (frame) {
    auto to_world = [&](V3<R> d) {
      return V3<R>{R(frame[0]) * d.x + R(frame[1]) * d.y + R(frame[2]) * d.z,
                   R(frame[4]) * d.x + R(frame[5]) * d.y + R(frame[6]) * d.z,
                   R(frame[8]) * d.x + R(frame[9]) * d.y + R(frame[10]) * d.z};
    };
    forward = to_world(forward);
    right = to_world(right);
  }
  c.apex = apex;
  c.right = right;
  c.up = cross(forward, right);
  c.forward = forward;
  c.window[0] = -1;
  c.window[1] = -1;
  c.window[2] = 1;
  c.window[3] = 1;
  c.far_normal = forward;
  c.far_offset = dot(forward, apex) + R(SKY_FAR);
  c.horizon = horizon_cull ? normal : V3<R>{0, 0, 0};
  bound_cone(c, forward);
  bool above = false;
  for (uint32_t k = 0; k < 4; ++k)
    if (dot(normal, direction(c, R(k & 1u), R(k >> 1))) > 0) above = true;
  return above;
}

// sky_face_coverage and sky_face_light (:1482-1498) for face f: the face's
// coverage (no walk cap; independent occluders unless `combine_max`) and its
// light per unit sky radiance.
template <class R> R sky_face_irradiance(const Scene& s, uint32_t f, V3<R> point, V3<R> normal, uint32_t hierarchy,
                                         bool combine_max, bool horizon_cull, R prefilter, bool object_prefilter,
                                         R* cov_out, Work* work, const float* frame = nullptr,
                                         uint32_t accumulate = kSumWalkOrder) {
  Cone<R> c;
  const bool above = sky_face(f, point, normal, horizon_cull, c, frame);
  Walk<R> wk;
  wk.accumulate = accumulate;
  std::fill(wk.cov, wk.cov + BINS, R(0));
  wk.independent = !combine_max;
  wk.prefilter = prefilter;
  wk.object_prefilter = object_prefilter;
  if (above) scene_coverage(s, c, wk, hierarchy);
  if (cov_out) std::copy(wk.cov, wk.cov + BINS, cov_out);
  if (work) *work = wk.work;
  if (!above) return 0;
  R blocked = 0;
  for (uint32_t b = 0; b < BINS; ++b)
    if (wk.cov[b] > 0) blocked += wk.cov[b] * clipped_bin_weight(c, normal, b);
  return std::max(clipped_window_weight(c, normal) - blocked, R(0));
}

// ---------------------------------------------------------------------------
// The reference CPU path: cone3.rs, coverage.rs, bvh.rs (FP32).
// ---------------------------------------------------------------------------

namespace cpu {
using V = V3<float>;

struct Plane {
  V normal;
  float offset;
  float signed_distance(V p) const { return offset - dot(normal, p); }
};

struct PyramidCone {  // cone3.rs:46-64
  V apex, right, up, forward;
  float window[4];
  float near_;
  Plane far_;
  float weights[BINS];
  V direction(float s, float t) const {
    return forward + right * (window[0] + s * (window[2] - window[0])) + up * (window[1] + t * (window[3] - window[1]));
  }
  V to_local(V p) const {
    V d = p - apex;
    return {dot(right, d), dot(up, d), dot(forward, d)};
  }
};

// projected_solid_angle (cone3.rs:69-82)
static float projected_solid_angle(V n, const V* verts, int count) {
  float sum = 0;
  for (int i = 0; i < count; ++i) {
    V a = normalize(verts[i]), b = normalize(verts[(i + 1) % count]);
    V g = cross(a, b);
    float len = length(g);
    if (len > 1e-12f) sum += std::atan2(len, dot(a, b)) * dot(n, g / len);
  }
  return std::fabs(0.5f * sum);
}

// toward_rect_light (cone3.rs:197-247)
static bool toward_rect_light(V apex, V corner, V edge_u, V edge_v, V receiver_normal, PyramidCone& cone) {
  V forward = normalize(cross(edge_u, edge_v));
  if (dot(forward, corner - apex) < 0) forward = -forward;
  float dist = dot(forward, corner - apex);
  if (dist <= 1e-6f) return false;
  V right = normalize(edge_u), up = cross(forward, right), rel = corner - apex;
  V corners[4] = {rel, rel + edge_u, rel + edge_v, rel + edge_u + edge_v};
  float u0 = FLT_MAX, v0 = FLT_MAX, u1 = -FLT_MAX, v1 = -FLT_MAX;
  for (V c : corners) {
    float u = dot(right, c) / dist, v = dot(up, c) / dist;
    u0 = std::min(u0, u);
    v0 = std::min(v0, v);
    u1 = std::max(u1, u);
    v1 = std::max(v1, v);
  }
  cone.apex = apex;
  cone.right = right;
  cone.up = up;
  cone.forward = forward;
  cone.window[0] = u0;
  cone.window[1] = v0;
  cone.window[2] = u1;
  cone.window[3] = v1;
  cone.near_ = 1e-4f;
  cone.far_ = {forward, dot(forward, apex) + dist * (1.0f - 1e-5f)};
  for (uint32_t bin = 0; bin < BINS; ++bin) {
    float col = float(bin % GRID), row = float(bin / GRID), g = float(GRID);
    V quad[4] = {cone.direction(col / g, row / g), cone.direction((col + 1) / g, row / g),
                 cone.direction((col + 1) / g, (row + 1) / g), cone.direction(col / g, (row + 1) / g)};
    cone.weights[bin] = projected_solid_angle(receiver_normal, quad, 4);
  }
  return true;
}

static float total_weight(const PyramidCone& c) {
  float s = 0;
  for (float w : c.weights) s += w;
  return s;
}

// may_touch / may_touch_box (cone3.rs:267-307)
template <int N> static bool may_touch_points(const PyramidCone& c, const V (&pts)[N]) {
  bool all_far = true;
  for (const V& p : pts)
    if (!(c.far_.signed_distance(p) < 0)) all_far = false;
  if (all_far) return false;
  V local[N];
  bool all_near = true;
  for (int i = 0; i < N; ++i) {
    local[i] = c.to_local(pts[i]);
    if (!(local[i].z < c.near_)) all_near = false;
  }
  if (all_near) return false;
  const float* w = c.window;
  auto outside = [&](auto f) {
    for (int i = 0; i < N; ++i)
      if (!(f(local[i]) < 0)) return false;
    return true;
  };
  return !(outside([&](V p) { return p.x - w[0] * p.z; }) || outside([&](V p) { return w[2] * p.z - p.x; }) ||
           outside([&](V p) { return p.y - w[1] * p.z; }) || outside([&](V p) { return w[3] * p.z - p.y; }));
}

static bool may_touch(const PyramidCone& c, const V (&tri)[3]) { return may_touch_points<3>(c, tri); }

static bool may_touch_box(const PyramidCone& c, V mn, V mx) {
  V corners[8];
  for (int i = 0; i < 8; ++i)
    corners[i] = {(i & 1) ? mx.x : mn.x, (i & 2) ? mx.y : mn.y, (i & 4) ? mx.z : mn.z};
  return may_touch_points<8>(c, corners);
}

template <class P, class D> static int clip_poly(const P* in, int n, P* out, D d) {  // Poly::clip (cone3.rs:110-126)
  int m = 0;
  for (int i = 0; i < n; ++i) {
    P a = in[i], b = in[(i + 1) % n];
    float da = d(a), db = d(b);
    if (da >= 0 && m < POLY_CAP) out[m++] = a;
    if ((da >= 0) != (db >= 0) && m < POLY_CAP) {
      float f = da / (da - db);
      out[m++] = P{a.x + (b.x - a.x) * f, a.y + (b.y - a.y) * f};
    }
  }
  return m;
}

// draw_edge (cone3.rs:140-190), weight 1
static void draw_edge(float* buf, V2<float> p0, V2<float> p1) {
  if (std::fabs(p0.y - p1.y) <= FLT_EPSILON) return;
  float dir = 1;
  if (!(p0.y < p1.y)) {
    dir = -1;
    std::swap(p0, p1);
  }
  float dxdy = (p1.x - p0.x) / (p1.y - p0.y);
  float x = p0.x;
  size_t y_end = std::min((size_t)std::ceil(p1.y), (size_t)GRID);
  for (size_t y = (size_t)p0.y; y < y_end; ++y) {
    size_t row = y * GRID;
    float dy = std::min(float(y + 1), p1.y) - std::max(float(y), p0.y);
    float x_next = clampv(x + dxdy * dy, 0.0f, float(GRID));
    float d = dy * dir;
    float x0 = x < x_next ? x : x_next, x1 = x < x_next ? x_next : x;
    float x0_floor = std::floor(x0);
    size_t x0i = (size_t)x0_floor;
    float x1_ceil = std::ceil(x1);
    size_t x1i = (size_t)x1_ceil;
    if (x1i <= x0i + 1) {
      float xmf = 0.5f * (x + x_next) - x0_floor;
      buf[row + x0i] += d - d * xmf;
      buf[row + x0i + 1] += d * xmf;
    } else {
      float s = 1.0f / (x1 - x0);
      float x0f = x0 - x0_floor;
      float a0 = 0.5f * s * (1.0f - x0f) * (1.0f - x0f);
      float x1f = x1 - x1_ceil + 1.0f;
      float am = 0.5f * s * x1f * x1f;
      buf[row + x0i] += d * a0;
      if (x1i == x0i + 2) {
        buf[row + x0i + 1] += d * (1.0f - a0 - am);
      } else {
        float a1 = s * (1.5f - x0f);
        buf[row + x0i + 1] += d * (a1 - a0);
        for (size_t xi = x0i + 2; xi < x1i - 1; ++xi) buf[row + xi] += d * s;
        float a2 = a1 + float(x1i - x0i - 3) * s;
        buf[row + x1i - 1] += d * (1.0f - a2 - am);
      }
      buf[row + x1i] += d * am;
    }
    x = x_next;
  }
}

// rasterize (cone3.rs:360-393)
static bool rasterize(const PyramidCone& c, float* buf, const V (&tri)[3]) {
  V a[POLY_CAP], b[POLY_CAP];
  int n = 0;
  {  // far clip: keep signed_distance >= 0
    for (int i = 0; i < 3; ++i) {
      V p = tri[i], q = tri[(i + 1) % 3];
      float da = c.far_.signed_distance(p), db = c.far_.signed_distance(q);
      if (da >= 0) a[n++] = p;
      if ((da >= 0) != (db >= 0)) a[n++] = p + (q - p) * (da / (da - db));
    }
  }
  for (int i = 0; i < n; ++i) a[i] = c.to_local(a[i]);
  int m = 0;
  for (int i = 0; i < n; ++i) {  // near clip: keep z - near >= 0
    V p = a[i], q = a[(i + 1) % n];
    float da = p.z - c.near_, db = q.z - c.near_;
    if (da >= 0 && m < POLY_CAP) b[m++] = p;
    if ((da >= 0) != (db >= 0) && m < POLY_CAP) b[m++] = p + (q - p) * (da / (da - db));
  }
  if (m < 3) return false;
  const float* w = c.window;
  float su = float(GRID) / (w[2] - w[0]), sv = float(GRID) / (w[3] - w[1]), g = float(GRID);
  V2<float> q0[POLY_CAP], q1[POLY_CAP];
  for (int i = 0; i < m; ++i) q0[i] = {(b[i].x / b[i].z - w[0]) * su, (b[i].y / b[i].z - w[1]) * sv};
  int k = m;
  k = clip_poly(q0, k, q1, [](V2<float> p) { return p.x; });
  k = clip_poly(q1, k, q0, [g](V2<float> p) { return g - p.x; });
  k = clip_poly(q0, k, q1, [](V2<float> p) { return p.y; });
  k = clip_poly(q1, k, q0, [g](V2<float> p) { return g - p.y; });
  if (k < 3) return false;
  auto at = [&](int i) {
    V2<float> p = q0[i % k];
    return V2<float>{clampv(p.x, 0.0f, g), clampv(p.y, 0.0f, g)};
  };
  for (int i = 0; i < k; ++i) draw_edge(buf, at(i), at(i + 1));
  return true;
}

struct CoverageMask {  // coverage.rs:22-126
  uint64_t full = 0;
  float partial[BINS] = {};
  void add_bin(uint32_t bin, float fraction) {
    if (fraction >= 1.0f)
      full |= 1ull << bin;
    else if (fraction > partial[bin])
      partial[bin] = fraction;
  }
  bool is_full() const { return full == ~0ull; }
  float visible_weighted(const float* weights) const {
    float visible = 0;
    for (uint32_t bin = 0; bin < BINS; ++bin)
      if (!((full >> bin) & 1)) visible += (1.0f - partial[bin]) * weights[bin];
    return visible;
  }
};

// add_mesh (cone3.rs:317-341): front-facing triangles of one mesh summed.
static void add_mesh(const PyramidCone& c, CoverageMask& mask, const std::vector<const float*>& tris) {
  float buf[BINS + 4] = {};
  bool touched = false;
  for (const float* t : tris) {
    V tri[3] = {{t[0], t[1], t[2]}, {t[4], t[5], t[6]}, {t[8], t[9], t[10]}};
    V normal = cross(tri[1] - tri[0], tri[2] - tri[0]);
    if (dot(normal, c.apex - tri[0]) <= 0) continue;
    touched |= rasterize(c, buf, tri);
  }
  if (touched) {
    float running = 0;
    for (uint32_t bin = 0; bin < BINS; ++bin) {
      running += buf[bin];
      float covered = std::fabs(running);
      if (covered > 1e-6f) mask.add_bin(bin, std::min(covered, 1.0f));
    }
  }
}

// bvh.rs: leaf-4 median BVH over all triangles of all meshes.
struct Bvh {
  struct N {
    V mn, mx;
    uint32_t start, count;
  };
  std::vector<N> nodes;
  std::vector<uint32_t> tri;  // triangle index (into the scene) per slot
  std::vector<uint32_t> mesh_of;
};

static void bvh_split(const Scene& s, Bvh& b, size_t node, std::vector<uint32_t>& items, size_t start, size_t end) {
  V mn{FLT_MAX, FLT_MAX, FLT_MAX}, mx{-FLT_MAX, -FLT_MAX, -FLT_MAX};
  V cmin = mn, cmax = mx;
  for (size_t i = start; i < end; ++i) {
    V t[3];
    for (int k = 0; k < 3; ++k) t[k] = tri_vertex<float>(s, items[i], k);
    for (int k = 0; k < 3; ++k) {
      mn = vmin(mn, t[k]);
      mx = vmax(mx, t[k]);
    }
    V c = (t[0] + t[1] + t[2]) / 3.0f;
    cmin = vmin(cmin, c);
    cmax = vmax(cmax, c);
  }
  b.nodes[node].mn = mn;
  b.nodes[node].mx = mx;
  if (end - start <= 4) {
    b.nodes[node].start = (uint32_t)start;
    b.nodes[node].count = (uint32_t)(end - start);
    return;
  }
  V e = cmax - cmin;
  int axis = (e.x >= e.y && e.x >= e.z) ? 0 : (e.y >= e.z ? 1 : 2);
  size_t mid = (start + end) / 2;
  auto key = [&](uint32_t t) {
    float k = 0;
    for (int j = 0; j < 3; ++j) k += (&s.tris[12 * (size_t)t + 4 * j])[axis];
    return k;
  };
  std::nth_element(items.begin() + start, items.begin() + mid, items.begin() + end, [&](uint32_t a, uint32_t c) {
    float ka = key(a), kc = key(c);
    return ka < kc || (ka == kc && a < c);
  });
  size_t left = b.nodes.size();
  b.nodes.push_back({});
  b.nodes.push_back({});
  b.nodes[node].start = (uint32_t)left;
  b.nodes[node].count = 0;
  bvh_split(s, b, left, items, start, mid);
  bvh_split(s, b, left + 1, items, mid, end);
}

static Bvh* build_bvh(const Scene& s) {
  Bvh* b = new Bvh;
  size_t total = s.tris.size() / 12;
  std::vector<uint32_t> items(total);
  std::iota(items.begin(), items.end(), 0u);
  b->nodes.assign(1, {});
  if (total) bvh_split(s, *b, 0, items, 0, total);
  b->tri = items;
  std::vector<uint32_t> mesh_of_tri(total);
  for (uint32_t m = 0; m < s.nmeshes; ++m)
    for (uint32_t t = s.ranges[4 * m]; t < s.ranges[4 * m] + s.ranges[4 * m + 1]; ++t) mesh_of_tri[t] = m;
  for (uint32_t t : items) b->mesh_of.push_back(mesh_of_tri[t]);
  return b;
}

// Receiver::new / with_bvh + Receiver::masked (experiments/room3d/src/lib.rs:180-243):
// irradiance per unit radiance and the cone's total weight.
static void receiver_masked(const Scene& s, const Bvh* bvh, V point, V normal, V corner, V eu, V ev, float& visible,
                            float& total, uint32_t& visited) {
  PyramidCone cone;
  visited = 0;
  if (!toward_rect_light(point, corner, eu, ev, normal, cone)) {
    visible = 0;
    total = 1;  // m2_gate1.rs:42: (0, 1) for receivers without a cone
    return;
  }
  std::vector<std::pair<uint32_t, const float*>> found;
  if (bvh) {
    std::vector<uint32_t> stack{0};
    while (!stack.empty()) {
      uint32_t i = stack.back();
      stack.pop_back();
      visited++;
      const auto& n = bvh->nodes[i];
      if (!may_touch_box(cone, n.mn, n.mx)) continue;
      if (n.count > 0) {
        for (uint32_t t = n.start; t < n.start + n.count; ++t) {
          const float* p = s.tris.data() + 12 * (size_t)bvh->tri[t];
          V tri[3] = {{p[0], p[1], p[2]}, {p[4], p[5], p[6]}, {p[8], p[9], p[10]}};
          if (may_touch(cone, tri)) found.push_back({bvh->mesh_of[t], p});
        }
      } else {
        stack.push_back(n.start);
        stack.push_back(n.start + 1);
      }
    }
    std::stable_sort(found.begin(), found.end(), [](auto& a, auto& b) { return a.first < b.first; });
  } else {
    for (uint32_t m = 0; m < s.nmeshes; ++m)
      for (uint32_t t = s.ranges[4 * m]; t < s.ranges[4 * m] + s.ranges[4 * m + 1]; ++t) {
        const float* p = s.tris.data() + 12 * (size_t)t;
        V tri[3] = {{p[0], p[1], p[2]}, {p[4], p[5], p[6]}, {p[8], p[9], p[10]}};
        if (may_touch(cone, tri)) found.push_back({m, p});
      }
  }
  CoverageMask mask;
  size_t i = 0;
  while (i < found.size()) {
    size_t j = i;
    std::vector<const float*> tris;
    while (j < found.size() && found[j].first == found[i].first) tris.push_back(found[j++].second);
    add_mesh(cone, mask, tris);
    if (mask.is_full()) break;
    i = j;
  }
  visible = mask.visible_weighted(cone.weights);
  total = total_weight(cone);
}
}  // namespace cpu

// Run `fn(i)` for i in [0, n) on `threads` threads, static contiguous chunks
// (the reference's par_map partitions rows among threads the same way).
template <class F> static void parallel_for(uint64_t n, int threads, F fn) {
  if (threads <= 1 || n < 2) {
    for (uint64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<uint64_t> next{0};
  const uint64_t chunk = 64;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        uint64_t start = next.fetch_add(chunk);
        if (start >= n) break;
        uint64_t end = std::min(n, start + chunk);
        for (uint64_t i = start; i < end; ++i) fn(i);
      }
    });
  for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------
// Camera pass: the receivers at a pinhole camera's primary hits. Input
// preparation, restated from the reference's camera pass (camera_dir
// mask_cones.wgsl:1724-1729, primary_hit :1732-1760, the lifted hit point
// surface_offset :2062-2064 and the facing normal of per_pixel_hit_color
// :2275-2277) over this file's own hierarchies, so that the CPU legs can build
// their inputs without the library. Every operation is the FP32 one the
// library's host caster performs, in the same order, with the same
// traversal order (right child popped first), so the two give the same
// receivers bit for bit.
// ---------------------------------------------------------------------------
namespace camera {

using V = V3<float>;

// The ray (origin o, inverse direction inv) meets the box nearer than limit.
inline bool slab(V o, V inv, const Node& n, float limit) {
  float near_t = 0.0f, far_t = limit;
  const float oc[3] = {o.x, o.y, o.z}, ic[3] = {inv.x, inv.y, inv.z};
  for (int k = 0; k < 3; ++k) {
    float a = (n.lo[k] - oc[k]) * ic[k];
    float b = (n.hi[k] - oc[k]) * ic[k];
    if (a > b) std::swap(a, b);
    near_t = std::max(near_t, a);
    far_t = std::min(far_t, b);
    if (near_t > far_t) return false;
  }
  return true;
}

// Moller and Trumbore's ray-triangle test: the distance, or -1 for a miss.
inline float hit_distance(V o, V d, V v0, V v1, V v2) {
  const V e1 = v1 - v0, e2 = v2 - v0;
  const V p = cross(d, e2);
  const float det = dot(e1, p);
  if (std::fabs(det) < 1e-12f) return -1.0f;
  const float inv = 1.0f / det;
  const V s = o - v0;
  const float u = dot(s, p) * inv;
  if (u < 0.0f || u > 1.0f) return -1.0f;
  const V q = cross(s, e1);
  const float v = dot(d, q) * inv;
  if (v < 0.0f || u + v > 1.0f) return -1.0f;
  const float t = dot(e2, q) * inv;
  return t > 0.0f ? t : -1.0f;
}

struct Nearest {
  float t = FLT_MAX;
  uint32_t tri = NONE;
  uint32_t xform = NONE;
  uint32_t object = NONE;
};

inline V tri_at(const Scene& s, uint32_t t, int k) {
  const float* p = &s.tris[12 * (size_t)t + 4 * k];
  return V{p[0], p[1], p[2]};
}

void nearest_hit(const Scene& s, V o, V d, Nearest& h) {
  const V inv{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  std::vector<uint32_t> objects{0};
  std::vector<uint32_t> tri_nodes;
  while (!objects.empty()) {
    const Node& n = s.nodes[objects.back()];
    objects.pop_back();
    if (!slab(o, inv, n, h.t)) continue;
    if (n.info[1] == 0) {
      objects.push_back(n.info[0]);
      objects.push_back(n.info[0] + 1);
      continue;
    }
    for (uint32_t k = n.info[0]; k < n.info[0] + n.info[1]; ++k) {
      const uint32_t* r = &s.ranges[4 * s.items[k]];
      if (r[2] == NONE) continue;
      V ro = o, rd = d, rinv = inv;
      if (r[3] != NONE) {  // the ray in the placed object's space: R^T (o - t) / s, R^T d / s
        const float* x = &s.xforms[16 * (size_t)r[3]];
        const V a{x[0], x[1], x[2]}, b{x[4], x[5], x[6]}, c{x[8], x[9], x[10]}, tr{x[3], x[7], x[11]};
        const float inv_scale = x[13];
        const V q = o - tr;
        ro = (a * q.x + b * q.y + c * q.z) * inv_scale;
        rd = (a * d.x + b * d.y + c * d.z) * inv_scale;
        rinv = V{1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z};
      }
      tri_nodes.assign(1, r[2]);
      while (!tri_nodes.empty()) {
        const Node& b = s.blas[tri_nodes.back()];
        tri_nodes.pop_back();
        if (!slab(ro, rinv, b, h.t)) continue;
        if (b.info[1] == 0) {
          tri_nodes.push_back(b.info[0]);
          tri_nodes.push_back(b.info[0] + 1);
          continue;
        }
        for (uint32_t j = b.info[0]; j < b.info[0] + b.info[1]; ++j) {
          const uint32_t t = s.blas_items[j];
          const float dist = hit_distance(ro, rd, tri_at(s, t, 0), tri_at(s, t, 1), tri_at(s, t, 2));
          if (dist > 0.0f && dist < h.t) {
            h.t = dist;
            h.tri = t;
            h.xform = r[3];
            h.object = s.items[k];
          }
        }
      }
    }
  }
}

// camera: eye.xyz, target.xyz, up.xyz, vertical fov in degrees. Per pixel
// (row-major) a receiver (point.xyz, the hit object's index as bits;
// normal.xyz, the hit triangle's index + 1 as bits) and 1 if the ray hit.
void primary_hits(const Scene& s, const float* camera, uint32_t width, uint32_t height, float* out8, uint8_t* hit,
                  int threads) {
  const V eye{camera[0], camera[1], camera[2]}, target{camera[3], camera[4], camera[5]};
  const V up_world{camera[6], camera[7], camera[8]};
  const float tan_half = std::tan(camera[9] * 3.14159265358979f / 360.0f);
  const V fwd = normalize(target - eye);
  const V right = normalize(cross(fwd, up_world));
  const V up = cross(right, fwd);
  const float aspect = float(width) / float(height);
  parallel_for(height, threads, [&](uint64_t row) {
    for (uint32_t x = 0; x < width; ++x) {
      const float sx = ((float(x) + 0.5f) / float(width) * 2.0f - 1.0f) * tan_half * aspect;
      const float sy = (1.0f - (float(row) + 0.5f) / float(height) * 2.0f) * tan_half;
      const V d = normalize(fwd + right * sx + up * sy);
      Nearest h;
      nearest_hit(s, eye, d, h);
      const size_t i = (size_t)row * width + x;
      float* o = out8 + 8 * i;
      std::fill(o, o + 8, 0.0f);
      hit[i] = h.tri != NONE;
      if (h.tri == NONE) continue;
      const V v0 = tri_at(s, h.tri, 0), v1 = tri_at(s, h.tri, 1), v2 = tri_at(s, h.tri, 2);
      V n = normalize(cross(v1 - v0, v2 - v0));
      if (h.xform != NONE) {  // the object's normal in world space: R n
        const float* x = &s.xforms[16 * (size_t)h.xform];
        n = normalize(V{x[0] * n.x + x[1] * n.y + x[2] * n.z, x[4] * n.x + x[5] * n.y + x[6] * n.z,
                        x[8] * n.x + x[9] * n.y + x[10] * n.z});
      }
      if (dot(n, d) > 0.0f) n = n * -1.0f;
      const V point = (eye + d * h.t) + n * std::max(1e-4f, 2e-6f * h.t);
      const uint32_t own = h.tri + 1u;  // w: the hit object, and the hit triangle + 1, as bits
      o[0] = point.x;
      o[1] = point.y;
      o[2] = point.z;
      std::memcpy(&o[3], &h.object, 4);
      o[4] = n.x;
      o[5] = n.y;
      o[6] = n.z;
      std::memcpy(&o[7], &own, 4);
    }
  });
}

}  // namespace camera

}  // namespace oracle

using namespace oracle;

extern "C" {

int oracle_cpu_masked_with(void* sp, void* bvh_p, const float* receivers, uint64_t npoints, const float* light9,
                           float* visible, float* total, uint32_t* visited, int threads);

// Builds the reference's host layouts from meshes given as 9 floats per
// triangle, `mesh_counts[m]` triangles each, consecutive.
void* oracle_scene_create(const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes) {
  return build_scene(tri9, mesh_counts, nmeshes);
}

// An instanced scene: geometries given as 9 floats per triangle (object
// space), instances as cc_instance records.
void* oracle_scene_create_instanced(const float* tri9, const uint32_t* geometry_counts, uint32_t ngeometries,
                                    const void* instances, uint32_t ninstances, const uint32_t* movable,
                                    uint32_t nmovable) {
  return build_instanced(tri9, geometry_counts, ngeometries, static_cast<const Instance*>(instances), ninstances,
                         movable, nmovable);
}

// Each object's clear (Placement::clear), in its transform's row 3 z; the
// prefiltered samples are rebuilt on their next use.
void oracle_scene_set_clear(void* sp, const float* clear, uint32_t n) {
  Scene* s = static_cast<Scene*>(sp);
  for (uint32_t m = 0; m < n && m < s->object_geometry.size(); ++m) s->xforms[16 * (size_t)s->ranges[4 * m + 3] + 14] = clear[m];
  s->coverage_built = false;
}

void oracle_scene_move(void* sp, const void* placements, float* boxes12) {
  move_objects(static_cast<Scene*>(sp), static_cast<const Instance*>(placements), boxes12);
}

// The cones moved objects may have changed (may_be_shadowed, mask_cones.wgsl:
// 3961-3974, for a point's box): for each (light, point), some mover box, old
// or new, whose shadow region (hierarchy.rs:418-457) holds the point and
// which meets the hull of the point and the light's box (hull_meets,
// :3903-3917). 1 byte per cone, light-major.
void oracle_stale_cones(void* sp, const float* rec8, uint64_t npoints, const float* lights16, uint32_t nlights,
                        const float* boxes12, uint32_t nmovers, uint8_t* out, int threads) {
  const Scene* s = static_cast<const Scene*>(sp);
  typedef std::pair<F3, F3> B;
  const B scene_box{F3{s->nodes[0].lo[0], s->nodes[0].lo[1], s->nodes[0].lo[2]},
                    F3{s->nodes[0].hi[0], s->nodes[0].hi[1], s->nodes[0].hi[2]}};
  auto light_box = [](const float* L) {  // :3887-3898
    F3 c;
    float radius;
    if (L[3] > 1.5f) {
      c = F3{L[0], L[1], L[2]};
      radius = 1.5f * L[4];
    } else {
      c = F3{L[0], L[1], L[2]} + (F3{L[4], L[5], L[6]} + F3{L[8], L[9], L[10]}) * 0.5f;
      radius = 0.5f * (length(F3{L[4], L[5], L[6]}) + length(F3{L[8], L[9], L[10]}));
    }
    const float far = std::max(std::max(std::fabs(c.x), 1.0f), std::max(std::max(std::fabs(c.y), 1.0f), std::max(std::fabs(c.z), 1.0f)));
    radius = radius * 1.001f + 1e-5f * far + 1e-4f;
    return B{c - F3{radius, radius, radius}, c + F3{radius, radius, radius}};
  };
  auto comp = [](const F3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); };
  auto region = [&](const B& m, const B& l, const B& sb, B& out) {  // shadow_region
    const F3 d_lo = m.first - l.second, d_hi = m.second - l.first;
    float t0 = 0.0f, t1 = INFINITY;
    for (int a = 0; a < 3; ++a) {
      float b = comp(d_lo, a), c = comp(sb.second, a) - comp(m.first, a);
      if (b > 0.0f) t1 = std::min(t1, c / b);
      else if (b < 0.0f) t0 = std::max(t0, c / b);
      else if (c < 0.0f) return false;
      b = comp(d_hi, a);
      c = comp(sb.first, a) - comp(m.second, a);
      if (b > 0.0f) t0 = std::max(t0, c / b);
      else if (b < 0.0f) t1 = std::min(t1, c / b);
      else if (c > 0.0f) return false;
    }
    if (t0 > t1 * (1.0f + 1e-6f) + 1e-6f) return false;
    if (!std::isfinite(t1)) {
      out = sb;
      return true;
    }
    const F3 lo = vmax(vmin(m.first + d_lo * t0, m.first + d_lo * t1), sb.first);
    const F3 hi = vmin(vmax(m.second + d_hi * t0, m.second + d_hi * t1), sb.second);
    const float pad = 1e-4f * std::max(std::max(std::max(std::fabs(lo.x), std::fabs(hi.x)),
                                                std::max(std::fabs(lo.y), std::fabs(hi.y))),
                                       std::max(std::max(std::fabs(lo.z), std::fabs(hi.z)), 1.0f));
    out = B{lo - F3{pad, pad, pad}, hi + F3{pad, pad, pad}};
    return true;
  };
  auto hull_meets = [&](const F3& p, const B& l, const B& m) {
    float s0 = 0.0f, s1 = 1.0f;
    for (int a = 0; a < 3; ++a) {
      const float b0 = comp(l.first, a) - comp(p, a), c0 = comp(m.second, a) - comp(p, a);
      if (b0 > 0.0f) s1 = std::min(s1, c0 / b0);
      else if (b0 < 0.0f) s0 = std::max(s0, c0 / b0);
      else if (c0 < 0.0f) return false;
      const float b1 = comp(l.second, a) - comp(p, a), c1 = comp(m.first, a) - comp(p, a);
      if (b1 > 0.0f) s0 = std::max(s0, c1 / b1);
      else if (b1 < 0.0f) s1 = std::min(s1, c1 / b1);
      else if (c1 > 0.0f) return false;
    }
    return s0 <= s1 + 1e-6f;
  };
  for (uint32_t l = 0; l < nlights; ++l) {
    const B lb = light_box(lights16 + 16 * (size_t)l);
    std::vector<B> boxes, regions;
    for (uint32_t b = 0; b < 2 * nmovers; ++b) {
      const float* v = boxes12 + 6 * (size_t)b;
      const B m{F3{v[0], v[1], v[2]}, F3{v[3], v[4], v[5]}};
      B r;
      if (region(m, lb, scene_box, r)) {
        boxes.push_back(m);
        regions.push_back(r);
      }
    }
    parallel_for(npoints, threads, [&](uint64_t p) {
      const F3 pt{rec8[8 * p], rec8[8 * p + 1], rec8[8 * p + 2]};
      uint8_t hit = 0;
      for (size_t k = 0; k < boxes.size() && !hit; ++k) {
        const B& r = regions[k];
        if (pt.x < r.first.x || pt.y < r.first.y || pt.z < r.first.z || pt.x > r.second.x || pt.y > r.second.y ||
            pt.z > r.second.z)
          continue;
        if (hull_meets(pt, lb, boxes[k])) hit = 1;
      }
      out[(size_t)l * npoints + p] = hit;
    });
  }
}

// The scene's transforms (16 floats each) into out (nullable); returns their count.
uint64_t oracle_scene_transforms(void* sp, float* out) {
  Scene* s = static_cast<Scene*>(sp);
  if (out) std::memcpy(out, s->xforms.data(), s->xforms.size() * sizeof(float));
  return s->xforms.size() / 16;
}

void oracle_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

// The prefiltered cones' coverage samples (27 per node) of the triangle-
// hierarchy nodes and, for instanced scenes, the object-hierarchy nodes.
void oracle_scene_coverage(void* sp, float* blas27, float* obj27) {
  Scene* s = static_cast<Scene*>(sp);
  build_coverage(*s);
  if (blas27) std::copy(s->blas_cov.begin(), s->blas_cov.end(), blas27);
  if (obj27) std::copy(s->obj_cov.begin(), s->obj_cov.end(), obj27);
}

// Sizes of the flattened arrays: ntris, nmeshes, nblas, nblas_items, nnodes, nitems.
void oracle_scene_sizes(void* sp, uint64_t* out6) {
  Scene* s = static_cast<Scene*>(sp);
  out6[0] = s->tris.size() / 12;
  out6[1] = s->nmeshes;
  out6[2] = s->blas.size();
  out6[3] = s->blas_items.size();
  out6[4] = s->nodes.size();
  out6[5] = s->items.size();
}

// Copies of the flattened arrays (NodeGpu = 12 x 4 bytes).
void oracle_scene_arrays(void* sp, uint32_t* ranges, void* blas, uint32_t* blas_items, void* nodes, uint32_t* items) {
  Scene* s = static_cast<Scene*>(sp);
  if (ranges) std::memcpy(ranges, s->ranges.data(), s->ranges.size() * 4);
  if (blas) std::memcpy(blas, s->blas.data(), s->blas.size() * sizeof(Node));
  if (blas_items) std::memcpy(blas_items, s->blas_items.data(), s->blas_items.size() * 4);
  if (nodes) std::memcpy(nodes, s->nodes.data(), s->nodes.size() * sizeof(Node));
  if (items) std::memcpy(items, s->items.data(), s->items.size() * 4);
}

struct OracleParams {
  uint32_t hierarchy;
  float wide_extent;
  uint32_t light_cone_cap;
  uint32_t wide_cone_cap;
  float prefilter;            // prefilter_bins (0: exact cones)
  uint32_t object_prefilter;  // object-level splats (instanced scenes)
  uint32_t accumulate;        // AccumulateMode: 0 the reference's walk-order sums, 1 fixed point, 2 double
  uint32_t back_facing;       // 1: vc_bake's estimator for a light below the horizon (receiver normal.w: own triangle + 1)
};

// Visibility of cones (light l, receiver p), cone id c = l * npoints + p,
// in the scalar type `precision` (4: float, 8: double). `cone_ids` (nullable)
// selects a subset; outputs are indexed by position in that subset.
// receivers: 8 floats each (point.xyzw, normal.xyzw); lights: 16 floats each.
// full/any: 2 u32 words per cone (bin b in word b/32, bit b%32).
int oracle_visibility(void* sp, const float* receivers, uint64_t npoints, const float* lights, uint32_t nlights,
                      const OracleParams* prm_in, const uint64_t* cone_ids, uint64_t ncones, int precision,
                      uint32_t* full, uint32_t* any, float* partial, float* irradiance, float* fraction,
                      uint32_t* work, float* unshadowed, int threads) {
  Scene* s = static_cast<Scene*>(sp);
  if (!s || !prm_in) return 1;
  uint64_t total = npoints * nlights;
  uint64_t n = cone_ids ? ncones : total;
  if (prm_in->prefilter > 0.0f) build_coverage(*s);
  auto run = [&](auto zero) {
    using R = decltype(zero);
    Params<R> prm{prm_in->hierarchy, R(prm_in->wide_extent), prm_in->light_cone_cap, prm_in->wide_cone_cap,
                  R(prm_in->prefilter), prm_in->object_prefilter != 0, prm_in->accumulate,
                  prm_in->back_facing != 0};
    parallel_for(n, threads, [&](uint64_t i) {
      uint64_t c = cone_ids ? cone_ids[i] : i;
      uint64_t l = c / npoints, p = c % npoints;
      const float* rc = receivers + 8 * p;
      const float* lt = lights + 16 * l;
      Light<R> L{{R(lt[0]), R(lt[1]), R(lt[2])}, R(lt[3]), {R(lt[4]), R(lt[5]), R(lt[6])}, R(lt[7]),
                 {R(lt[8]), R(lt[9]), R(lt[10])}, R(lt[11])};
      ConeResult<R> res;
      uint32_t own;
      std::memcpy(&own, rc + 7, 4);
      visibility_cone<R>(*s, V3<R>{R(rc[0]), R(rc[1]), R(rc[2])}, V3<R>{R(rc[4]), R(rc[5]), R(rc[6])}, L, prm, res,
                         own);
      uint32_t f[2] = {0, 0}, a[2] = {0, 0};
      for (uint32_t b = 0; b < BINS; ++b) {
        if (res.cov[b] >= R(1)) f[b >> 5] |= 1u << (b & 31);
        if (res.cov[b] > R(0)) a[b >> 5] |= 1u << (b & 31);
      }
      if (full) { full[2 * i] = f[0]; full[2 * i + 1] = f[1]; }
      if (any) { any[2 * i] = a[0]; any[2 * i + 1] = a[1]; }
      if (partial)
        for (uint32_t b = 0; b < BINS; ++b) partial[64 * i + b] = float(res.cov[b]);
      if (irradiance) irradiance[i] = float(res.irradiance);
      if (fraction) fraction[i] = float(res.fraction);
      if (unshadowed) unshadowed[i] = float(res.unshadowed);
      if (work) {
        work[4 * i + 0] = res.work.object_nodes;
        work[4 * i + 1] = res.work.blas_nodes;
        work[4 * i + 2] = res.work.tris;
        work[4 * i + 3] = res.work.flags;
      }
    });
  };
  if (precision == 8)
    run(double(0));
  else
    run(float(0));
  return 0;
}

// Sky irradiance per unit radiance per receiver (sky_irradiance, :1411-1426:
// the six faces summed in order) and, nullable, per face cone c = face *
// npoints + point: its light, FULL/ANY words, coverage and work counters.
// flags: 1 combine by the maximum, 2 no horizon cull, 4 no object-level
// splats, 8 faces in the frame of the object each receiver lies on (its
// point.w holds the object's index as bits; sky_frame, :1432-1456, :2286).
int oracle_sky_visibility(void* sp, const float* receivers, uint64_t npoints, uint32_t hierarchy, uint32_t flags,
                          float prefilter, int precision, float* irradiance, float* face_light, uint32_t* full,
                          uint32_t* any, float* partial, uint32_t* work, int threads, uint32_t accumulate) {
  Scene* s = static_cast<Scene*>(sp);
  if (!s || !irradiance) return 1;
  if (prefilter > 0.0f) build_coverage(*s);
  auto run = [&](auto zero) {
    using R = decltype(zero);
    parallel_for(npoints, threads, [&](uint64_t p) {
      const float* rc = receivers + 8 * p;
      const V3<R> point{R(rc[0]), R(rc[1]), R(rc[2])}, normal{R(rc[4]), R(rc[5]), R(rc[6])};
      const float* frame = nullptr;
      if (flags & 8u) {
        uint32_t m;
        std::memcpy(&m, rc + 3, 4);
        if (m < s->nmeshes && s->ranges[4 * m + 3] != NONE) frame = &s->xforms[16 * (size_t)s->ranges[4 * m + 3]];
      }
      R total = 0;
      for (uint32_t f = 0; f < 6; ++f) {
        R cov[BINS];
        Work wk;
        const R v = sky_face_irradiance(*s, f, point, normal, hierarchy, (flags & 1u) != 0, (flags & 2u) == 0,
                                        R(prefilter), (flags & 4u) == 0, cov, &wk, frame, accumulate);
        total += v;
        const uint64_t c = f * npoints + p;
        if (face_light) face_light[c] = float(v);
        uint32_t fw[2] = {0, 0}, aw[2] = {0, 0};
        for (uint32_t b = 0; b < BINS; ++b) {
          if (cov[b] >= R(1)) fw[b >> 5] |= 1u << (b & 31);
          if (cov[b] > R(0)) aw[b >> 5] |= 1u << (b & 31);
        }
        if (full) { full[2 * c] = fw[0]; full[2 * c + 1] = fw[1]; }
        if (any) { any[2 * c] = aw[0]; any[2 * c + 1] = aw[1]; }
        if (partial)
          for (uint32_t b = 0; b < BINS; ++b) partial[64 * c + b] = float(cov[b]);
        if (work) {
          work[4 * c + 0] = wk.object_nodes;
          work[4 * c + 1] = wk.blas_nodes;
          work[4 * c + 2] = wk.tris;
          work[4 * c + 3] = wk.flags;
        }
      }
      irradiance[p] = float(total);
    });
  };
  if (precision == 8)
    run(double(0));
  else
    run(float(0));
  return 0;
}

// The reference CPU path (Receiver::masked over cone3 + coverage), FP32:
// irradiance per unit radiance and each cone's total weight, for a rect light
// (corner, edge_u, edge_v: 9 floats). use_bvh: 0 brute-force may_touch per
// triangle (Receiver::new), 1 the leaf-4 BVH (Receiver::with_bvh).
int oracle_cpu_masked(void* sp, const float* receivers, uint64_t npoints, const float* light9, int use_bvh,
                      float* visible, float* total, uint32_t* visited, int threads) {
  Scene* s = static_cast<Scene*>(sp);
  cpu::Bvh* bvh = use_bvh ? cpu::build_bvh(*s) : nullptr;
  oracle_cpu_masked_with(sp, bvh, receivers, npoints, light9, visible, total, visited, threads);
  delete bvh;
  return 0;
}

// The reference CPU path's leaf-4 BVH (bvh.rs) alone, so that its build time
// is measured apart from the cones (lib.rs:3497-3510 reports them apart).
void* oracle_cpu_bvh_create(void* sp) { return cpu::build_bvh(*static_cast<Scene*>(sp)); }
void oracle_cpu_bvh_destroy(void* bvh) { delete static_cast<cpu::Bvh*>(bvh); }

// oracle_cpu_masked over a BVH made by oracle_cpu_bvh_create (null: brute
// force). Threads take rows in chunks of 64 from a shared counter, as the
// reference's par_map does (experiments/flatland/src/incremental.rs:124-154).
int oracle_cpu_masked_with(void* sp, void* bvh_p, const float* receivers, uint64_t npoints, const float* light9,
                           float* visible, float* total, uint32_t* visited, int threads) {
  Scene* s = static_cast<Scene*>(sp);
  const cpu::Bvh* bvh = static_cast<const cpu::Bvh*>(bvh_p);
  cpu::V corner{light9[0], light9[1], light9[2]}, eu{light9[3], light9[4], light9[5]}, ev{light9[6], light9[7], light9[8]};
  parallel_for(npoints, threads, [&](uint64_t p) {
    const float* rc = receivers + 8 * p;
    float v, t;
    uint32_t vis;
    cpu::receiver_masked(*s, bvh, cpu::V{rc[0], rc[1], rc[2]}, cpu::V{rc[4], rc[5], rc[6]}, corner, eu, ev, v, t, vis);
    visible[p] = v;
    if (total) total[p] = t;
    if (visited) visited[p] = vis;
  });
  return 0;
}

// Receivers at a pinhole camera's primary hits (camera::primary_hits).
void oracle_primary_hits(void* sp, const float* camera10, uint32_t width, uint32_t height, float* out8, uint8_t* hit,
                         int threads) {
  camera::primary_hits(*static_cast<const Scene*>(sp), camera10, width, height, out8, hit, threads);
}

// The DISK table as this file computes it (64 doubles).
void oracle_disk_table(double* out) {
  const double* d = disk_table();
  std::copy(d, d + BINS, out);
}

// Bin weights of the reference CPU cone (cone3.rs weights), 64 floats; 0 if no cone.
int oracle_cpu_weights(const float* point, const float* normal, const float* light9, float* weights) {
  cpu::PyramidCone cone;
  if (!cpu::toward_rect_light(cpu::V{point[0], point[1], point[2]}, cpu::V{light9[0], light9[1], light9[2]},
                              cpu::V{light9[3], light9[4], light9[5]}, cpu::V{light9[6], light9[7], light9[8]},
                              cpu::V{normal[0], normal[1], normal[2]}, cone))
    return 1;
  std::copy(cone.weights, cone.weights + BINS, weights);
  return 0;
}

uint64_t oracle_poly_overflows() { return g_poly_overflow.load(); }
}
