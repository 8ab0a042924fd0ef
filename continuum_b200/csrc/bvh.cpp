// Host hierarchy builder. Follows crates/continuum-gpu/src/hierarchy.rs:
//   flatten              :29-66
//   split                :128-179  (median split on the longest centroid axis)
//   object_hierarchy     :198-253  (two objects per leaf, oversized subtree)
//   triangle_hierarchy   :527-545  (eight triangles per leaf)
//   padded               :762-765
// The reference partitions with select_nth_unstable, whose order among equal
// keys is unspecified; here the `mid` smallest (key, item) pairs go left and a
// leaf lists its items in increasing index, so the tree depends only on the
// input. Meshes build in parallel, and the top levels of a large mesh split
// their two halves on separate threads; the result is the same tree.
#include "bvh.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <future>
#include <numeric>
#include <thread>

namespace cc {
namespace {

struct Box {
  float lo[3];
  float hi[3];
};

void padded(Box& b) {
  float m = 0.0f;
  for (int k = 0; k < 3; ++k) m = std::max(m, std::max(std::fabs(b.lo[k]), std::fabs(b.hi[k])));
  float pad = 1e-5f * std::max(m, 1.0f);
  for (int k = 0; k < 3; ++k) {
    b.lo[k] -= pad;
    b.hi[k] += pad;
  }
}

// Nodes of a tree over n > 0 items with at most `leaf` per leaf: fixed by n.
uint64_t node_count_for(uint64_t n, uint64_t leaf) {
  if (n <= leaf) return 1;
  return 1 + node_count_for(n / 2, leaf) + node_count_for(n - n / 2, leaf);
}

Box bounds_of(const float* tris12, uint32_t first, uint32_t count) {
  Box b{{FLT_MAX, FLT_MAX, FLT_MAX}, {-FLT_MAX, -FLT_MAX, -FLT_MAX}};
  for (uint32_t t = first; t < first + count; ++t)
    for (int v = 0; v < 3; ++v)
      for (int k = 0; k < 3; ++k) {
        float x = tris12[12 * (size_t)t + 4 * v + k];
        b.lo[k] = std::min(b.lo[k], x);
        b.hi[k] = std::max(b.hi[k], x);
      }
  return b;
}

// A subtree is built into its own node vector and spliced in afterwards, so
// two halves can build concurrently; node numbering is fixed up at splice time
// to the order a serial depth-first build would produce.
struct Builder {
  const std::vector<Box>& bounds;
  uint32_t leaf;
  uint32_t node_base;
  uint32_t item_base;
  int parallel_depth;

  // Builds the subtree over items[0..count) (slots start..start+count) into
  // `nodes`, root at nodes[root]. Children of a node are allocated as a pair
  // at the end of `nodes`, left first, in depth-first order.
  void split(std::vector<NodeGpu>& nodes, size_t root, uint32_t* items, size_t count, size_t start, int depth) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (size_t i = 0; i < count; ++i) {
      const Box& b = bounds[items[i]];
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], b.lo[k]);
        hi[k] = std::max(hi[k], b.hi[k]);
        float c = (b.lo[k] + b.hi[k]) * 0.5f;
        clo[k] = std::min(clo[k], c);
        chi[k] = std::max(chi[k], c);
      }
    }
    NodeGpu& n = nodes[root];
    std::memset(&n, 0, sizeof(n));
    for (int k = 0; k < 3; ++k) {
      n.lo[k] = lo[k];
      n.hi[k] = hi[k];
    }
    if (count <= leaf) {
      std::sort(items, items + count);
      n.info[0] = item_base + (uint32_t)start;
      n.info[1] = (uint32_t)count;
      return;
    }
    float e[3] = {chi[0] - clo[0], chi[1] - clo[1], chi[2] - clo[2]};
    int axis = (e[0] >= e[1] && e[0] >= e[2]) ? 0 : (e[1] >= e[2] ? 1 : 2);
    size_t mid = count / 2;
    const std::vector<Box>& bb = bounds;
    std::nth_element(items, items + mid, items + count, [&bb, axis](uint32_t a, uint32_t b) {
      float ka = bb[a].lo[axis] + bb[a].hi[axis];
      float kb = bb[b].lo[axis] + bb[b].hi[axis];
      return ka < kb || (ka == kb && a < b);
    });
    size_t left = nodes.size();
    nodes.push_back(NodeGpu{});
    nodes.push_back(NodeGpu{});
    nodes[root].info[0] = node_base + (uint32_t)left;
    if (depth < parallel_depth && count > 65536) {
      // The right half builds on another thread into a separate vector; its
      // nodes are appended after the left subtree's, renumbered.
      std::vector<NodeGpu> right_nodes(1);
      auto fut = std::async(std::launch::async, [&] {
        split(right_nodes, 0, items + mid, count - mid, start + mid, depth + 1);
      });
      split(nodes, left, items, mid, start, depth + 1);
      fut.get();
      splice(nodes, left + 1, right_nodes);
    } else {
      split(nodes, left, items, mid, start, depth + 1);
      split(nodes, left + 1, items + mid, count - mid, start + mid, depth + 1);
    }
  }

  // Moves subtree `sub` (root at sub[0], children numbered within `sub` plus
  // node_base) into `nodes`: its root into nodes[root_slot], the rest
  // appended, child links shifted by where they land.
  void splice(std::vector<NodeGpu>& nodes, size_t root_slot, const std::vector<NodeGpu>& sub) {
    size_t offset = nodes.size() - 1;  // sub index i (i >= 1) lands at offset + i
    nodes[root_slot] = sub[0];
    if (sub[0].info[1] == 0) nodes[root_slot].info[0] += (uint32_t)offset;
    for (size_t i = 1; i < sub.size(); ++i) {
      NodeGpu n = sub[i];
      if (n.info[1] == 0) n.info[0] += (uint32_t)offset;
      nodes.push_back(n);
    }
  }
};

// object_hierarchy (hierarchy.rs:198-253): two objects per leaf over the
// objects' padded world bounds, with oversized objects in a subtree of their
// own under the root.
void object_hierarchy(const std::vector<Box>& mesh_box, const std::vector<uint32_t>& keep,
                      std::vector<NodeGpu>& nodes_out, std::vector<uint32_t>& items_out) {
  std::vector<uint32_t> items = keep;
  const size_t nmeshes = items.size();
  std::vector<NodeGpu>& nodes = nodes_out;
  nodes.assign(1, NodeGpu{});
  if (items.empty()) {
    items_out = {0};
    nodes[0].info[1] = 1;
    return;
  }
  auto diagonal = [&](uint32_t m) {
    float d2 = 0;
    for (int k = 0; k < 3; ++k) {
      float e = mesh_box[m].hi[k] - mesh_box[m].lo[k];
      d2 += e * e;
    }
    return std::sqrt(d2);
  };
  std::vector<float> sizes(nmeshes);
  for (size_t i = 0; i < nmeshes; ++i) sizes[i] = diagonal(items[i]);
  size_t mid = sizes.size() / 2;
  std::nth_element(sizes.begin(), sizes.begin() + mid, sizes.end());
  const float median = sizes[mid];
  std::vector<uint32_t> big, small;
  for (uint32_t m : items) (diagonal(m) > kOversized * median ? big : small).push_back(m);
  Builder ob{mesh_box, kLeafObjects, 0, 0, 0};
  if (big.empty() || small.empty()) {
    ob.split(nodes, 0, items.data(), items.size(), 0, 0);
  } else {
    const size_t nb = big.size();
    items = big;
    items.insert(items.end(), small.begin(), small.end());
    nodes.push_back(NodeGpu{});
    nodes.push_back(NodeGpu{});
    ob.split(nodes, 1, items.data(), nb, 0, 0);
    ob.split(nodes, 2, items.data() + nb, items.size() - nb, nb, 0);
    NodeGpu& r = nodes[0];
    for (int k = 0; k < 3; ++k) {
      r.lo[k] = std::min(nodes[1].lo[k], nodes[2].lo[k]);
      r.hi[k] = std::max(nodes[1].hi[k], nodes[2].hi[k]);
    }
    r.info[0] = 1;
  }
  items_out = items;
}

}  // namespace

void build_flat_scene(const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes, FlatScene& out,
                      int threads) {
  if (threads < 1) threads = 1;
  out = FlatScene{};
  out.nmeshes = nmeshes;
  std::vector<uint64_t> first(nmeshes + 1, 0);
  for (uint32_t m = 0; m < nmeshes; ++m) first[m + 1] = first[m] + mesh_counts[m];
  const uint64_t total = first[nmeshes];
  out.tris.resize(total * 12);
  for (uint64_t t = 0; t < total; ++t)
    for (int v = 0; v < 3; ++v) {
      float* d = &out.tris[12 * t + 4 * v];
      const float* s = &tri9[9 * t + 3 * v];
      d[0] = s[0];
      d[1] = s[1];
      d[2] = s[2];
      d[3] = 0.0f;
    }

  // Per-mesh triangle hierarchies, built concurrently, then concatenated in
  // mesh order (each numbered from its final position).
  std::vector<std::vector<NodeGpu>> mesh_nodes(nmeshes);
  std::vector<std::vector<uint32_t>> mesh_items(nmeshes);
  std::vector<Box> mesh_box(nmeshes);
  std::vector<uint32_t> root_of(nmeshes, kNone);
  // Node numbering needs each mesh's node count before its own; a tree over
  // n > 0 items with leaves of at most L has a count fixed by n alone, so
  // the counts are computed first.
  auto node_count = [](uint64_t n, uint64_t leaf) {
    // count(n) = 1 if n <= leaf else 1 + count(n/2) + count(n - n/2)
    struct R {
      static uint64_t f(uint64_t n, uint64_t leaf) {
        if (n <= leaf) return 1;
        return 1 + f(n / 2, leaf) + f(n - n / 2, leaf);
      }
    };
    return R::f(n, leaf);
  };
  std::vector<uint64_t> node_first(nmeshes + 1, 0);
  for (uint32_t m = 0; m < nmeshes; ++m)
    node_first[m + 1] = node_first[m] + (mesh_counts[m] ? node_count(mesh_counts[m], kLeafTriangles) : 0);

  std::atomic<uint32_t> next{0};
  auto work = [&] {
    for (;;) {
      uint32_t m = next.fetch_add(1);
      if (m >= nmeshes) break;
      uint32_t count = mesh_counts[m];
      mesh_box[m] = bounds_of(out.tris.data(), (uint32_t)first[m], count);
      padded(mesh_box[m]);
      if (count == 0) continue;
      std::vector<Box> bounds(count);
      for (uint32_t t = 0; t < count; ++t) {
        bounds[t] = bounds_of(out.tris.data(), (uint32_t)first[m] + t, 1);
        padded(bounds[t]);
      }
      std::vector<uint32_t> items(count);
      std::iota(items.begin(), items.end(), 0u);
      std::vector<NodeGpu>& nodes = mesh_nodes[m];
      nodes.assign(1, NodeGpu{});
      nodes.reserve(node_first[m + 1] - node_first[m]);
      uint32_t root = (uint32_t)node_first[m];
      Builder b{bounds, kLeafTriangles, root, (uint32_t)first[m], count > 1000000 ? 3 : 0};
      b.split(nodes, 0, items.data(), count, 0, 0);
      for (uint32_t& t : items) t += (uint32_t)first[m];
      mesh_items[m] = std::move(items);
      root_of[m] = root;
    }
  };
  std::vector<std::thread> pool;
  int nt = std::min<int>(threads, std::max<uint32_t>(1, nmeshes));
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();

  out.blas.reserve(node_first[nmeshes]);
  out.blas_items.reserve(total);
  for (uint32_t m = 0; m < nmeshes; ++m) {
    out.blas.insert(out.blas.end(), mesh_nodes[m].begin(), mesh_nodes[m].end());
    out.blas_items.insert(out.blas_items.end(), mesh_items[m].begin(), mesh_items[m].end());
    out.ranges.insert(out.ranges.end(), {(uint32_t)first[m], mesh_counts[m], root_of[m], kNone});
  }

  // The object hierarchy over meshes (object_hierarchy, hierarchy.rs:198-253).
  std::vector<uint32_t> all(nmeshes);
  std::iota(all.begin(), all.end(), 0u);
  object_hierarchy(mesh_box, all, out.nodes, out.items);
}

namespace {

// The padded world bounds of an object-space box placed by `o`
// (Placement::world_bounds, hierarchy.rs:287-303).
Box world_bounds(const Box& b, const Instance& o) {
  const float* R = o.rotation;
  const float* t = o.translation;
  Box w{{FLT_MAX, FLT_MAX, FLT_MAX}, {-FLT_MAX, -FLT_MAX, -FLT_MAX}};
  for (int c = 0; c < 8; ++c) {
    const float p[3] = {(c & 1) ? b.hi[0] : b.lo[0], (c & 2) ? b.hi[1] : b.lo[1], (c & 4) ? b.hi[2] : b.lo[2]};
    for (int i = 0; i < 3; ++i) {
      // rotation * p (columns scaled by p's components, summed in order),
      // then * scale + translation.
      const float v = (R[3 * i] * p[0] + R[3 * i + 1] * p[1] + R[3 * i + 2] * p[2]) * o.scale + t[i];
      w.lo[i] = std::min(w.lo[i], v);
      w.hi[i] = std::max(w.hi[i], v);
    }
  }
  padded(w);
  return w;
}

void to_node_bounds(const Box& b, NodeGpu& n) {
  for (int k = 0; k < 3; ++k) {
    n.lo[k] = b.lo[k];
    n.hi[k] = b.hi[k];
  }
}

// The root over the static subtree (node 1) and the movers' (node 2)
// (union_root, hierarchy.rs:372-381).
NodeGpu union_root(const NodeGpu& a, const NodeGpu& b) {
  NodeGpu r{};
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = std::min(a.lo[k], b.lo[k]);
    r.hi[k] = std::max(a.hi[k], b.hi[k]);
  }
  r.info[0] = 1;
  r.info[2] = kNoSplat;
  return r;
}

// mover_subtree (hierarchy.rs:383-410): the movers' subtree over their
// current bounds, in the movers' order; its shape depends only on their
// count. Writes its root to nodes[2], its other nodes from first_node and
// its items from first_item.
void mover_subtree(FlatScene& s, const std::vector<Box>& mover_bounds) {
  const MoverTree& t = s.movers;
  std::vector<NodeGpu> local(1);
  std::vector<uint32_t> order(mover_bounds.size());
  std::iota(order.begin(), order.end(), 0u);
  Builder b{mover_bounds, kLeafObjects, t.first_node - 1, t.first_item, 0};
  b.split(local, 0, order.data(), order.size(), 0, 0);
  for (NodeGpu& n : local) n.info[2] = kNoSplat;
  s.nodes[2] = local[0];
  for (size_t i = 1; i < local.size(); ++i) s.nodes[t.first_node + i - 1] = local[i];
  for (size_t k = 0; k < order.size(); ++k) s.items[t.first_item + k] = t.objects[order[k]];
  s.nodes[0] = union_root(s.nodes[1], s.nodes[2]);
}

}  // namespace

void build_instanced_scene(const float* tri9, const uint32_t* geometry_counts, uint32_t ngeometries,
                           const Instance* instances, uint32_t ninstances, const uint32_t* movable,
                           uint32_t nmovable, FlatScene& out, int threads) {
  // Each geometry's triangles and hierarchy once (flatten, triangle_hierarchy).
  build_flat_scene(tri9, geometry_counts, ngeometries, out, threads);
  const std::vector<uint32_t> geometry_ranges = out.ranges;
  out.geometry_roots.assign(ngeometries, kNone);
  for (uint32_t g = 0; g < ngeometries; ++g) out.geometry_roots[g] = geometry_ranges[4 * g + 2];
  std::vector<Box> local(ngeometries);
  for (uint32_t g = 0; g < ngeometries; ++g)
    local[g] = bounds_of(out.tris.data(), geometry_ranges[4 * g], geometry_ranges[4 * g + 1]);
  // Per object: its geometry's range with its transform, the transform's
  // rows, and its padded world bounds (flatten_instanced, hierarchy.rs:464-522;
  // Placement::rows and world_bounds, :272-303).
  out.ranges.clear();
  out.xforms.clear();
  std::vector<Box> bounds(ninstances);
  out.object_geometry.assign(ninstances, 0);
  for (uint32_t k = 0; k < ninstances; ++k) {
    const Instance& o = instances[k];
    const uint32_t* r = &geometry_ranges[4 * o.geometry];
    out.ranges.insert(out.ranges.end(), {r[0], r[1], r[2], k});
    const float* R = o.rotation;  // row-major
    const float* t = o.translation;
    out.xforms.insert(out.xforms.end(), {R[0], R[1], R[2], t[0], R[3], R[4], R[5], t[1], R[6], R[7], R[8], t[2],
                                         o.scale, 1.0f / o.scale, 0.0f, 0.0f});
    out.object_geometry[k] = o.geometry;
    bounds[k] = world_bounds(local[o.geometry], o);
  }
  out.geometry_bounds.resize(6 * (size_t)ngeometries);
  for (uint32_t g = 0; g < ngeometries; ++g)
    for (int k = 0; k < 3; ++k) {
      out.geometry_bounds[6 * g + k] = local[g].lo[k];
      out.geometry_bounds[6 * g + 3 + k] = local[g].hi[k];
    }
  if (out.ranges.empty()) out.ranges.insert(out.ranges.end(), {0u, 0u, kNone, kNone});
  if (out.xforms.empty()) out.xforms.assign(16, 0.0f);
  out.nmeshes = (uint32_t)(out.ranges.size() / 4);
  out.movers = MoverTree{};
  if (nmovable == 0) {
    std::vector<uint32_t> all(ninstances);
    std::iota(all.begin(), all.end(), 0u);
    object_hierarchy(bounds, all, out.nodes, out.items);
    return;
  }
  // object_hierarchy_with_movers (hierarchy.rs:331-369): the static objects'
  // hierarchy under node 1 (its node i >= 1 at i + 2), the movers' subtree
  // under node 2, the root over both.
  std::vector<uint8_t> is_movable(ninstances, 0);
  for (uint32_t i = 0; i < nmovable; ++i) is_movable[movable[i]] = 1;
  std::vector<uint32_t> fixed_items;
  for (uint32_t m = 0; m < ninstances; ++m)
    if (!is_movable[m]) fixed_items.push_back(m);
  std::vector<NodeGpu> fixed;
  std::vector<uint32_t> items;
  object_hierarchy(bounds, fixed_items, fixed, items);
  auto place = [](uint32_t i) { return i == 0 ? 1u : i + 2u; };
  MoverTree& t = out.movers;
  t.first_node = (uint32_t)fixed.size() + 2;
  t.first_item = (uint32_t)items.size();
  t.objects.assign(movable, movable + nmovable);
  const uint64_t mover_nodes = node_count_for(nmovable, kLeafObjects);
  t.nodes = (uint32_t)(mover_nodes - 1);
  out.nodes.assign(t.first_node + t.nodes, NodeGpu{});
  for (size_t i = 0; i < fixed.size(); ++i) {
    NodeGpu n = fixed[i];
    if (n.info[1] == 0) n.info[0] = place(n.info[0]);
    out.nodes[place((uint32_t)i)] = n;
  }
  out.items = items;
  out.items.resize(items.size() + nmovable);
  std::vector<Box> mover_bounds(nmovable);
  for (uint32_t i = 0; i < nmovable; ++i) mover_bounds[i] = bounds[movable[i]];
  mover_subtree(out, mover_bounds);
}

void move_instances(FlatScene& s, const Instance* placements, float* boxes12) {
  const MoverTree& t = s.movers;
  std::vector<Box> mover_bounds(t.objects.size());
  for (size_t i = 0; i < t.objects.size(); ++i) {
    const uint32_t m = t.objects[i];
    const uint32_t x = s.ranges[4 * m + 3];
    float* X = &s.xforms[16 * (size_t)x];
    const uint32_t g = s.object_geometry[m];
    Box local;
    for (int k = 0; k < 3; ++k) {
      local.lo[k] = s.geometry_bounds[6 * g + k];
      local.hi[k] = s.geometry_bounds[6 * g + 3 + k];
    }
    // The old place: the transform as stored.
    Instance old{};
    old.geometry = g;
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) old.rotation[3 * r + c] = X[4 * r + c];
      old.translation[r] = X[4 * r + 3];
    }
    old.scale = X[12];
    const Box before = world_bounds(local, old);
    const Instance& o = placements[i];
    const float* R = o.rotation;
    const float* tr = o.translation;
    // The object keeps its `clear` (row 3's z) where it moves.
    const float row[16] = {R[0], R[1], R[2], tr[0], R[3], R[4], R[5], tr[1], R[6], R[7], R[8], tr[2],
                           o.scale, 1.0f / o.scale, X[14], 0.0f};
    std::memcpy(X, row, sizeof(row));
    mover_bounds[i] = world_bounds(local, o);
    if (boxes12) {
      for (int k = 0; k < 3; ++k) {
        boxes12[12 * i + k] = before.lo[k];
        boxes12[12 * i + 3 + k] = before.hi[k];
        boxes12[12 * i + 6 + k] = mover_bounds[i].lo[k];
        boxes12[12 * i + 9 + k] = mover_bounds[i].hi[k];
      }
    }
  }
  mover_subtree(s, mover_bounds);
}

// coverage_directions (hierarchy.rs:714-723): (i, j, k) normalized, the zero
// direction kept zero (glam's normalize_or_zero: v times 1 / |v|).
static void coverage_directions(float d[kCoverageSamples][3]) {
  for (uint32_t n = 0; n < kCoverageSamples; ++n) {
    const float v[3] = {float(n / 9) - 1.0f, float(n / 3 % 3) - 1.0f, float(n % 3) - 1.0f};
    const float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const float rcp = 1.0f / len;
    const bool ok = std::isfinite(rcp) && rcp > 0.0f;
    for (int k = 0; k < 3; ++k) d[n][k] = ok ? v[k] * rcp : 0.0f;
  }
}

// A placed object's opacity for its geometry's coverage samples: blended
// (clear in (0, 1)), transmissive at normal incidence (clear below 0), a
// volume's two surfaces (clear at most -2) (flatten_instanced,
// hierarchy.rs:488-497).
static float clear_opacity(float clear) {
  if (clear > 0.0f) return 1.0f - clear;
  if (clear <= -2.0f) {
    const float t = 0.96f * (-2.0f - clear);
    return 1.0f - t * t;
  }
  return 1.0f - 0.96f * -clear;
}

std::vector<float> blas_coverage(const FlatScene& s) {
  float dirs[kCoverageSamples][3];
  coverage_directions(dirs);
  const size_t n = s.blas.size();
  std::vector<float> cov(n * kCoverageSamples, 0.0f);
  // Children always follow their parent: a reverse sweep sees them first.
  for (size_t i = n; i-- > 0;) {
    float* out = cov.data() + i * kCoverageSamples;
    const uint32_t x = s.blas[i].info[0], count = s.blas[i].info[1];
    if (count > 0) {
      for (uint32_t k = x; k < x + count; ++k) {
        const float* t = s.tris.data() + 12 * (size_t)s.blas_items[k];
        const float e1[3] = {t[4] - t[0], t[5] - t[1], t[6] - t[2]};
        const float e2[3] = {t[8] - t[0], t[9] - t[1], t[10] - t[2]};
        const float an[3] = {(e1[1] * e2[2] - e2[1] * e1[2]) * 0.5f, (e1[2] * e2[0] - e2[2] * e1[0]) * 0.5f,
                             (e1[0] * e2[1] - e2[0] * e1[1]) * 0.5f};
        for (uint32_t d = 0; d < kCoverageSamples; ++d)
          out[d] += std::max(an[0] * dirs[d][0] + an[1] * dirs[d][1] + an[2] * dirs[d][2], 0.0f);
      }
    } else {
      const float* a = cov.data() + (size_t)x * kCoverageSamples;
      const float* b = a + kCoverageSamples;
      for (uint32_t d = 0; d < kCoverageSamples; ++d) out[d] = a[d] + b[d];
    }
  }
  // Instanced scenes: a geometry whose first placing object is blended or
  // transmissive has its nodes' samples (its root's and those after it, up
  // to the next geometry's root) scaled by that object's opacity
  // (hierarchy.rs:469-503).
  if (!s.xforms.empty()) {
    const uint32_t ngeom = (uint32_t)s.geometry_roots.size();
    std::vector<uint32_t> first_object(ngeom, kNone);
    for (uint32_t m = (uint32_t)s.object_geometry.size(); m-- > 0;)
      if (s.object_geometry[m] < ngeom) first_object[s.object_geometry[m]] = m;
    std::vector<std::pair<uint32_t, uint32_t>> roots;  // (root, geometry) of every geometry with triangles
    for (uint32_t g = 0; g < ngeom; ++g)
      if (s.geometry_roots[g] != kNone) roots.push_back({s.geometry_roots[g], g});
    std::sort(roots.begin(), roots.end());
    for (size_t k = 0; k < roots.size(); ++k) {
      const uint32_t m = first_object[roots[k].second];
      if (m == kNone) continue;
      const float clear = s.xforms[16 * (size_t)s.ranges[4 * m + 3] + 14];
      if (clear == 0.0f) continue;
      const float opacity = clear_opacity(clear);
      const size_t end = k + 1 < roots.size() ? roots[k + 1].first : n;
      for (size_t i = (size_t)roots[k].first * kCoverageSamples; i < end * kCoverageSamples; ++i) cov[i] *= opacity;
    }
  }
  return cov;
}

// front_area (hierarchy.rs:625-652): a node's coverage seen along v,
// bilinear on the face of the cube of sample directions v points through.
static float front_area(const float* cov, const float v[3]) {
  const float a[3] = {std::fabs(v[0]), std::fabs(v[1]), std::fabs(v[2])};
  int axis = 0;
  if (a[1] > a[0] && a[1] >= a[2]) axis = 1;
  else if (a[2] > a[0] && a[2] > a[1]) axis = 2;
  float main, s, t;
  if (axis == 0) main = v[0], s = v[1] / a[0], t = v[2] / a[0];
  else if (axis == 1) main = v[1], s = v[0] / a[1], t = v[2] / a[1];
  else main = v[2], s = v[0] / a[2], t = v[1] / a[2];
  const int m = main >= 0.0f ? 1 : -1;
  const int s0 = s < 0.0f ? -1 : 0, t0 = t < 0.0f ? -1 : 0;
  const float fs = s - float(s0), ft = t - float(t0);
  auto sample = [&](int i, int j, int k) { return cov[9 * (i + 1) + 3 * (j + 1) + (k + 1)]; };
  float f[4];
  for (int c = 0; c < 4; ++c) {
    const int gs = s0 + (c & 1), gt = t0 + (c >> 1);
    f[c] = axis == 0 ? sample(m, gs, gt) : axis == 1 ? sample(gs, m, gt) : sample(gs, gt, m);
  }
  auto lerp = [](float x, float y, float u) { return x + (y - x) * u; };
  return lerp(lerp(f[0], f[1], fs), lerp(f[2], f[3], fs), ft);
}

std::vector<float> object_coverage(const FlatScene& s, const std::vector<float>& blas_cov) {
  float dirs[kCoverageSamples][3];
  coverage_directions(dirs);
  const uint32_t nobj = s.nmeshes;
  std::vector<float> per_object((size_t)nobj * kCoverageSamples, 0.0f);
  for (uint32_t m = 0; m < nobj; ++m) {
    const uint32_t root = s.ranges[4 * m + 2];
    const uint32_t x = s.ranges[4 * m + 3];
    if (root == kNone || x == kNone) continue;
    const float* cov = blas_cov.data() + (size_t)root * kCoverageSamples;
    const float* X = s.xforms.data() + 16 * (size_t)x;
    const float scale = X[12];
    float* out = per_object.data() + (size_t)m * kCoverageSamples;
    for (uint32_t n = 0; n < kCoverageSamples; ++n) {
      const float* d = dirs[n];
      if (d[0] == 0.0f && d[1] == 0.0f && d[2] == 0.0f) continue;
      // The direction turned into the object: the rotation's transpose (its
      // rows as columns) times d.
      const float v[3] = {X[0] * d[0] + X[4] * d[1] + X[8] * d[2], X[1] * d[0] + X[5] * d[1] + X[9] * d[2],
                          X[2] * d[0] + X[6] * d[1] + X[10] * d[2]};
      out[n] = scale * scale * front_area(cov, v);
    }
  }
  const size_t nn = s.nodes.size();
  std::vector<float> cov(nn * kCoverageSamples, 0.0f);
  for (size_t i = nn; i-- > 0;) {
    float* out = cov.data() + i * kCoverageSamples;
    const uint32_t x = s.nodes[i].info[0], count = s.nodes[i].info[1];
    if (count > 0) {
      for (uint32_t k = x; k < x + count; ++k) {
        const float* po = per_object.data() + (size_t)s.items[k] * kCoverageSamples;
        for (uint32_t d = 0; d < kCoverageSamples; ++d) out[d] += po[d];
      }
    } else {
      const float* a = cov.data() + (size_t)x * kCoverageSamples;
      const float* b = a + kCoverageSamples;
      for (uint32_t d = 0; d < kCoverageSamples; ++d) out[d] = a[d] + b[d];
    }
  }
  for (size_t i = 0; i < nn; ++i)
    if (s.nodes[i].info[2] == kNoSplat) cov[i * kCoverageSamples + 13] = 1.0f;
  return cov;
}

}  // namespace cc