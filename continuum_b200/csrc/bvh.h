// Host-side scene hierarchies: the reference's layouts, built the way the
// reference builds them (crates/continuum-gpu/src/hierarchy.rs), so the
// device walk visits the same nodes in the same order as the reference's
// and its walk caps cut at the same place.
#pragma once
#include <cstdint>
#include <vector>

namespace cc {

// NodeGpu (hierarchy.rs:68-76): lo.xyzw, hi.xyzw, info.xyzw. Leaf: info =
// [first item, item count, 0, 0]; interior: [left child, 0, 0, 0] with the
// right child at left + 1.
struct NodeGpu {
  float lo[4];
  float hi[4];
  uint32_t info[4];
};
static_assert(sizeof(NodeGpu) == 48, "NodeGpu is 48 bytes");

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kLeafTriangles = 8;  // LEAF_TRIANGLES, hierarchy.rs:727
constexpr uint32_t kLeafObjects = 2;    // object_hierarchy leaves, hierarchy.rs:198
constexpr float kOversized = 64.0f;     // OVERSIZED, hierarchy.rs:257
constexpr uint32_t kNoSplat = 1;        // NO_SPLAT (info.z of the movers' nodes and the root), hierarchy.rs:307

// Where the movable objects' subtree lives (MoverTree, hierarchy.rs:309-327):
// its root is node 2 (node 1 roots the static objects), its other nodes are
// `nodes` from `first_node`, its items the movers' count from `first_item`.
struct MoverTree {
  uint32_t first_node = 0;
  uint32_t nodes = 0;
  uint32_t first_item = 0;
  std::vector<uint32_t> objects;  // the movable objects, in the order their placements are given
};

struct FlatScene {
  std::vector<float> tris;          // 12 floats per triangle
  std::vector<uint32_t> ranges;     // 4 per mesh
  std::vector<NodeGpu> blas;
  std::vector<uint32_t> blas_items;
  std::vector<NodeGpu> nodes;
  std::vector<uint32_t> items;
  uint32_t nmeshes = 0;
  // Instanced scenes: per object transform, 16 floats (rows 0-2 of the
  // rotation with the translation in w, then scale, 1 / scale, 0, 0); the
  // object's range points at its geometry and ranges[4 * m + 3] at its
  // transform. Empty for scenes whose triangles are in world space.
  std::vector<float> xforms;
  std::vector<uint32_t> object_geometry;  // instanced scenes: each object's geometry
  std::vector<float> geometry_bounds;     // instanced scenes: each geometry's object-space box (lo, hi)
  std::vector<uint32_t> geometry_roots;   // instanced scenes: each geometry's triangle-hierarchy root (kNone: none)
  MoverTree movers;                       // instanced scenes built with movable objects
};

// An object placing a geometry: world = scale * rotation * p + translation
// (Placement, hierarchy.rs:258-270; opaque).
struct Instance {
  uint32_t geometry;
  float rotation[9];  // row-major
  float scale;
  float translation[3];
};

// flatten + triangle_hierarchy per mesh + mesh_hierarchy. `tri9`: 9 floats
// per triangle, meshes consecutive.
void build_flat_scene(const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes, FlatScene& out,
                      int threads);

// flatten_instanced (hierarchy.rs:464-522) + object_hierarchy over the
// objects' world bounds: each geometry's triangles and triangle hierarchy
// once, one object per instance.
// With `nmovable` > 0 the object hierarchy keeps the movable objects in a
// subtree of their own (object_hierarchy_with_movers, hierarchy.rs:331-369).
void build_instanced_scene(const float* tri9, const uint32_t* geometry_counts, uint32_t ngeometries,
                           const Instance* instances, uint32_t ninstances, const uint32_t* movable,
                           uint32_t nmovable, FlatScene& out, int threads);

// Places the movable objects anew (placements in MoverTree::objects order,
// same geometries) and rebuilds their subtree and the root (mover_subtree,
// hierarchy.rs:383-410). boxes12 (nullable): per mover, the padded world
// bounds before and after (lo.xyz, hi.xyz each).
void move_instances(FlatScene& s, const Instance* placements, float* boxes12);

// Coverage samples per hierarchy node for prefiltered cones
// (COVERAGE_SAMPLES, hierarchy.rs:710-723): the projected front area of the
// node's triangles from the 26 directions (i, j, k) in {-1, 0, 1}^3 \ 0
// (normalized), at index 9(i+1) + 3(j+1) + (k+1); index 13 is unused.
constexpr uint32_t kCoverageSamples = 27;
// triangle_hierarchy's coverage (hierarchy.rs:546-569), for every node of
// every mesh's triangle hierarchy: a leaf sums its triangles' max(0,
// area-normal . d), an interior node its children's.
std::vector<float> blas_coverage(const FlatScene& s);
// object_coverage (hierarchy.rs:661-707) for an instanced scene: per object
// node, its objects' projected front areas, each its geometry root's
// coverage seen along the direction turned into the object, times scale^2.
// Sample 13 of a node without prefiltered coverage (NO_SPLAT: the root over
// movers and the movers' subtree) is set to 1 as its flag.
std::vector<float> object_coverage(const FlatScene& s, const std::vector<float>& blas_cov);

// Primary hits of a pinhole camera (raycast.cpp).
void primary_hits(const FlatScene& s, const float* camera, uint32_t width, uint32_t height, float* out8,
                  uint8_t* hit_mask, int threads);

}  // namespace cc
