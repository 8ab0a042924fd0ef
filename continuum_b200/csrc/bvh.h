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
void build_instanced_scene(const float* tri9, const uint32_t* geometry_counts, uint32_t ngeometries,
                           const Instance* instances, uint32_t ninstances, FlatScene& out, int threads);

// Primary hits of a pinhole camera (raycast.cpp).
void primary_hits(const FlatScene& s, const float* camera, uint32_t width, uint32_t height, float* out8,
                  uint8_t* hit_mask, int threads);

}  // namespace cc
