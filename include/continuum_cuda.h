/* continuum_cuda.h — C ABI of the B200-native mask-cone visibility path.
 *
 * One cone per (shading point, area light) is traversed through the scene's
 * bounding volume hierarchy; the occluding triangles are rasterized as exact
 * areas into the cone's 8x8 bins, and the bins are integrated into the
 * irradiance per unit radiance and the visible fraction of the light.
 *
 * Conventions
 *  - Every entry point returns an int status (CC_OK = 0). No exception or
 *    abort crosses the ABI; cc_last_error() gives a message for the calling
 *    thread's last failure.
 *  - Buffers are owned by the caller. Unless a call says otherwise, pointers
 *    are host pointers; with CC_DEVICE_POINTERS in cc_options.flags the
 *    receivers, lights and every output of cc_visibility are device pointers
 *    and the call is asynchronous on the given stream.
 *  - A context is used from one host thread at a time and serves one call at
 *    a time (the reference's MaskConeKernel is !Sync for the same reason):
 *    its buffers, copy stream and events are shared by its calls, so two
 *    calls on one context must not overlap, even on different streams.
 *    Scenes belong to the context that built them.
 *  - Cone c = light * npoints + point (light-major). Mask words: bin b of a
 *    cone is bit (b % 32) of word (b / 32); bin b = row * 8 + col.
 *
 * Layouts match the reference's GPU buffers:
 *  receivers: 8 floats each, point.xyz w, normal.xyz w  (ReceiverGpu,
 *             crates/continuum-gpu/src/lib.rs:54-60)
 *  lights:    16 floats each (LightGpu, crates/continuum-gpu/src/lib.rs:710-749):
 *             rect:   corner.xyz, w = 0 two-sided / 1 one-sided; edge_u.xyz 0;
 *                     edge_v.xyz 0; radiance.xyz 0
 *             sphere: center.xyz, w = 2; (radius, spot scale, spot offset, 0);
 *                     (spot axis.xyz, 1 if spot else 0); radiance.xyz 0
 *  triangles: 12 floats each in flat scenes (three vec4 vertices,
 *             crates/continuum-gpu/src/hierarchy.rs:12-13), 9 floats each
 *             where a call builds the hierarchy itself.
 */
#ifndef CONTINUUM_CUDA_H
#define CONTINUUM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CC_API __attribute__((visibility("default")))
#else
#define CC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CC_OK 0
#define CC_ERR_INVALID 1      /* bad argument or layout */
#define CC_ERR_CUDA 2         /* a CUDA call failed (message in cc_last_error) */
#define CC_ERR_OOM 3          /* device memory exhausted */
#define CC_ERR_NO_DEVICE 4    /* no CUDA device (MaskConeKernel::new() -> None) */
#define CC_ERR_STACK 5        /* a traversal stack overflowed: flagged cones are not exact */
#define CC_ERR_TIMEOUT 6      /* a bounded device wait gave up */
#define CC_ERR_BUSY 7         /* a batch or server queue is full */

#define CC_NONE 0xffffffffu

/* cc_options.flags */
#define CC_DEVICE_POINTERS 1u /* receivers, lights and outputs are device pointers */
#define CC_NO_REDO 2u         /* skip the solo re-walk (diagnostic): order-diverged and overflowed cones keep their packet results */
#define CC_KEEP_ORDER 4u      /* walk points in the given order (default: Morton order of their positions) */
#define CC_NO_OBJECT_PREFILTER 8u /* with prefilter: splat triangle-hierarchy nodes only (set_object_prefilter(false)) */

/* Status bits in cc_outputs.work[4 * c + 3] */
#define CC_CONE_CAPPED 1u     /* the walk stopped at its cap (LIGHT_CONE_CAP / WIDE_CONE_CAP) */
#define CC_CONE_STACK 2u      /* the traversal stack overflowed */
#define CC_CONE_DIVERGED 4u   /* its packet's child order differed from its own */
#define CC_CONE_REWALKED 8u   /* recomputed walking alone */
#define CC_CONE_FULL_STOP 16u /* the walk stopped early with every bin full */
#define CC_CONE_ACC_WIDE 32u  /* its 32-bit accumulation overflowed: recomputed with 64-bit cells */

typedef struct cc_context cc_context;
typedef struct cc_scene cc_scene;

/* Replaces MaskConeKernel::new / with_device
 * (crates/continuum-gpu/src/lib.rs:1145-1190): a context on CUDA device
 * `device`. CC_ERR_NO_DEVICE where the reference returns None. */
CC_API int cc_context_create(int device, cc_context** out);
CC_API int cc_context_destroy(cc_context* ctx);

/* Cones one chunk of the split path holds at most (32 .. 2^31; default
 * 33,554,432). Exact light cones are set up, walked and integrated a chunk at
 * a time, with 368 bytes of device scratch per slot of one chunk (cone
 * records and masks): cc_visibility, batches submitted after the call, and
 * servers created after it (which hold at most 4,194,304) take the bound.
 * Results do not depend on it. No counterpart in the reference (its wgpu
 * path sizes buffers per dispatch). */
CC_API int cc_context_set_split_chunk(cc_context* ctx, uint64_t cones);

/* The calling thread's last error message ("" if none). */
CC_API const char* cc_last_error(void);

/* A scene from the reference's flattened layout: Flat (hierarchy.rs:11-25,
 * flatten :29-66) plus the object hierarchy (mesh_hierarchy :183-194).
 * NodeGpu records are 48 bytes: lo.xyzw, hi.xyzw, info.xyzw (hierarchy.rs:68-76).
 * The library repacks nodes into its own 32-byte device records. */
typedef struct cc_flat_scene {
  const float* tris;          /* 12 floats per triangle */
  uint32_t ntris;
  const uint32_t* ranges;     /* 4 per mesh: first, count, blas root or CC_NONE, transform index or CC_NONE */
  uint32_t nmeshes;
  const void* blas;           /* NodeGpu per triangle-hierarchy node */
  uint32_t nblas;
  const uint32_t* blas_items; /* triangle index per leaf slot */
  uint32_t nblas_items;
  const void* nodes;          /* NodeGpu per object-hierarchy node */
  uint32_t nnodes;
  const uint32_t* items;      /* mesh index per object leaf slot */
  uint32_t nitems;
  const float* xforms;        /* instanced scenes: 16 floats per transform (nullable), see cc_scene_build_instanced */
  uint32_t nxforms;
} cc_flat_scene;

CC_API int cc_scene_upload(cc_context* ctx, const cc_flat_scene* flat, cc_scene** out);

/* A scene from meshes, with the hierarchies built on the host exactly as the
 * reference builds them (flatten, triangle_hierarchy, mesh_hierarchy:
 * hierarchy.rs:29-66, 128-253, 527-571, 762-765). tri9: 9 floats per
 * triangle, meshes consecutive, mesh_counts[m] triangles in mesh m.
 * With ctx NULL the scene stays on the host (no device is needed): it can be
 * inspected and ray cast, but not passed to cc_visibility. */
CC_API int cc_scene_build(cc_context* ctx, const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes,
                   cc_scene** out);
CC_API int cc_scene_destroy(cc_scene* scene);

/* An object placing a geometry: world = scale * rotation * p + translation,
 * rotation orthonormal (row-major), scale positive (Placement,
 * crates/continuum-gpu/src/hierarchy.rs:258-270; opaque objects). */
typedef struct cc_instance {
  uint32_t geometry;
  float rotation[9];
  float scale;
  float translation[3];
} cc_instance;

/* An instanced scene (flatten_instanced, hierarchy.rs:464-522): each
 * geometry's triangles (9 floats each, object space) and triangle hierarchy
 * once, one object per instance pointing at its geometry with a transform,
 * and the object hierarchy over the objects' padded world bounds
 * (object_hierarchy, :198-253). Cones are walked into each object's space as
 * the reference's cone_to_object does (mask_cones.wgsl:623-638). The
 * transforms are stored as the reference's shader reads them: rows 0-2 of the
 * rotation with the translation in w, then (scale, 1 / scale, clear, 0)
 * (clear 0: see cc_scene_set_clear). With ctx
 * NULL the scene stays on the host. */
CC_API int cc_scene_build_instanced(cc_context* ctx, const float* tri9, const uint32_t* geometry_counts,
                                    uint32_t ngeometries, const cc_instance* instances, uint32_t ninstances,
                                    const uint32_t* movable, uint32_t nmovable, cc_scene** out);
/* With `movable` objects (nmovable > 0, some object staying static) the
 * object hierarchy keeps them in a subtree of their own under the root
 * (object_hierarchy_with_movers, hierarchy.rs:331-369); cc_scene_move places
 * them anew (placements in `movable` order, same geometries), rebuilds that
 * subtree (mover_subtree, :383-410) and updates the device copy. boxes12
 * (nullable) receives per mover its padded world bounds before and after
 * (lo.xyz, hi.xyz each): the input of cc_stale_cones. */
CC_API int cc_scene_move(cc_scene* scene, const cc_instance* placements, uint32_t nplacements, float* boxes12);
/* Each object's `clear` (Placement::clear, hierarchy.rs:266-270; one value per
 * object, in build order): 0 opaque; in (0, 1) alpha-blended, its shadows
 * keeping that share of the light (its triangles drawn with weight 1 - clear);
 * below 0 transmissive, thin glass passing -clear of the light less Schlick's
 * Fresnel reflectance at the cone's central direction; at most -2 a volume
 * passing -2 - clear through two surfaces (add_mesh_coverage_if and
 * cover_triangle, mask_cones.wgsl:600-614, :725-741). Stored in each
 * transform's row 3 (its z) as the reference stores it, kept by
 * cc_scene_move; prefiltered cones' coverage samples scale by the opacity of
 * the first object placing each geometry (hierarchy.rs:469-503). Values of
 * 1 and more, and non-finite ones, are refused. */
CC_API int cc_scene_set_clear(cc_scene* scene, const float* clear, uint32_t nobjects);
/* The cones that moved objects may have changed: cone (light l, point p) is
 * stale when a mover's box, old or new, meets the convex hull of p and the
 * light's box (hull_meets, mask_cones.wgsl:3903-3917, after the shadow-region
 * prefilter of hierarchy.rs:418-457). receivers and stale (1 byte per cone,
 * light-major) are device pointers; lights (16 floats each) and boxes12 are
 * host arrays. Waits for the result; *count receives the stale cones. */
CC_API int cc_stale_cones(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                          const float* lights, uint32_t nlights, const float* boxes12, uint32_t nmovers,
                          uint8_t* stale, uint64_t* count, void* stream);
/* The scene's transforms (16 floats each) into out16 (nullable, at most
 * max_transforms); returns their count (0 for a scene without instancing). */
CC_API uint64_t cc_scene_transforms(const cc_scene* scene, float* out16, uint64_t max_transforms);

/* Sizes of the scene's flattened host arrays: ntris, nmeshes, nblas,
 * nblas_items, nnodes, nitems; and copies of them (NodeGpu layout, any
 * pointer may be NULL). For checking the host builder. */
CC_API int cc_scene_sizes(const cc_scene* scene, uint64_t out6[6]);
CC_API int cc_scene_arrays(const cc_scene* scene, uint32_t* ranges, void* blas, uint32_t* blas_items, void* nodes,
                    uint32_t* items);
/* Device bytes the scene holds. */
CC_API uint64_t cc_scene_device_bytes(const cc_scene* scene);

/* Shading points of a pinhole camera: for each pixel (row-major) the nearest
 * hit's point lifted off the surface and its geometric normal facing the
 * camera, as the reference's camera pass forms them (camera_dir, primary_hit,
 * surface_offset: mask_cones.wgsl:1724-1760, 2062-2064, 2275-2277). Host
 * threads; for preparing inputs. camera: eye.xyz, target.xyz, up.xyz,
 * vertical fov in degrees. out8: 8 floats per pixel (receiver layout; point.w
 * holds the hit object's index and normal.w the hit triangle's index + 1, as
 * the bits of uint32s: the inputs of CC_SKY_OBJECT_FRAME and CC_BACK_FACING);
 * hit: 1 per pixel, 0 where the ray misses (its receiver is zero). */
CC_API int cc_scene_primary_hits(const cc_scene* scene, const float camera[10], uint32_t width, uint32_t height,
                                 float* out8, uint8_t* hit);

typedef struct cc_options {
  uint32_t hierarchy;        /* 0: every triangle; 1: mesh hierarchy; 2: + triangle hierarchies (Hierarchy, hierarchy.rs:731-749) */
  float wide_extent;         /* WIDE_EXTENT, mask_cones.wgsl:1048 (8.0) */
  uint32_t light_cone_cap;   /* LIGHT_CONE_CAP, mask_cones.wgsl:1052 (4096) */
  uint32_t wide_cone_cap;    /* WIDE_CONE_CAP, mask_cones.wgsl:1056 (512) */
  uint32_t points_per_warp;  /* cones walked together per warp: 1..32 (32); results do not depend on it */
  uint32_t flags;            /* CC_DEVICE_POINTERS, CC_NO_REDO, CC_KEEP_ORDER, CC_NO_OBJECT_PREFILTER, CC_BACK_FACING */
  float prefilter;           /* prefiltered cones (MaskConeKernel::set_prefilter, lib.rs:1508): a hierarchy node
                                wholly between the near and far planes projecting to at most this many bins is
                                splatted with its directional coverage instead of descended into
                                (node_cone_test, mask_cones.wgsl:519-574; object nodes of instanced scenes:
                                splat_object_node, :1096-1150). 0: exact cones. Needs hierarchy 2; cc_visibility
                                and cc_sky_visibility only */
} cc_options;

/* cc_options.flags: the lighting cache's estimator for a light below a
 * receiver's horizon (vc_bake's `back`, mask_cones.wgsl:3476-3494): a cone
 * whose light gives the receiver no unshadowed light (its normal turns away)
 * but which faces the light is traced with a horizon facing the light (the
 * normal replaced by the direction to the light's centre), past the
 * receiver's own triangle, so its fraction is the light's share seen past
 * that triangle (1 on a convex object's terminator, the shadow's where
 * something else covers it); its irradiance is 0. The receiver's normal.w
 * holds its own triangle's index in the scene's triangle order plus one, as
 * the bits of a uint32 (cc_scene_primary_hits writes it); a receiver without
 * one (0) keeps its normal. cc_visibility only, exact cones of a scene
 * without instancing. */
#define CC_BACK_FACING 16u

/* Defaults: hierarchy 2, 8.0, 4096, 512, 32, 0, prefilter 0. */
CC_API void cc_options_default(cc_options* opt);

typedef struct cc_outputs {
  uint32_t* full;        /* 2 words per cone: bins wholly covered (nullable) */
  uint32_t* any;         /* 2 words per cone: bins with coverage > 0 (nullable) */
  float* partial;        /* 64 per cone: per-bin coverage in [0, 1] (nullable) */
  float* irradiance;     /* 1 per cone: irradiance per unit radiance (nullable) */
  float* fraction;       /* 1 per cone: visible fraction of the unshadowed light (nullable) */
  uint32_t* work;        /* 4 per cone: object nodes, triangle-hierarchy nodes, triangles tested; status bits (nullable) */
} cc_outputs;

/* Visibility of every (point, light) cone. Replaces the reference's light
 * cones as traced by hit_irradiance_rect (mask_cones.wgsl:2125-2128) for each
 * light of the `lights` list, with the lighting cache's ratio
 * (vc_bake, mask_cones.wgsl:3453-3510) as `fraction`. `stream` is a
 * cudaStream_t (NULL: the context's stream). With host pointers the call
 * returns when the results are in the host buffers. */
CC_API int cc_visibility(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                  const float* lights, uint32_t nlights, const cc_options* opt, const cc_outputs* out,
                  void* stream);

/* The prefiltered cones' coverage samples of a scene's nodes (27 per node,
 * hierarchy.rs:710-723): of every triangle-hierarchy node (blas27, nullable,
 * up to max_blas nodes) and, for an instanced scene, of every object-hierarchy
 * node (obj27, nullable; sample 13 is 1 for a node without prefiltered
 * coverage, 0 otherwise). Host scenes too. Returns the triangle-hierarchy
 * node count, or minus a status code. */
CC_API int64_t cc_scene_coverage(const cc_scene* scene, float* blas27, uint64_t max_blas, float* obj27,
                                 uint64_t max_obj);

/* cc_sky_visibility flags */
#define CC_SKY_COMBINE_MAX 1u      /* meshes combine by the maximum, as light cones do (MaskConeKernel::set_sky_combination_max) */
#define CC_SKY_NO_HORIZON_CULL 2u  /* walk geometry below the receiver's horizon too (set_sky_horizon_cull(false)) */
#define CC_SKY_OBJECT_FRAME 4u     /* faces turn with the object each receiver lies on (set_sky_object_frame(true)):
                                      the receiver's point.w holds that object's index among the scene's meshes as
                                      the bits of a uint32 (0xffffffff, or an object without a transform: world
                                      axes); the cube's axes are the object's, turned to world space (sky_frame,
                                      mask_cones.wgsl:1432-1456, :2286) */

/* A uniform sky through six cube-face mask cones per receiver (the sky light
 * of mask_cones.wgsl:1323-1511, sky_irradiance :1411-1426, for a uniform sky
 * in world axes without prefiltering): `irradiance` receives per receiver the
 * irradiance per unit sky radiance, Σ over faces of the face's window clipped
 * to the receiver's horizon less its covered bins' clipped weights. Each face
 * (axis f / 2, negative for odd f) is a cone with a [-1, 1]^2 window reaching
 * 1e7 past the receiver, walked without a cap; meshes combine as independent
 * occluders, and geometry wholly below the receiver's tangent plane is
 * skipped (both as the reference defaults). `faces` (nullable) receives the
 * face cones' outputs as cc_visibility's, cone c = face * npoints + point.
 * opt->flags: CC_DEVICE_POINTERS (receivers, irradiance and faces on the
 * device; asynchronous), CC_NO_REDO, CC_KEEP_ORDER; the walk caps are unused. */
CC_API int cc_sky_visibility(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                             const cc_options* opt, uint32_t sky_flags, float* irradiance, const cc_outputs* faces,
                             void* stream);

/* Recomputes the stale cones of a cache of results (device arrays, as
 * cc_visibility with CC_DEVICE_POINTERS writes them; full, any, irradiance
 * and fraction) and leaves every other cone's results as they are. receivers,
 * lights and stale are device pointers. *recomputed (nullable) receives the
 * cones solved. Waits for the result. */
CC_API int cc_visibility_update(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                                const float* lights, uint32_t nlights, const uint8_t* stale, const cc_options* opt,
                                const cc_outputs* out, uint64_t* recomputed, void* stream);

/* No counterpart in the reference (whose kernel owns its wgpu buffers).
 * cc_visibility without allocation: the same results as cc_visibility with
 * CC_DEVICE_POINTERS, for at most CC_STATIC_MAX_CONES cones and as many points
 * per call (larger calls are rejected with CC_ERR_INVALID), with its scratch
 * in one fixed 48 MiB device array of the library per device instead of
 * context buffers: the counters (256 B), the re-walk list (4 B per cone), the
 * walk order (4 B per point), then the walk order's sort space, which the
 * split path's cone records (112 B per cone) and masks (256 B per cone) reuse
 * once the order is made. Every GPU that loads the library holds the 48 MiB
 * until the process exits. It calls no cudaMalloc, cudaFree or allocating library routine, so
 * it suits callers that cannot let the library allocate: a server that admits
 * scenes against a fixed device-memory budget or whose memory a caching
 * allocator owns (cc_visibility grows its context's buffers with cudaMalloc
 * to the largest call seen and keeps them), a loop that overlaps work on other
 * streams (cudaFree waits for the whole device), and a caller that must keep
 * working when device memory is exhausted.
 *  - Every pointer is a device pointer (CC_DEVICE_POINTERS is implied); the
 *    call is asynchronous on `stream` (NULL: the scene's context's stream).
 *  - The first call on a device looks up the array's address
 *    (cudaGetSymbolAddress, which loads the array's module) and may set the
 *    kernel's shared-memory attribute; make it before any stream capture.
 *  - The call zeroes the array's four counter words on the stream before its
 *    kernels run; nothing else in it needs a starting value.
 *  - All calls on one device share the array: calls whose work can overlap on
 *    the device (on different streams, or from several host threads) race and
 *    corrupt each other's results. Issue them on one stream, or order them.
 *  - No kernel times are recorded (cc_context_kernel_times does not see it).
 *  - The call does not wait, so it cannot return CC_ERR_STACK: a cone whose
 *    traversal stack overflowed is flagged only in its status word
 *    (CC_CONE_STACK in out->work's fourth word); ask for `work` to see it.
 *    The array's error word is cleared by the next call. */
#define CC_STATIC_MAX_CONES 131072u
CC_API int cc_visibility_static(const cc_scene* scene, const float* receivers, uint64_t npoints, const float* lights,
                                uint32_t nlights, const cc_options* opt, const cc_outputs* out, void* stream);

/* ---- Batched form -------------------------------------------------------
 * Many visibility jobs (each its own scene, receivers, lights, options and
 * outputs) solved by one persistent launch: a job table on the device, one
 * Morton sort over every job's points, then warps take packets of any job
 * from one device counter (a packet never straddles two jobs), so small and
 * uneven jobs share the GPU instead of each leaving it idle behind its own
 * tail. Each job's results equal cc_visibility's for that job alone.
 * The reference's counterpart is its bake job list (vc_bake's job packing,
 * mask_cones.wgsl:3433-3443), which packs many cache entries into one
 * dispatch; it has no general batch of scenes. */
typedef struct cc_batch cc_batch;

#define CC_BATCH_GRAPH 8u /* replay submissions from a captured CUDA graph (cc_batch_options.flags) */

typedef struct cc_batch_options {
  uint32_t points_per_warp; /* cones per packet: 1..32 (32) */
  uint32_t blocks_per_sm;   /* resident blocks per SM launched: 1..8 (8) */
  uint32_t flags;           /* CC_KEEP_ORDER, CC_NO_REDO, CC_BATCH_GRAPH */
} cc_batch_options;

/* Defaults: 32 cones per packet, 8 blocks per SM, CC_BATCH_GRAPH. */
CC_API void cc_batch_options_default(cc_batch_options* opt);

CC_API int cc_batch_create(cc_context* ctx, cc_batch** out);
CC_API int cc_batch_destroy(cc_batch* batch);
/* Removes every job (the batch's device buffers are kept for reuse). */
CC_API int cc_batch_clear(cc_batch* batch);
/* Appends a job. Receivers, lights and outputs are device pointers that must
 * stay valid while the batch is submitted; opt gives the job's hierarchy,
 * wide extent and walk caps (its points_per_warp and flags are ignored: the
 * batch's options apply). `job` (nullable) receives the job's index. At most
 * 2^32 - 1 cones over all jobs. The scene may be instanced
 * (cc_scene_build_instanced); a batch with such a job runs the instanced
 * kernel for all its jobs. */
CC_API int cc_batch_add(cc_batch* batch, const cc_scene* scene, const float* receivers, uint64_t npoints,
                        const float* lights, uint32_t nlights, const cc_options* opt, const cc_outputs* out,
                        uint32_t* job);
/* Appends an update job: cc_visibility_update's work inside the batch (the
 * reference has no batched form; its view cache re-bakes the stale entries of
 * moved objects' shadows, vcache.rs). `stale` (device, one byte per cone,
 * light-major, nonzero = stale) is read at each submission: only those cones
 * are walked, in the walk order, and written to out (full, any, irradiance,
 * fraction; partial and work are refused); every other cone's outputs keep
 * their contents. Each result equals cc_visibility_update's. */
CC_API int cc_batch_add_update(cc_batch* batch, const cc_scene* scene, const float* receivers, uint64_t npoints,
                               const float* lights, uint32_t nlights, const uint8_t* stale, const cc_options* opt,
                               const cc_outputs* out, uint32_t* job);
/* Enqueues the whole batch on `stream` (NULL: the context's stream) and
 * returns. The first submission after a change of jobs or options sizes the
 * batch's buffers and uploads the job table; with CC_BATCH_GRAPH it runs the
 * work directly and captures it into a CUDA graph, and later submissions with
 * the same jobs and options launch that graph. */
CC_API int cc_batch_submit(cc_batch* batch, const cc_batch_options* opt, void* stream);
/* Waits at most timeout_ms for the last submission: CC_ERR_TIMEOUT if it has
 * not finished, CC_ERR_STACK if a traversal stack overflowed, else CC_OK. */
CC_API int cc_batch_wait(cc_batch* batch, uint32_t timeout_ms);
/* The autotuner: times every candidate launch configuration (cones per
 * packet 8, 16, 32 x Morton or given walk order x 4 or 8 blocks per SM) on
 * this batch, `reps` runs each, and writes the fastest to *best (keeping
 * base->flags' CC_BATCH_GRAPH and CC_NO_REDO; base nullable). ms_out
 * (nullable, max_candidates entries) receives each candidate's best time in
 * candidate order. Returns the number of candidates, or minus a status.
 * Results do not depend on the configuration. */
CC_API int cc_batch_tune(cc_batch* batch, const cc_batch_options* base, uint32_t reps, cc_batch_options* best,
                         float* ms_out, uint32_t max_candidates);
/* jobs, points, cones, and device bytes the batch holds. */
CC_API int cc_batch_sizes(const cc_batch* batch, uint64_t out4[4]);

/* ---- Served form --------------------------------------------------------
 * A request loop on its own host thread. Scenes stay resident; requests
 * (a scene, receivers, 1 or more lights) queue on submission and are admitted
 * earliest deadline first (deadline_ns_per_cone > 0, the default) or in
 * arrival order (0), while launch slots and device memory under the server's
 * budget allow: a
 * request's deadline is its submission time plus deadline_ns_per_cone for each
 * of its cones, so small requests overtake large ones that have not waited
 * about as long as the small ones take, and no request waits forever. The
 * first (most urgent) queued request that does not fit the memory left holds
 * back the rest. In arrival order, admission into a launch stops at the first
 * request that does not fit its cone limit. By deadline, such a request waits
 * for the next launch while less urgent ones join this one, and while a
 * request within the limit waits, requests above it (each launched alone)
 * take at most max_inflight - 1 slots, so that smaller ones find a slot.
 * Each launch takes every admitted request (continuous
 * batching: requests that arrive while earlier launches run join the next
 * one, and up to max_inflight launches overlap on the device on their own
 * streams); every (request, light) pair is one job of a batched launch.
 * Results of a request with a nonzero cache_key stay on the device as a
 * lighting cache, one entry per (cache_key, light geometry): a later request
 * with the same key and a light of the same geometry (a recoloured light:
 * only the radiance differs) is served from the entry without tracing.
 * Entries are evicted least recently used when admission needs the memory.
 * Each result equals cc_visibility's for that request alone.
 * The reference has no request server; its nearest counterpart is the
 * lighting cache's frame-budgeted bake (CacheOptions.bake_budget and
 * frame_target_ms, crates/continuum/src/vcache.rs:183-207). */
typedef struct cc_server cc_server;

typedef struct cc_server_options {
  uint64_t hbm_budget;       /* device bytes for requests in flight and cached results, reserved by the
                                server at creation when the device has room (held until destroyed) */
  uint32_t max_inflight;     /* launches in flight at once: 1..8 (4) */
  uint32_t max_queue;        /* queued requests before submissions are refused with CC_ERR_BUSY (256) */
  uint64_t max_launch_cones; /* cones one launch takes at most (2M); one larger request runs alone */
  uint32_t points_per_warp;  /* 1..32 (32) */
  uint32_t blocks_per_sm;    /* 1..8 (8) */
  uint32_t deadline_ns_per_cone; /* admission earliest deadline first, deadline = submission + this per
                                    cone (12: about one B200's rate on a plain scene); 0: arrival order */
} cc_server_options;

/* Defaults: 8 GiB budget, 4 in flight, 256 queued, 2M cones per launch, 32, 8, 12 ns per cone. */
CC_API void cc_server_options_default(cc_server_options* opt);

typedef struct cc_request {
  uint32_t scene;            /* an index from cc_server_add_scene */
  const float* receivers;    /* host, 8 floats per point (pinned memory lets the copies overlap) */
  uint64_t npoints;
  const float* lights;       /* host, 16 floats per light */
  uint32_t nlights;
  uint32_t hierarchy;        /* 0, 1 or 2 */
  uint64_t cache_key;        /* 0: no caching; else names this receiver set for the lighting cache */
  uint32_t* full;            /* host outputs, light-major as cc_visibility's (nullable); written when done */
  uint32_t* any;
  float* irradiance;
  float* fraction;
  float prefilter;           /* prefiltered cones, as cc_options.prefilter (bins; 0: exact cones; needs hierarchy 2) */
} cc_request;

typedef struct cc_request_stats {
  double queued_ms;          /* submission to admission */
  double total_ms;           /* submission to completion (results in the host buffers) */
  uint32_t launch_requests;  /* requests in the launch that served it */
  uint32_t cached_lights;    /* lights served from the lighting cache */
} cc_request_stats;

CC_API int cc_server_create(cc_context* ctx, const cc_server_options* opt, cc_server** out);
/* Finishes every queued and running request, then stops the loop. */
CC_API int cc_server_destroy(cc_server* server);
/* Makes a scene of the server's context resident for requests (instanced or
 * not); `id` receives its index. The scene must outlive the server. */
CC_API int cc_server_add_scene(cc_server* server, const cc_scene* scene, uint32_t* id);
/* Queues a request (its receivers are read, and its outputs written, by the
 * server's thread: they must stay valid until the request completes; its
 * lights are copied). CC_ERR_BUSY when the queue is full or the request alone
 * exceeds the budget. */
CC_API int cc_server_submit(cc_server* server, const cc_request* req, uint64_t* ticket);
/* Waits at most timeout_ms for a request: CC_OK with its stats (nullable)
 * when done, CC_ERR_TIMEOUT if not, or the status it failed with. A ticket is
 * forgotten once its wait returns anything but CC_ERR_TIMEOUT. */
CC_API int cc_server_wait(cc_server* server, uint64_t ticket, uint32_t timeout_ms, cc_request_stats* stats);
/* Counters: completed, refused, launches, cached lights served, lights
 * traced, device bytes in use, peak device bytes, cache entries. */
CC_API int cc_server_stats(cc_server* server, uint64_t out8[8]);

/* Kernel times of the cc_visibility calls made on this context since the
 * last query, oldest first (the last 256 calls at most): per call, the packet
 * pass and the solo re-walk pass in milliseconds, from CUDA events recorded
 * on the call's stream around each launch. The reference's counterpart is its
 * GPU timestamp queries (crates/continuum-gpu/src/lib.rs:1081-1090). Waits
 * for those calls to finish. Returns the number of calls written to out2
 * (2 floats each, at most max_calls), or minus a status code. */
CC_API int cc_context_kernel_times(cc_context* ctx, float* out2, int max_calls);

/* Replaces MaskConeKernel::irradiance / irradiance_with
 * (crates/continuum-gpu/src/lib.rs:1706-1730): irradiance per unit radiance
 * at each receiver (6 floats: point.xyz, normal.xyz) from a rect light
 * (9 floats: corner, edge_u, edge_v; one_sided 0/1) over meshes given as
 * 9 floats per triangle. The hierarchy is built and the scene uploaded on
 * every call, as the reference does; `best_seconds` (nullable) receives the
 * fastest of `runs` kernel executions (upload and readback excluded, as in
 * lib.rs:3496-3512). hierarchy: 0 (irradiance), 1 or 2 (irradiance_with). */
CC_API int cc_irradiance(cc_context* ctx, const float* receivers6, uint64_t npoints, const float* light9, int one_sided,
                  const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes, uint32_t hierarchy,
                  uint32_t runs, float* out, double* best_seconds);

/* Replaces MaskConeKernel::coverage (crates/continuum-gpu/src/lib.rs:3289-3298):
 * 64 per-bin coverages per receiver, every triangle tested (hierarchy 0). */
CC_API int cc_coverage(cc_context* ctx, const float* receivers6, uint64_t npoints, const float* light9, int one_sided,
                const float* tri9, const uint32_t* mesh_counts, uint32_t nmeshes, float* out64);

/* ---- The lighting cache's bake (the consumer of the visible fraction) ------
 * Replaces the direct-light bake of crates/continuum-gpu/src/vcache.rs
 * (`VirtualCache`: the page manager `plan` :3704, `plan_page` :3928, the
 * adaptive budget of `begin_frame` :2976-3080) and the `vc_bake` pass
 * (mask_cones.wgsl:3433-3554) for static lights. Pages are 8 x 8 texels
 * stored 9 x 9 (81, row-major); the pool holds one channel per light:
 * pool[(slot * 81 + texel) * nlights + light]. Each frame the page requests
 * are planned in priority order within the bake budget (cones: a page costs
 * its inside texels x lights; the first page always fits), new pages take
 * free slots (pages unused for 64 frames are evicted once a quarter of the
 * pool is resident; when the pool is full, pages unused for 2 frames), and
 * the planned pages' listed texels (inside + 1 per axis, at most 9) are baked
 * for every light: one cone per job [bake-list index, texel | light << 8].
 * The pool receives the visible fraction of the unshadowed light (the
 * reference's `light_ratio`) or the shadowed light; a texel without a
 * surface receives 0, one outside the chart's grid nothing. Not built: sky
 * samples, bounce light, moving lights (lattice, ledger), lighting levels and
 * the light-below-the-horizon estimator (such texels take ratio 1, as the
 * reference gives moving lights). */
typedef struct cc_cache cc_cache;
typedef struct cc_planner cc_planner;

typedef struct cc_cache_options {
  uint32_t pages;          /* pool slots (CacheOptions::pages, vcache.rs:218) */
  uint32_t bake_budget;    /* the most cones a frame (CacheOptions::bake_budget, :183) */
  float frame_target_ms;   /* the frame period the bake aims for; 0: always bake_budget (:194) */
  float frame_budget_ms;   /* frames are capped to this period (0: no cap; :196-207) */
  float floor_overrun;     /* CacheOptions::floor_overrun (:208-213) */
  uint32_t light_ratio;    /* 1: the pool keeps the visible fraction; 0: the shadowed light */
} cc_cache_options;

/* Defaults: 65,536 pages, 1,048,576 cones, 0 ms, 0 ms, 0.25, light_ratio 1. */
CC_API void cc_cache_options_default(cc_cache_options* opt);

typedef struct cc_page_request {
  uint32_t key[3];        /* the page's identity (object, chart and mip, page coordinates: the caller's packing) */
  uint32_t priority;      /* lower first */
  uint32_t inside[2];     /* texels of the page inside its chart's grid along x and y (0..9) */
  const float* texels;    /* 81 receiver records of 8 floats (point.xyz, flag, normal.xyz, own), row-major 9 x 9;
                             flag 0: outside the chart's grid, 1: inside without a surface, 2: a surface to bake;
                             own: the texel's triangle's index + 1 as the bits of a uint32 (0: not named), so that
                             a light below the texel's horizon bakes the share seen past that triangle (vc_bake's
                             `back`, mask_cones.wgsl:3476-3494; scenes without instancing), else ratio 1.
                             Host memory, read during cc_cache_frame; may be null for pages that are resident */
} cc_page_request;

typedef struct cc_cache_frame_info {
  float period_ms;        /* the previous frame's period (<= 0: not known) */
  float render_ms;        /* the previous frame's camera passes on the GPU (ms) */
  uint32_t gpu_waited;    /* 1 if the CPU waited more than 1 ms for the GPU in the previous frame */
} cc_cache_frame_info;

typedef struct cc_cache_stats {
  float budget;           /* this frame's bake budget (cones) */
  uint32_t frame;         /* this frame's number */
  uint32_t pages_planned; /* pages baked this frame */
  uint32_t jobs;          /* cones baked this frame (listed texels x lights) */
  uint32_t spent;         /* budget spent (inside texels x lights) */
  uint32_t resident;      /* pages resident after planning */
  uint32_t evicted;       /* pages evicted so far */
  float last_bake_ms;     /* the previous frame's bake on the GPU (ms; < 0: none) */
} cc_cache_stats;

/* A cache of `scene` (which must outlive it) lit by `nlights` static lights
 * (16 floats each, copied). */
CC_API int cc_cache_create(cc_context* ctx, const cc_scene* scene, const float* lights, uint32_t nlights,
                           const cc_cache_options* opt, cc_cache** out);
CC_API int cc_cache_destroy(cc_cache* cache);
/* One frame: the previous bake's GPU time feeds the budget, the requests are
 * planned, and the planned pages are baked on the context's stream (not
 * waited for). A request for a resident page counts as its use this frame.
 * `info` and `stats` are nullable. */
CC_API int cc_cache_frame(cc_cache* cache, const cc_page_request* requests, uint32_t nrequests,
                          const cc_cache_frame_info* info, cc_cache_stats* stats);
/* A resident page's 81 x nlights pool values (texel-major), after its bake:
 * CC_OK, or CC_ERR_INVALID if the page is not resident. */
CC_API int cc_cache_read(cc_cache* cache, const uint32_t key[3], float* out);
/* The device pool and its channel count (lights). */
CC_API int cc_cache_pool(cc_cache* cache, float** pool, uint32_t* channels);
/* The last frame's bake job list: pairs [bake-list index, texel | light << 8]
 * (at most max_jobs written), and per planned page its slot. Returns the job
 * count, or minus a status code. */
CC_API int64_t cc_cache_jobs(cc_cache* cache, uint32_t* jobs2, uint64_t max_jobs, uint32_t* page_slots,
                             uint32_t max_pages);

/* The page manager alone, on the host (no device work): the same planning
 * and budget as cc_cache_frame, with the bake's GPU time supplied. */
CC_API int cc_planner_create(const cc_cache_options* opt, uint32_t nlights, cc_planner** out);
CC_API int cc_planner_destroy(cc_planner* planner);
/* begin the frame (bake_ms < 0: no timing of the previous bake, else its GPU
 * time over the previous frame's spent budget), plan it, end it. */
CC_API int cc_planner_frame(cc_planner* planner, const cc_page_request* requests, uint32_t nrequests,
                            const cc_cache_frame_info* info, float bake_ms, cc_cache_stats* stats);
/* The last planned frame's jobs and page slots, as cc_cache_jobs. */
CC_API int64_t cc_planner_jobs(cc_planner* planner, uint32_t* jobs2, uint64_t max_jobs, uint32_t* page_slots,
                               uint32_t max_pages);
/* The slot of a resident page, or -1. */
CC_API int64_t cc_planner_slot(cc_planner* planner, const uint32_t key[3]);

#ifdef __cplusplus
}
#endif

#endif /* CONTINUUM_CUDA_H */
