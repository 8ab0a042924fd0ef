// Launch interface between the host library and the device kernels.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "cone_device.cuh"

namespace cc {

constexpr int kWarpsPerBlock = 2;
// Resident blocks per SM the shared memory allows. Passes that keep each
// cone's coverages in thread-local memory (the split path's, exact sky
// cones'): the packet pass (32-bit accumulator cells, 22 KB per block) fits
// 8, the solo pass (64-bit cells, 38 KB) 5; prefiltering sky cones, whose
// walk needs more registers, 6 and 5. Prefiltering light cones keep them in
// shared memory: 5 and 4.
constexpr int kBlocksPerSm = 8;
constexpr int kSoloBlocksPerSm = 5;
constexpr int kFusedBlocksPerSm = 5;
constexpr int kFusedSoloBlocksPerSm = 4;
constexpr int kSkySplatBlocksPerSm = 6;  // prefiltering sky cones' packet pass (thread-local coverages)

struct DevQuery {
  const float4* receivers;  // 2 per point: point, normal
  const float4* lights;     // 4 per light (LightGpu)
  uint64_t npoints;
  uint32_t nlights;
  uint32_t hierarchy;
  float wide_extent;
  uint32_t light_cone_cap;
  uint32_t wide_cone_cap;
  // The walk order of the points (a permutation; null: as given). Slot s
  // walks cone (s / npoints) * npoints + order[s % npoints].
  const uint32_t* order;
  // kSkyCones: the query's cones are sky cones, the six cube faces around
  // each receiver (nlights = 6, lights unused), with the flags below.
  uint32_t sky = 0;
  // Prefiltering cones: nodes projecting to at most this many bins are
  // splatted (0: exact cones). Hierarchy level 2 only.
  float prefilter = 0.0f;
  // A cone list (null: every cone): slot s walks cone cones[s] for s below
  // *cones_count (device memory), in the list's order; outputs stay indexed
  // by cone (light * npoints + point).
  const uint32_t* cones = nullptr;
  const uint32_t* cones_count = nullptr;
  // The split plain path (exact light cones): slots slot_base .. + slot_count
  // of this call's walk, each set up beforehand in records[slot - slot_base].
  const struct ConeRecord* records = nullptr;
  uint64_t slot_base = 0;
  uint64_t slot_count = 0;
  // CC_BACK_FACING (exact light cones of a world-space scene): a cone whose
  // light lies below its receiver's horizon is traced with a horizon facing
  // the light, past the receiver's own triangle, whose index + 1 the
  // receiver's normal.w holds as bits (0: none); tri_slot maps a triangle's
  // index to its slot on the device (ntris of them).
  uint32_t back = 0;
  uint32_t ntris = 0;
  const uint32_t* tri_slot = nullptr;
  // The split path's light order (null: the given order): slots of light
  // rank r walk light light_order[r]'s cones. Results do not depend on it;
  // lights whose cones are wider go first, so their costlier packets do not
  // start last (light_order_kernel).
  const uint32_t* light_order = nullptr;
};

// A light cone set up before its walk (the split plain path): frame, window,
// far plane and bounding cone, its walk cap, flags and spot factor, and its
// cone number.
struct ConeRecord {
  float4 a;  // apex.xyz, far_offset
  float4 b;  // right.xyz, u0
  float4 c;  // up.xyz, v0
  float4 d;  // fwd.xyz, u1
  float4 e;  // baxis.xyz, v1
  float4 f;  // bcos, bsin, spot, flags (bits: 1 traced, 2 wide window, 4 wide window clipped, 8 traced past
             // the receiver's own triangle toward a light below its horizon; bits 4-31: that triangle's slot + 1)
  uint4 g;   // cone number (low, high words), walk cap, job (batched; else 0)
};
// Slots per split chunk by default (records and masks: 368 bytes a slot).
static_assert(sizeof(ConeRecord) == 112, "cone record layout");
constexpr uint64_t kSplitChunk = 1ull << 25;
constexpr uint32_t kSkyCones = 1u;
constexpr uint32_t kSkyCombineMax = 2u;      // combine meshes by the maximum, as light cones do (a diagnostic)
constexpr uint32_t kSkyNoHorizonCull = 4u;   // walk geometry below the receiver's horizon too
constexpr uint32_t kSkyObjectFrame = 8u;     // faces turn with the object each receiver lies on (point.w)

// Scratch bytes walk_order needs for `npoints` receivers.
size_t walk_order_scratch_bytes(uint64_t npoints);
// Morton order of the receivers' positions in the scene's bounds, into
// `order` (npoints entries), on `stream`.
cudaError_t walk_order(const float4* receivers, uint64_t npoints, const float* scene_lo, const float* scene_hi,
                       void* scratch, size_t scratch_bytes, uint32_t* order, cudaStream_t stream);

// The stale cones of a (light, point) grid as one list, each light's in the
// points' walk order (`order`, or their own order when null): `stale` holds a
// byte per cone (light-major), `perm` and `flags` take a word and a byte per
// cone, `count` the list's length; `temp` (stale_list_scratch_bytes) is the
// selection's scratch. On `stream`.
size_t stale_list_scratch_bytes(uint64_t ncones);
cudaError_t stale_list(const uint32_t* order, const uint8_t* stale, uint64_t npoints, uint32_t nlights, uint32_t* perm,
                       uint8_t* flags, uint32_t* list, uint32_t* count, void* temp, size_t temp_bytes,
                       cudaStream_t stream);

struct DevOut {
  uint2* full;
  uint2* any;
  float* partial;
  float* irradiance;
  float* fraction;
  uint4* work;
  // Scratch: cones to walk again alone, their count, the list's capacity,
  // and an error word (bit 0: list overflow, bit 1: stack overflow).
  uint32_t* redo_list;
  uint32_t* redo_count;
  uint32_t redo_capacity;
  uint32_t* error;
  // Work counters: the next packet of the packet pass and of the solo pass.
  uint32_t* next_packet;
  uint32_t* next_solo;
  // The split plain path: each slot's mask (64 coverages), for the
  // integration after the walk; the solo pass lists slots, not cones.
  float* cov_out = nullptr;
};

// Scratch words per call: redo count, error word, packet and solo counters.
constexpr int kCounterWords = 4;

// One job of a batch: its scene, query and outputs, and where its packets,
// cones and points start in the batch's numbering. A batch's packets never
// straddle two jobs.
struct JobGpu {
  DevScene scene;
  DevQuery query;  // query.order is unused: the batch's order array holds every job's
  uint2* full;
  uint2* any;
  float* partial;
  float* irradiance;
  float* fraction;
  uint4* work;
  uint64_t packet_start;
  uint64_t cone_start;
  uint64_t point_start;
  float lo[3], hi[3];  // the scene's bounds (Morton quantization)
};

// A batch launch: the job table and the batch's sizes. The redo list and
// counters are DevOut's scratch fields (its output pointers are unused).
struct BatchLaunch {
  const JobGpu* jobs;
  uint32_t njobs;
  uint64_t packets;  // packets of all jobs at `pw` cones per packet
  uint64_t points;   // points of all jobs
  uint32_t pw;
  // The walk order of every job's points (job j's at order + point_start,
  // job-local indices), or null: each job's points in their given order.
  const uint32_t* order;
  // The split path's chunk (set by launch_batch): packets packet_base ..
  // + packet_count, whose cones are batch cones cone_base .. + cone_count,
  // each set up in records[cone - cone_base].
  ConeRecord* records = nullptr;
  uint64_t packet_base = 0, packet_count = 0;
  uint64_t cone_base = 0, cone_count = 0;
  // Some job walks hierarchy level 0 or 1 (the kernel variant that carries
  // those levels' code is launched).
  uint32_t flat_levels = 0;
  // Some job's scene is instanced (the instanced variant is launched).
  uint32_t inst = 0;
};

// A chunk of a batch for the split path: whole packets, at most the chunk's
// slot count of cones.
struct BatchChunk {
  uint64_t packet_base, packet_count, cone_base, cone_count;
};
// The chunks of a batch whose jobs (in order) hold `cones[j]` cones, at `pw`
// cones a packet and at most `max_slots` cones a chunk (max_slots >= pw).
std::vector<BatchChunk> batch_chunks(const std::vector<uint64_t>& cones, uint32_t pw, uint64_t max_slots);

// Morton walk order of every job's points in one sort: keys are the job index
// above each point's 30-bit code, values the job-local point index; job j's
// order lands at order + jobs[j].point_start.
size_t batch_order_scratch_bytes(uint64_t points);
cudaError_t batch_order(const BatchLaunch& b, void* scratch, size_t scratch_bytes, uint32_t* order,
                        cudaStream_t stream);

// Per chunk (batch_chunks), the cones set up into b.records, the packet pass,
// the solo pass over the slots it listed, and the masks (o.cov_out, one
// chunk's) integrated into each job's irradiance and fraction.
// o.redo_count, o.error and the two packet counters must be zero on entry.
// blocks_per_sm: resident blocks per SM to launch (1..kBlocksPerSm).
// A batch's prefiltering jobs (visibility_splat.cu): one persistent launch of
// the prefiltering kernel over their packets (walk and integration), then
// their listed cones alone.
cudaError_t launch_batch_splat(const BatchLaunch& b, const DevOut& o, bool count, int sm_count, int blocks_per_sm,
                               cudaStream_t stream);
cudaError_t launch_batch(const BatchLaunch& b, const DevOut& o, const BatchChunk* chunks, size_t nchunks,
                         bool count_work, int sm_count, int blocks_per_sm, cudaStream_t stream);

// Scratch of cc_visibility_static: a file-scope device array of
// kStaticScratchBytes per device, laid out as the counters (256 bytes), the
// redo list (4 bytes per cone), the walk order (4 bytes per point) and the
// rest, which holds the walk order's sort scratch while the order is made,
// then the split path's cone records (112 bytes per cone) and masks (256).
constexpr uint32_t kStaticMaxCones = 1u << 17;  // cones (and points) per call: 131,072
constexpr size_t kStaticRedoOffset = 256;
constexpr size_t kStaticOrderOffset = kStaticRedoOffset + 4 * size_t(kStaticMaxCones);
constexpr size_t kStaticSortOffset = kStaticOrderOffset + 4 * size_t(kStaticMaxCones);
constexpr size_t kStaticRecordsOffset = kStaticSortOffset;
constexpr size_t kStaticMasksOffset = kStaticRecordsOffset + sizeof(ConeRecord) * size_t(kStaticMaxCones);
constexpr size_t kStaticScratchBytes = size_t(48) << 20;
static_assert(kStaticMasksOffset + 256 * size_t(kStaticMaxCones) <= kStaticScratchBytes, "static scratch too small");
static_assert(kStaticMaxCones <= kSplitChunk, "a static call is one split chunk");
// The array's device address on `device` (the current device). The first
// call per device looks it up; later calls return the cached address.
cudaError_t static_scratch(int device, void** ptr);

cudaError_t upload_disk_table(const float* table64);
// The prefiltering unit's copy of the table, and its plain passes (packet
// pass with 32-bit cells, or solo pass with 64-bit ones when `wide`).
cudaError_t upload_disk_table_splat(const float* table64);
cudaError_t launch_splat_pass(bool wide, bool count, bool inst, bool sky, const DevScene& s, const DevQuery& q,
                              const DevOut& o, const uint32_t* list, const uint32_t* list_count, uint32_t pw,
                              uint32_t blocks, cudaStream_t stream);

// The split plain path's kernels (visibility_split.cu): the unit's copy of
// the table; slots base .. base + n - 1 set up into records[0 .. n - 1]; and
// their masks (o.cov_out) integrated into o.irradiance and o.fraction.
cudaError_t upload_disk_table_split(const float* table64);
cudaError_t launch_cone_setup(const DevQuery& q, uint64_t base, uint64_t n, ConeRecord* records, cudaStream_t stream);
// The query's lights in decreasing order of the mean window of their cones
// over a sample of the points (at most 1024 lights), into `out`.
constexpr uint32_t kMaxOrderedLights = 1024;
cudaError_t launch_light_order(const DevQuery& q, uint32_t* out, cudaStream_t stream);
cudaError_t launch_integrate(const DevQuery& q, const DevOut& o, uint64_t base, uint64_t n, const ConeRecord* records,
                             cudaStream_t stream);
// Batched: the batch cones of chunk b (b.cone_base .. + b.cone_count).
cudaError_t launch_batch_setup(const BatchLaunch& b, cudaStream_t stream);
cudaError_t launch_batch_integrate(const BatchLaunch& b, const DevOut& o, cudaStream_t stream);

// The packet pass over every cone, then (with o.redo_list) the solo pass over
// the cones it listed. o.redo_count and o.error must be zero on entry. Exact
// light cones take the split path: per chunk of chunk_slots slots, setup,
// the two passes and the integration; q.records and o.cov_out then hold
// min(cones, chunk_slots) slots.
// `marks` (nullable): three events recorded before the packet pass (split:
// after the first chunk's setup), between the passes and after the solo pass
// (split: after the last integration).
// `walked` (nullable, split path): recorded once every walk pass has run,
// when FULL, ANY and the per-bin coverages are final.
cudaError_t launch_visibility(const DevScene& s, const DevQuery& q, const DevOut& o, uint32_t points_per_warp,
                              bool count_work, uint64_t chunk_slots, int sm_count, cudaStream_t stream,
                              const cudaEvent_t* marks, cudaEvent_t walked);

}  // namespace cc
