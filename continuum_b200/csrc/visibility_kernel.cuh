// The visibility kernel and its launch templates, shared by the translation
// units that instantiate its variants: visibility.cu (exact cones) and
// visibility_splat.cu (prefiltering cones). Instantiating both families in
// one unit changed the exact kernel's code, which is sensitive to its size
// (instruction fetch), so each family is compiled alone.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "cone_device.cuh"
#include "kernels.h"
#include "splat_device.cuh"

namespace cc {

static __constant__ float c_disk[kBins];  // DISK (mask_cones.wgsl:888-897), uploaded by the host

constexpr int kStack = 64;         // entries; the reference's is 48 (mask_cones.wgsl:111)
constexpr int kConeFields = 17;    // apex, right, up, forward, window, far offset
// Pairs passed to rasterization wait in a per-warp queue until 32 are ready:
// a cull round adds at most 32 to at most 31 waiting. Pairs that need the
// general clip path wait in a second queue of the same size.
constexpr int kQueueCap = 64;
constexpr uint32_t kQueueOwnerShift = 26;  // entry: cone lane << 26 | triangle slot (< 2^26)
// Both queues' lengths in one word: fast queue in the low byte, general
// queue in the next (each below 32 between rounds).
__device__ __forceinline__ uint32_t fast_len(uint32_t q) { return q & 255u; }
__device__ __forceinline__ uint32_t general_len(uint32_t q) { return q >> 8; }
__device__ __forceinline__ uint32_t queue_lens(uint32_t fast, uint32_t general) { return fast | (general << 8); }

// Shared memory of one warp; Cell is the accumulator's cell: 32 bits in the
// packet pass, 64 in the solo pass. Sky: the warp walks sky cones, whose
// horizons are kept beside their frames. SmemCov: each cone's coverages are
// kept here, where the integration in the same kernel reads every lane's
// (else each lane keeps its own in thread-local memory, and the smaller
// block lets more warps be resident).
// Back: the launch's cones may skip their receiver's own triangle
// (CC_BACK_FACING); other launches compile without the check.
// Weighted: instanced scenes, whose placed objects may be alpha-blended or
// transmissive (the transform's `clear`): triangles are drawn with the
// current object's weight; other launches draw every triangle whole.
template <class CellT, bool Sky, bool SmemCov, bool Back = false, bool Weighted = false>
struct WarpShared {
  using Cell = CellT;
  static constexpr bool kSky = Sky;
  static constexpr bool kSmemCov = SmemCov;
  static constexpr bool kBack = Back;
  static constexpr bool kWeighted = Weighted;
  Cell acc[kBins * 32];                 // each cone's accumulator (fixed point, units of kFixUnit)
  float cone[kConeFields * 32];         // each cone's frame, field-major; the integration's scratch after the walk
  uint32_t span_lo[32], span_hi[32];    // each cone's accumulator rows written (the WGSL's span)
  uint32_t queue[kQueueCap];            // (cone, triangle) pairs that passed the cull, waiting to be rasterized
  uint32_t general[kQueueCap];          // pairs that need rasterize's general path, waiting for it
  uint32_t overflow[4];                 // word 0: cones whose 32-bit accumulation overflowed in the current mesh
  float horizon[Sky ? 3 * 32 : 4];      // sky cones: each cone's horizon, field-major
  float cov[SmemCov ? kBins * 32 : 4];  // each cone's 64 coverages, bin-major, lane innermost
  // The placed object being walked (Weighted): its triangles' weight and its
  // transmission (add_mesh_coverage_if's tri_weight / tri_transmit /
  // tri_volume, :725-741); weight 1 and no transmission elsewhere.
  float object_weight, object_transmit;
  uint32_t object_volume, object_pad;
};
static_assert(sizeof(WarpShared<unsigned int, false, true>) % 16 == 0, "warp shared block keeps 16-byte alignment");
static_assert(sizeof(WarpShared<unsigned long long, false, true>) % 16 == 0, "warp shared block keeps 16-byte alignment");
static_assert(sizeof(WarpShared<unsigned int, true, true>) % 16 == 0, "warp shared block keeps 16-byte alignment");
static_assert(sizeof(WarpShared<unsigned int, false, false>) % 16 == 0, "warp shared block keeps 16-byte alignment");
template <bool kSky, bool kSmemCov, bool kBack = false, bool kWeighted = false>
using NarrowShared = WarpShared<unsigned int, kSky, kSmemCov, kBack, kWeighted>;
template <bool kSky, bool kSmemCov, bool kBack = false, bool kWeighted = false>
using WideShared = WarpShared<unsigned long long, kSky, kSmemCov, kBack, kWeighted>;
// The shared memory of a kernel variant's warps, and the blocks per SM it
// fits. Prefiltering light cones integrate in the walk kernel, reading every
// lane's coverages (warp_blocked): their table stays in shared memory. The
// split path's cones and sky cones (whose integration reads only the lane's
// own) keep coverages in thread-local memory; the prefiltering walk of sky
// cones needs about 165 registers, so its packet pass takes 6 blocks per SM
// (8 would cap registers at 128 and spill).
template <bool kSky, bool kSplat>
constexpr bool smem_cov() { return kSplat && !kSky; }
template <bool kWide, bool kSky, bool kSplat, bool kBack = false, bool kInst = false>
using KernelShared = typename std::conditional<kWide, WideShared<kSky, smem_cov<kSky, kSplat>(), kBack, kInst>,
                                               NarrowShared<kSky, smem_cov<kSky, kSplat>(), kBack, kInst>>::type;
constexpr int resident_blocks_for(bool wide, bool sky, bool splat) {
  return (splat && !sky) ? (wide ? kFusedSoloBlocksPerSm : kFusedBlocksPerSm)
                         : (wide ? kSoloBlocksPerSm : (splat ? kSkySplatBlocksPerSm : kBlocksPerSm));
}
template <bool kWide, bool kSky, bool kSplat>
constexpr int resident_blocks() { return resident_blocks_for(kWide, kSky, kSplat); }
// Per SM (228 KB): 8 x 22.8 KB and 5 x 38.9 KB with thread-local coverages,
// 5 x 38.9 KB and 4 x 55.3 KB with shared ones, 1 KB reserved per block.
static_assert(8 * (kWarpsPerBlock * sizeof(KernelShared<false, false, false>) + 1024) <= 233472, "split packet pass");
static_assert(5 * (kWarpsPerBlock * sizeof(KernelShared<true, false, false>) + 1024) <= 233472, "split solo pass");
static_assert(8 * (kWarpsPerBlock * sizeof(KernelShared<false, true, false>) + 1024) <= 233472, "sky packet pass");
static_assert(5 * (kWarpsPerBlock * sizeof(KernelShared<true, true, false>) + 1024) <= 233472, "sky solo pass");
static_assert(5 * (kWarpsPerBlock * sizeof(KernelShared<false, false, true>) + 1024) <= 233472, "prefiltering packet pass");
static_assert(4 * (kWarpsPerBlock * sizeof(KernelShared<true, false, true>) + 1024) <= 233472, "prefiltering solo pass");
static_assert(6 * (kWarpsPerBlock * sizeof(KernelShared<false, true, true>) + 1024) <= 233472, "prefiltering sky packet pass");
static_assert(5 * (kWarpsPerBlock * sizeof(KernelShared<true, true, true>) + 1024) <= 233472, "prefiltering sky solo pass");
constexpr uint32_t kStatusAccOverflow = 32u;
static_assert(kConeFields * 32 >= 387, "the integration scratch fits in the cone table");

// A stack entry packed in one word: its kind in the top 2 bits (an
// object-hierarchy node, a triangle-hierarchy node, or a mesh's resolve
// marker), then a node's item count in 4 bits (0: interior), then its first
// item (leaf) or left child (interior) in 26 bits. Each lane keeps two bits
// per entry: whether its own walk needs the entry, and whether its cone
// passed the entry's box test, which is done when the parent is visited (the
// two children of a node are adjacent, so one 64-byte load serves both
// tests and the nearest-first choice).
constexpr uint32_t kRefIndexBits = 26;
constexpr uint32_t kRefIndexMask = (1u << kRefIndexBits) - 1u;
constexpr uint32_t kRefKindShift = 30;
__device__ __forceinline__ uint32_t node_ref(float4 a, float4 b, uint32_t kind) {
  return (kind << kRefKindShift) | ((__float_as_uint(b.w) & 15u) << kRefIndexBits) |
         (__float_as_uint(a.w) & kRefIndexMask);
}
__device__ __forceinline__ uint32_t ref_kind(uint32_t r) { return r >> kRefKindShift; }
__device__ __forceinline__ uint32_t ref_count(uint32_t r) { return (r >> kRefIndexBits) & 15u; }
__device__ __forceinline__ uint32_t ref_index(uint32_t r) { return r & kRefIndexMask; }

struct WarpStack {
  uint32_t r0 = 0, r1 = 0;  // entry i held by lane i % 32, register i / 32
  uint32_t need_lo = 0, need_hi = 0;
  uint32_t pass_lo = 0, pass_hi = 0;
  __device__ __forceinline__ void push(int i, uint32_t v, bool need, bool pass, int lane) {
    if ((i & 31) == lane) {
      if (i < 32) r0 = v; else r1 = v;
    }
    const uint32_t bit = 1u << (i & 31);
    if (i < 32) {
      need_lo = need ? (need_lo | bit) : (need_lo & ~bit);
      pass_lo = pass ? (pass_lo | bit) : (pass_lo & ~bit);
    } else {
      need_hi = need ? (need_hi | bit) : (need_hi & ~bit);
      pass_hi = pass ? (pass_hi | bit) : (pass_hi & ~bit);
    }
  }
  __device__ __forceinline__ uint32_t get(int i) const {
    return __shfl_sync(0xffffffffu, i < 32 ? r0 : r1, i & 31);
  }
  __device__ __forceinline__ bool need(int i) const {
    return ((i < 32 ? need_lo : need_hi) >> (i & 31)) & 1u;
  }
  __device__ __forceinline__ bool pass(int i) const {
    return ((i < 32 ? pass_lo : pass_hi) >> (i & 31)) & 1u;
  }
};

template <class WS>
struct LaneState {
  Cone cone;   // the cone in the space of the object being walked (the world's elsewhere)
  Cone world;  // instanced scenes: the cone in world space
  WS* ws;
  // The cone's coverages: bin b at cov[32 * b] in the warp's shared table
  // (&ws->cov[lane]), or at cov[b] in a thread-local array.
  float* cov;
  uint32_t full;
  uint32_t queued;  // both queues' lengths (queue_lens; the same in every lane)
  uint32_t cone_work;
  uint32_t cap;
  uint32_t status;
  uint32_t n_obj, n_blas, n_tris;
  uint32_t skip;     // the cone's own triangle slot, which it does not draw (kNoneU: none)
  bool skips;        // some lane of the warp has one (warp-uniform)
  bool independent;  // sky cones: meshes combine as independent occluders (else by the maximum)
  f3 horizon;        // sky cones: the horizon in the space of the object being walked (the world's elsewhere)
  f3 world_horizon;  // sky cones in instanced scenes: the horizon in world space
  // The cone's coverage of bin b.
  __device__ __forceinline__ float& cov_at(int b) { return cov[(WS::kSmemCov ? 32 : 1) * b]; }
};

__device__ __forceinline__ f3 node_lo(float4 a) { return mk(a.x, a.y, a.z); }

template <class WS>
__device__ __forceinline__ void store_cone(WS* ws, const Cone& c, int lane) {
  float* t = ws->cone + lane;
  const float f[kConeFields] = {c.apex.x, c.apex.y, c.apex.z, c.right.x, c.right.y, c.right.z, c.up.x, c.up.y,
                                c.up.z,   c.fwd.x,  c.fwd.y,  c.fwd.z,   c.u0,      c.v0,      c.u1,   c.v1,
                                c.far_offset};
#pragma unroll
  for (int k = 0; k < kConeFields; ++k) t[32 * k] = f[k];
}

// Sky cones: the lane's horizon beside its cone (the cull reads both).
template <class WS>
__device__ __forceinline__ void store_horizon(WS* ws, f3 h, int lane) {
  if constexpr (WS::kSky) {
    ws->horizon[lane] = h.x;
    ws->horizon[32 + lane] = h.y;
    ws->horizon[64 + lane] = h.z;
  }
}

template <class WS>
__device__ __forceinline__ Cone load_cone(const WS* ws, int owner) {
  const float* t = ws->cone + owner;
  Cone c;
  c.apex = mk(t[0], t[32], t[64]);
  c.right = mk(t[96], t[128], t[160]);
  c.up = mk(t[192], t[224], t[256]);
  c.fwd = mk(t[288], t[320], t[352]);
  c.u0 = t[384];
  c.v0 = t[416];
  c.u1 = t[448];
  c.v1 = t[480];
  c.far_offset = t[512];
  c.baxis = mk(0.f, 0.f, 0.f);
  c.bcos = c.bsin = 0.f;
  return c;
}

// The tests of cover_triangle (:594-616) for one (triangle, cone) pair: back
// face, the window-direction test, may_touch. A pair that passes is
// rasterized.
template <class WS>
__device__ __forceinline__ bool pair_survives(const DevScene& s, const WS* ws, int owner, uint32_t t) {
  const Cone c = load_cone(ws, owner);
  const f3 v0 = xyz(__ldg(&s.tris[3 * (size_t)t + 0]));
  const f3 v1 = xyz(__ldg(&s.tris[3 * (size_t)t + 1]));
  const f3 v2 = xyz(__ldg(&s.tris[3 * (size_t)t + 2]));
  const f3 n = cross(v1 - v0, v2 - v0);
  if (dot(n, c.apex - v0) <= 0.0f) return false;  // faces away (:600)
  if (dot(n, direction(c, 0.f, 0.f)) >= 0.f && dot(n, direction(c, 1.f, 0.f)) >= 0.f &&
      dot(n, direction(c, 0.f, 1.f)) >= 0.f && dot(n, direction(c, 1.f, 1.f)) >= 0.f)
    return false;  // every window direction leaves its plane (:601-606)
  if constexpr (WS::kSky)
    return may_touch<true>(c, v0, v1, v2, mk(ws->horizon[owner], ws->horizon[32 + owner], ws->horizon[64 + owner]));
  else
    return may_touch(c, v0, v1, v2);
}

template <class WS>
__device__ __forceinline__ void load_pair(const DevScene& s, const WS* ws, uint32_t e, int& owner, Cone& c,
                                          f3& v0, f3& v1, f3& v2) {
  owner = (int)(e >> kQueueOwnerShift);
  const uint32_t t = e & ((1u << kQueueOwnerShift) - 1u);
  c = load_cone(ws, owner);
  v0 = xyz(__ldg(&s.tris[3 * (size_t)t + 0]));
  v1 = xyz(__ldg(&s.tris[3 * (size_t)t + 1]));
  v2 = xyz(__ldg(&s.tris[3 * (size_t)t + 2]));
}

// The weight a (triangle, cone) pair is drawn with: the current object's
// (1 - clear for a blended one), or for a transmissive object one less what
// passes through the triangle at the cone's central direction, Schlick's
// Fresnel with F0 0.04, twice for a volume (cover_triangle, :608-614). The
// fifth power is taken by multiplications.
template <class WS>
__device__ __forceinline__ float pair_weight(const WS* ws, const Cone& c, f3 v0, f3 v1, f3 v2) {
  const float transmit = ws->object_transmit;
  if (!(transmit > 0.0f)) return ws->object_weight;
  const f3 n = cross(v1 - v0, v2 - v0);
  const float cos_t = fabsf(dot(normalize(n), normalize(direction(c, 0.5f, 0.5f))));
  const float x = 1.0f - cos_t;
  const float x2 = x * x;
  const float f = 0.04f + 0.96f * (x2 * x2 * x);
  float passes = transmit * (1.0f - f);
  if (ws->object_volume) passes *= 1.0f - f;
  return 1.0f - passes;
}

// Entering placed object X's triangles: its weight and transmission from
// its transform's `clear` (row 3's z; add_mesh_coverage_if, :733-741); and
// leaving it. The caller syncs the warp before the values are read.
template <class WS>
__device__ __forceinline__ void enter_object(WS* ws, const float4* __restrict__ X, int lane) {
  if constexpr (WS::kWeighted) {
    const float clear = __ldg(&X[3]).z;
    if (lane == 0) {
      float transmit = fmaxf(-clear, 0.0f);
      uint32_t volume = 0u;
      if (clear <= -2.0f) {  // a volume: two surfaces
        transmit = -2.0f - clear;
        volume = 1u;
      }
      ws->object_weight = 1.0f - fmaxf(clear, 0.0f);
      ws->object_transmit = transmit;
      ws->object_volume = volume;
    }
  }
}
template <class WS>
__device__ __forceinline__ void leave_object(WS* ws, int lane) {
  if constexpr (WS::kWeighted) {
    if (lane == 0) {
      ws->object_weight = 1.0f;
      ws->object_transmit = 0.0f;
      ws->object_volume = 0u;
    }
  }
}

template <class WS, class Acc>
__device__ __forceinline__ void note_span(WS* ws, int owner, const Acc& acc) {
  if (acc.span_lo < acc.span_hi) {
    atomicMin(&ws->span_lo[owner], acc.span_lo);
    atomicMax(&ws->span_hi[owner], acc.span_hi);
  }
}

// The general path for general-queue entries first .. first+n (n <= 32),
// one per lane.
template <class WS>
__device__ __noinline__ void raster_general(const DevScene& s, WS* ws, uint32_t first, uint32_t n, int lane) {
  if ((uint32_t)lane < n) {
    int owner;
    Cone c;
    f3 v0, v1, v2;
    load_pair(s, ws, ws->general[first + lane], owner, c, v0, v1, v2);
    LaneAcc<typename WS::Cell> acc{ws->acc + owner, 68u, 0u, &ws->overflow[0], 1u << owner};
    float weight = 1.0f;
    if constexpr (WS::kWeighted) weight = pair_weight(ws, c, v0, v1, v2);
    rasterize_general<decltype(acc), WS::kWeighted>(c, acc, v0, v1, v2, crosses_far(c, v0, v1, v2), weight);
    note_span(ws, owner, acc);
  }
  __syncwarp();
}

// Rasterizes queue entries first .. first+n (n <= 32), one per lane, each
// into its cone's accumulator by the common case; pairs that need the
// general path join the general queue, which is run whenever 32 wait.
// Returns the general queue's new length (below 32).
template <class WS>
__device__ __noinline__ uint32_t raster_queue(const DevScene& s, WS* ws, uint32_t first, uint32_t n,
                                              uint32_t general, int lane) {
  bool defer = false;
  uint32_t e = 0;
  if ((uint32_t)lane < n) {
    e = ws->queue[first + lane];
    int owner;
    Cone c;
    f3 v0, v1, v2;
    load_pair(s, ws, e, owner, c, v0, v1, v2);
    LaneAcc<typename WS::Cell> acc{ws->acc + owner, 68u, 0u, &ws->overflow[0], 1u << owner};
    float weight = 1.0f;
    if constexpr (WS::kWeighted) weight = pair_weight(ws, c, v0, v1, v2);
    defer = !rasterize_fast(c, acc, v0, v1, v2, weight);
    note_span(ws, owner, acc);
  }
  const uint32_t m = __ballot_sync(0xffffffffu, defer);
  if (defer) ws->general[general + __popc(m & ((1u << lane) - 1u))] = e;
  general += __popc(m);
  __syncwarp();
  if (general >= 32) {
    general -= 32;
    raster_general(s, ws, general, 32, lane);
  }
  return general;
}

// Triangles t0 .. t0+nt, each tested against the cones of the lanes in
// `owners`: the pairs, triangle-major (consecutive lanes read the same
// triangle), are dealt out over the warp for the cull tests; the survivors
// join the warp's queue, and every 32 queued pairs are rasterized by the
// whole warp at once, so lanes whose pair was culled do not sit idle while
// the others rasterize. `queues` and the result are both queues' lengths.
// `skip` is the lane's cone's own triangle slot (kNoneU: none), which it
// does not draw; `skips` (warp-uniform) says some lane has one.
template <class WS>
__device__ __noinline__ uint32_t cover_leaf(const DevScene& s, WS* ws, uint32_t owners, uint32_t t0,
                                            uint32_t nt, uint32_t queues, int lane, uint32_t skip, bool skips) {
  uint32_t queued = fast_len(queues), general = general_len(queues);
  const uint32_t n_owners = __popc(owners);
  const uint32_t n_pairs = n_owners * nt;
  // pair / n_owners as a multiply and a shift: pairs stay below 32 x 15 and
  // there are 1 to 32 owners, so (pair * magic) >> 16 with magic =
  // 65536 / n_owners + 1 exceeds the quotient by under 480 / 65536, less than
  // the 1 / n_owners a quotient's fraction stays below 1 by.
  const uint32_t magic = 65536u / n_owners + 1u;
  for (uint32_t base = 0; base < n_pairs; base += 32) {
    const uint32_t pair = base + lane;
    bool pass = false;
    uint32_t entry = 0;
    int owner = 0;
    uint32_t t = kNoneU;
    if (pair < n_pairs) {
      const uint32_t k = (pair * magic) >> 16;
      const uint32_t r = pair - k * n_owners;
      owner = (int)__fns(owners, 0, r + 1);
      t = t0 + k;
      pass = pair_survives(s, ws, owner, t);
      entry = ((uint32_t)owner << kQueueOwnerShift) | t;
    }
    // The owner's own triangle is not drawn (cover_triangle's cover_skip, :595).
    if constexpr (WS::kBack) {
      if (skips && __shfl_sync(0xffffffffu, skip, owner) == t) pass = false;
    }
    const uint32_t m = __ballot_sync(0xffffffffu, pass);
    if (pass) ws->queue[queued + __popc(m & ((1u << lane) - 1u))] = entry;
    queued += __popc(m);
    __syncwarp();
    if (queued >= 32) {
      queued -= 32;
      general = raster_queue(s, ws, queued, 32, general, lane);
    }
  }
  return queue_lens(queued, general);
}

// The mesh's coverage for the lane's own cone: running sum over the touched
// cells (exact), snapped to whole within 1e-5, combined into the cone's bins
// by max (:809-828), or for sky cones as independent occluders
// (1 - (1 - before)(1 - covered), :819-821); then the cells are cleared for
// the next mesh.
template <class WS>
__device__ __forceinline__ void resolve_mesh(const DevScene& s, LaneState<WS>& st, int lane, bool splat = false) {
  WS* ws = st.ws;
  // The mesh's last pairs: the common case, then the general path.
  uint32_t general = general_len(st.queued);
  if (fast_len(st.queued)) general = raster_queue(s, ws, 0, fast_len(st.queued), general, lane);
  if (general) raster_general(s, ws, 0, general, lane);
  st.queued = 0;
  const uint32_t lo = ws->span_lo[lane];
  const uint32_t end = min(ws->span_hi[lane], (uint32_t)kBins);
  // 32-bit cells: a cone whose adds overflowed in this mesh is walked again
  // with 64-bit cells (its result here is discarded).
  if (sizeof(typename WS::Cell) == 4) {
    if ((ws->overflow[0] >> lane) & 1u) st.status |= kStatusAccOverflow;
    __syncwarp();
    if (lane == 0) ws->overflow[0] = 0u;
  }
  long long running = 0;
  for (uint32_t b = lo; b < end; ++b) {
    typename WS::Cell* cell = &ws->acc[32 * b + lane];
    if (sizeof(typename WS::Cell) == 4) running += (long long)(int)*cell;
    else running += (long long)*cell;
    *cell = 0;
    float covered = fabsf(__ll2float_rn(running) * kFixUnit);
    // An object-level splat is combined without the whole-bin snap (:1137).
    if (splat) covered = fminf(covered, 1.0f);
    else if (covered >= 1.0f - 1e-5f) covered = 1.0f;
    if (covered > 1e-6f) {
      const float before = st.cov_at(b);
      float after;
      if constexpr (WS::kSky) {
        after = st.independent ? 1.0f - (1.0f - before) * (1.0f - fminf(covered, 1.0f))
                               : fmaxf(before, fminf(covered, 1.0f));
      } else {
        after = fmaxf(before, fminf(covered, 1.0f));
      }
      st.cov_at(b) = after;
      if (before < 1.0f && after >= 1.0f) st.full++;
    }
  }
  ws->span_lo[lane] = 68u;
  ws->span_hi[lane] = 0u;
  __syncwarp();
}

// Stack entry kinds for the walk of both hierarchy levels in one loop.
constexpr uint32_t kObjNode = 0;   // an object-hierarchy node
constexpr uint32_t kTriNode = 1;   // a node of the current mesh's triangle hierarchy
constexpr uint32_t kResolve = 2;   // the current mesh is done: resolve its coverage (index 1: and return to world space)
constexpr uint32_t kObjRoot = 3;   // instanced scenes: the root of object `index`'s triangle hierarchy

// add_mesh_coverage_if (:713-829) for hierarchy levels 0 and 1: every
// triangle of mesh m for the lanes with `on`, in leaf-sized groups, then the
// mesh's resolve.
template <bool kCount, bool kInst, class WS>
__device__ __forceinline__ void add_mesh_flat(const DevScene& s, LaneState<WS>& st, bool on, uint32_t m, int lane) {
  const uint32_t owners = __ballot_sync(0xffffffffu, on);
  if (!owners) return;
  const uint4 range = __ldg(&s.meshes[m]);
  const bool placed = kInst && range.w != kNoneU;
  if (placed) {
    st.cone = cone_to_object(st.world, s.xforms + 4 * (size_t)range.w);  // cone_to_object (:623-638)
    store_cone(st.ws, st.cone, lane);
    enter_object(st.ws, s.xforms + 4 * (size_t)range.w, lane);
    if constexpr (WS::kSky) {
      st.horizon = rotate_to_object(st.world_horizon, s.xforms + 4 * (size_t)range.w);
      store_horizon(st.ws, st.horizon, lane);
    }
    __syncwarp();
  }
  if (kCount && on) st.n_tris += range.y;
  for (uint32_t t = range.x; t < range.x + range.y; t += 8)
    st.queued = cover_leaf(s, st.ws, owners, t, min(8u, range.x + range.y - t), st.queued, lane, st.skip,
                           st.skips);
  resolve_mesh(s, st, lane);
  if (placed) {
    st.cone = st.world;
    store_cone(st.ws, st.cone, lane);
    leave_object(st.ws, lane);
    if constexpr (WS::kSky) {
      st.horizon = st.world_horizon;
      store_horizon(st.ws, st.horizon, lane);
    }
    __syncwarp();
  }
}

// The cone walk (scene_coverage_if, :1160-1227, with add_mesh_coverage_if,
// :713-829, for each mesh it reaches). Hierarchy level 2 walks both levels in
// one loop: an object leaf that a lane descends into pushes, for each of its
// meshes (first mesh on top), a resolve marker under the mesh's triangle
// hierarchy root, so each mesh is walked and then resolved in the reference's
// order. Object nodes are visited nearest child first along the bounding
// cone's axis while some bin is open; triangle-hierarchy nodes right child
// first (:783-787) with no full check, as in the reference; every popped node
// a lane needs counts toward its walk cap, though its box was tested when its
// parent was visited. Levels 0 and 1 keep the reference's loops over meshes
// and triangles; they are compiled only into the kernels of kFlat, which
// launches at those levels take, so the level-2 walk's code stays small.
template <bool kCount, bool kInst, bool kFlat, class WS>
__device__ __forceinline__ void scene_walk(const DevScene& s, uint32_t hierarchy, LaneState<WS>& st, bool traced,
                                           int lane) {
  const Cone& c = st.cone;
  if constexpr (kFlat) {
    if (hierarchy == 0) {
      for (uint32_t m = 0; m < s.nmeshes; ++m)
        add_mesh_flat<kCount, kInst, WS>(s, st, traced && st.full < (uint32_t)kBins, m, lane);
      return;
    }
  }
  WarpStack stk;
  const float4 ra = __ldg(&s.nodes[0]);
  const float4 rb = __ldg(&s.nodes[1]);
  const bool root_pass = traced && may_touch_box<WS::kSky, false>(c, node_lo(ra), node_lo(rb), st.horizon);
  stk.push(0, node_ref(ra, rb, kObjNode), traced, root_pass, lane);
  int sp = 1;
  while (sp > 0) {
    --sp;
    uint32_t ref = stk.get(sp);
    uint32_t kind = ref_kind(ref);
    if (kind == kResolve) {
      resolve_mesh(s, st, lane);
      if (kInst && ref_index(ref) == 1) {  // back to world space
        st.cone = st.world;
        store_cone(st.ws, st.cone, lane);
        leave_object(st.ws, lane);
        if constexpr (WS::kSky) {
          st.horizon = st.world_horizon;
          store_horizon(st.ws, st.horizon, lane);
        }
        __syncwarp();
      }
      continue;
    }
    if (kInst && kind == kObjRoot) {
      // Entering a placed object: the cone in its space (cone_to_object,
      // :623-638), then its triangle hierarchy's root.
      const uint4 range = __ldg(&s.meshes[ref_index(ref)]);
      st.cone = cone_to_object(st.world, s.xforms + 4 * (size_t)range.w);
      store_cone(st.ws, st.cone, lane);
      enter_object(st.ws, s.xforms + 4 * (size_t)range.w, lane);
      if constexpr (WS::kSky) {
        // The horizon turns with the cone (:634).
        st.horizon = rotate_to_object(st.world_horizon, s.xforms + 4 * (size_t)range.w);
        store_horizon(st.ws, st.horizon, lane);
      }
      __syncwarp();
      ref = node_ref(__ldg(&s.blas[2 * (size_t)range.z + 0]), __ldg(&s.blas[2 * (size_t)range.z + 1]), kTriNode);
      kind = kTriNode;
    }
    const bool is_obj = kind == kObjNode;
    const bool mine = stk.need(sp) && st.cone_work < st.cap && (!is_obj || st.full < (uint32_t)kBins);
    if (mine) st.cone_work++;
    if (kCount && mine) {
      if (is_obj) st.n_obj++; else st.n_blas++;
    }
    const bool descend = mine && stk.pass(sp);
    const uint32_t owners = __ballot_sync(0xffffffffu, descend);
    if (!owners) continue;
    const uint32_t ia = ref_index(ref), ib = ref_count(ref);
    if (ib > 0 && !is_obj) {
      // A triangle-hierarchy leaf: its triangles against every descending cone.
      if (descend) {
        st.cone_work += ib;
        if (kCount) st.n_tris += ib;
      }
      st.queued = cover_leaf(s, st.ws, owners, ia, ib, st.queued, lane, st.skip, st.skips);
    } else if (ib > 0) {
      // An object leaf: its meshes.
      if constexpr (kFlat) {
        if (hierarchy == 1) {
          for (uint32_t k = ia; k < ia + ib; ++k)
            add_mesh_flat<kCount, kInst, WS>(s, st, descend, __ldg(&s.items[k]), lane);
          continue;
        }
      }
      for (int k = (int)(ia + ib) - 1; k >= (int)ia; --k) {
        const uint4 range = __ldg(&s.meshes[__ldg(&s.items[k])]);
        if (range.z == kNoneU) continue;  // no triangles: nothing to draw or resolve
        if (sp + 2 > kStack) {
          if (descend) st.status |= 2u;
          continue;
        }
        const float4 ma = __ldg(&s.blas[2 * (size_t)range.z + 0]);
        const float4 mb = __ldg(&s.blas[2 * (size_t)range.z + 1]);
        const uint32_t m = __ldg(&s.items[k]);
        if (kInst && range.w != kNoneU) {
          // A placed object: its root's box in its own space; the entry names
          // the object, whose cone is set up when the entry is popped.
          const Cone oc = cone_to_object(st.world, s.xforms + 4 * (size_t)range.w);
          f3 oh = st.horizon;
          if constexpr (WS::kSky) oh = rotate_to_object(st.world_horizon, s.xforms + 4 * (size_t)range.w);
          const bool mesh_pass = descend && may_touch_box<WS::kSky>(oc, node_lo(ma), node_lo(mb), oh);
          stk.push(sp, (kResolve << kRefKindShift) | 1u, false, false, lane);
          stk.push(sp + 1, (kObjRoot << kRefKindShift) | m, descend, mesh_pass, lane);
        } else {
          const bool mesh_pass = descend && may_touch_box<WS::kSky, false>(c, node_lo(ma), node_lo(mb), st.horizon);
          stk.push(sp, kResolve << kRefKindShift, false, false, lane);
          stk.push(sp + 1, node_ref(ma, mb, kTriNode), descend, mesh_pass, lane);
        }
        sp += 2;
      }
    } else {
      // An interior node: both children's boxes tested now.
      const float4* base = (is_obj ? s.nodes : s.blas) + 2 * (size_t)ia;
      const float4 la = __ldg(base + 0), lb = __ldg(base + 1), xa = __ldg(base + 2), xb = __ldg(base + 3);
      bool pl = false, pr = false;
      if (descend) {
#pragma unroll 1
        for (int ch = 0; ch < 2; ++ch) {
          const bool t = may_touch_box<WS::kSky>(c, node_lo(ch ? xa : la), node_lo(ch ? xb : lb), st.horizon);
          if (ch) pr = t; else pl = t;
        }
      }
      bool swap = false;  // left child popped first (object level: when it is the nearer)
      // Nearest child first where meshes combine by the maximum; sky cones
      // combining as independent occluders keep the left child first, as
      // their products would round differently in another order (:1188-1207).
      bool nearest = is_obj;
      if constexpr (WS::kSky) nearest = nearest && !st.independent;
      if (nearest) {
        const float da = dot(c.baxis, (node_lo(la) + node_lo(lb)) * 0.5f - c.apex);
        const float db = dot(c.baxis, (node_lo(xa) + node_lo(xb)) * 0.5f - c.apex);
        const bool pref = db < da;  // this lane's own order: right child nearer
        // The packet takes the order most of its descending lanes prefer;
        // the others are flagged (their walk is redone alone if its order
        // could matter).
        swap = 2u * __popc(__ballot_sync(0xffffffffu, descend && pref)) > __popc(owners);
        if (descend && pref != swap) st.status |= 4u;
      } else if (!is_obj) {
        swap = true;  // triangle hierarchies pop the right child first (:783-787)
      }
      if (sp + 2 > kStack) {
        if (descend) st.status |= 2u;
        continue;
      }
      const uint32_t rl = node_ref(la, lb, kind), rr = node_ref(xa, xb, kind);
      // The child popped second below the one popped first.
      stk.push(sp, swap ? rl : rr, descend, swap ? pl : pr, lane);
      stk.push(sp + 1, swap ? rr : rl, descend, swap ? pr : pl, lane);
      sp += 2;
    }
  }
}

// The walk of prefiltering cones (hierarchy level 2): scene_coverage_if
// (:1160-1227) with splat_object_node (:1096-1150) and add_mesh_coverage_if
// (:750-790) with node_cone_test (:519-574). Each entry is a node index, and
// a node is tested when popped, as the reference tests it: a node small in
// the cone is splatted instead of descended into (a triangle-hierarchy node
// into its mesh's accumulator, an object node into the mask as one more
// mesh), and the walk cap counts the popped nodes a lane needs.
constexpr uint32_t kSplatIndexMask = (1u << kRefKindShift) - 1u;

template <bool kCount, bool kInst, class WS>
__device__ __forceinline__ void scene_walk_splat(const DevScene& s, float prefilter, LaneState<WS>& st, bool traced,
                                                 int lane) {
  WS* ws = st.ws;
  WarpStack stk;
  stk.push(0, (kObjNode << kRefKindShift) | 0u, traced, true, lane);
  int sp = 1;
  while (sp > 0) {
    --sp;
    const uint32_t entry = stk.get(sp);
    uint32_t kind = entry >> kRefKindShift;
    uint32_t idx = entry & kSplatIndexMask;
    if (kind == kResolve) {
      resolve_mesh(s, st, lane);
      if (kInst && idx == 1) {  // back to world space
        st.cone = st.world;
        store_cone(ws, st.cone, lane);
        leave_object(ws, lane);
        if constexpr (WS::kSky) {
          st.horizon = st.world_horizon;
          store_horizon(ws, st.horizon, lane);
        }
        __syncwarp();
      }
      continue;
    }
    if (kInst && kind == kObjRoot) {
      // Entering a placed object: the cone (and horizon) in its space, then
      // its triangle hierarchy's root, tested as any popped node.
      const uint4 range = __ldg(&s.meshes[idx]);
      st.cone = cone_to_object(st.world, s.xforms + 4 * (size_t)range.w);
      store_cone(ws, st.cone, lane);
      enter_object(ws, s.xforms + 4 * (size_t)range.w, lane);
      if constexpr (WS::kSky) {
        st.horizon = rotate_to_object(st.world_horizon, s.xforms + 4 * (size_t)range.w);
        store_horizon(ws, st.horizon, lane);
      }
      __syncwarp();
      kind = kTriNode;
      idx = range.z;
    }
    const bool is_obj = kind == kObjNode;
    const bool mine = stk.need(sp) && st.cone_work < st.cap && (!is_obj || st.full < (uint32_t)kBins);
    if (mine) st.cone_work++;
    if (kCount && mine) {
      if (is_obj) st.n_obj++; else st.n_blas++;
    }
    if (!__any_sync(0xffffffffu, mine)) continue;
    const float4* rec = (is_obj ? s.nodes : s.blas) + 2 * (size_t)idx;
    const float4 ra = __ldg(rec), rb = __ldg(rec + 1);
    const f3 lo = node_lo(ra), hi = node_lo(rb);
    const uint32_t ref = node_ref(ra, rb, kind);
    const uint32_t ia = ref_index(ref), ib = ref_count(ref);
    bool descend = false;
    if (is_obj) {
      bool splatted = false;
      if (mine && may_touch_box<WS::kSky>(st.cone, lo, hi, st.horizon)) {
        const float* cov = s.obj_cov ? s.obj_cov + kCoverageSamples * (size_t)idx : nullptr;
        if (cov && __ldg(&cov[13]) == 0.0f) {
          LaneAcc<typename WS::Cell> acc{ws->acc + lane, 68u, 0u, &ws->overflow[0], 1u << lane};
          splatted = splat_object_node(st.cone, acc, cov, lo, hi, prefilter);
          if (acc.span_lo < acc.span_hi) {
            ws->span_lo[lane] = min(ws->span_lo[lane], acc.span_lo);
            ws->span_hi[lane] = max(ws->span_hi[lane], acc.span_hi);
          }
        }
        descend = !splatted;
      }
      // Splats are combined into the mask at once, as one more mesh each.
      if (__any_sync(0xffffffffu, splatted)) resolve_mesh(s, st, lane, true);
    } else if (mine) {
      LaneAcc<typename WS::Cell> acc{ws->acc + lane, 68u, 0u, &ws->overflow[0], 1u << lane};
      const int test = node_cone_test<WS::kSky>(st.cone, st.horizon, acc, s.blas_cov + kCoverageSamples * (size_t)idx,
                                                lo, hi, prefilter);
      if (acc.span_lo < acc.span_hi) {
        ws->span_lo[lane] = min(ws->span_lo[lane], acc.span_lo);
        ws->span_hi[lane] = max(ws->span_hi[lane], acc.span_hi);
      }
      descend = test == 3;
    }
    const uint32_t owners = __ballot_sync(0xffffffffu, descend);
    if (!owners) continue;
    if (is_obj && ib > 0) {
      // An object leaf: its meshes, first on top, each under its resolve marker.
      for (int k = (int)(ia + ib) - 1; k >= (int)ia; --k) {
        const uint32_t m = __ldg(&s.items[k]);
        const uint4 range = __ldg(&s.meshes[m]);
        if (range.z == kNoneU) continue;  // no triangles: nothing to draw or resolve
        if (sp + 2 > kStack) {
          if (descend) st.status |= 2u;
          continue;
        }
        const bool placed = kInst && range.w != kNoneU;
        stk.push(sp, (kResolve << kRefKindShift) | (placed ? 1u : 0u), false, false, lane);
        stk.push(sp + 1, placed ? ((kObjRoot << kRefKindShift) | m) : ((kTriNode << kRefKindShift) | range.z), descend,
                 true, lane);
        sp += 2;
      }
    } else if (!is_obj && ib > 0) {
      // A triangle-hierarchy leaf: its triangles against every descending cone.
      if (descend) {
        st.cone_work += ib;
        if (kCount) st.n_tris += ib;
      }
      st.queued = cover_leaf(s, ws, owners, ia, ib, st.queued, lane, st.skip, st.skips);
    } else {
      if (sp + 2 > kStack) {
        if (descend) st.status |= 2u;
        continue;
      }
      bool swap = !is_obj;  // triangle hierarchies pop the right child first (:783-787)
      bool nearest = is_obj;
      if constexpr (WS::kSky) nearest = nearest && !st.independent;
      if (nearest) {
        const float4* base = s.nodes + 2 * (size_t)ia;
        const float4 la = __ldg(base + 0), lb = __ldg(base + 1), xa = __ldg(base + 2), xb = __ldg(base + 3);
        const float da = dot(st.cone.baxis, (node_lo(la) + node_lo(lb)) * 0.5f - st.cone.apex);
        const float db = dot(st.cone.baxis, (node_lo(xa) + node_lo(xb)) * 0.5f - st.cone.apex);
        const bool pref = db < da;
        swap = 2u * __popc(__ballot_sync(0xffffffffu, descend && pref)) > __popc(owners);  // the majority's order
        if (descend && pref != swap) st.status |= 4u;
      }
      const uint32_t l = (kind << kRefKindShift) | ia, r = (kind << kRefKindShift) | (ia + 1u);
      stk.push(sp, swap ? l : r, descend, true, lane);
      stk.push(sp + 1, swap ? r : l, descend, true, lane);
      sp += 2;
    }
  }
}

__device__ __forceinline__ f3 shfl3(f3 v, int src) {
  return mk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src), __shfl_sync(0xffffffffu, v.z, src));
}

// The blocked light of lane j's cone, Σ coverage × bin weight (cone_visible,
// :1244-1272), computed by the whole warp. With the window above the
// horizon every bin weight is Lambert's formula over its quad
// (bin_weight, :1232-1242); the 64 quads share 81 corner directions and 144
// edges, so the warp normalizes each corner once and integrates each edge
// once (a quad's edges are its neighbours' reversed, exact negatives in
// IEEE arithmetic) and each lane combines two bins. A window crossing the
// horizon clips each bin on its own (clipped_bin_weight, :1331-1369).
// `cov_j` is lane j's coverage column (bin b at cov_j[32 * b]); `scratch`
// holds 387 floats. Every lane returns the sum.
static __device__ __noinline__ float warp_blocked(const Cone& mine, f3 my_normal, bool my_all_above, const float* cov_j,
                                           float* scratch, int j, int lane) {
  Cone c;
  c.fwd = shfl3(mine.fwd, j);
  c.right = shfl3(mine.right, j);
  c.up = shfl3(mine.up, j);
  c.u0 = __shfl_sync(0xffffffffu, mine.u0, j);
  c.v0 = __shfl_sync(0xffffffffu, mine.v0, j);
  c.u1 = __shfl_sync(0xffffffffu, mine.u1, j);
  c.v1 = __shfl_sync(0xffffffffu, mine.v1, j);
  const f3 n = shfl3(my_normal, j);
  const bool all_above = __shfl_sync(0xffffffffu, my_all_above, j);
  float sum = 0.0f;
  if (all_above) {
    const float g = float(kGrid);
    float* corner = scratch;       // 81 unit directions, point (col, row) at 3 * (row * 9 + col)
    float* edge = scratch + 243;   // 72 row edges (col, row)->(col+1, row), then 72 column edges (col, row)->(col, row+1)
    for (int p = lane; p < 81; p += 32) {
      const f3 u = normalize(direction(c, float(p % 9) / g, float(p / 9) / g));
      corner[3 * p] = u.x;
      corner[3 * p + 1] = u.y;
      corner[3 * p + 2] = u.z;
    }
    __syncwarp();
    for (int e = lane; e < 144; e += 32) {
      int a, b;
      if (e < 72) {
        a = (e / 8) * 9 + e % 8;
        b = a + 1;
      } else {
        a = ((e - 72) / 9) * 9 + (e - 72) % 9;
        b = a + 9;
      }
      edge[e] = lambert_edge_unit(n, mk(corner[3 * a], corner[3 * a + 1], corner[3 * a + 2]),
                                  mk(corner[3 * b], corner[3 * b + 1], corner[3 * b + 2]));
    }
    __syncwarp();
    for (int b = lane; b < kBins; b += 32) {
      const float cv = cov_j[32 * b];
      if (cv > 0.0f) {
        const int col = b % kGrid, row = b / kGrid;
        const float e01 = edge[row * 8 + col];                 // d0 -> d1
        const float e12 = edge[72 + row * 9 + col + 1];        // d1 -> d2
        const float e23 = -edge[(row + 1) * 8 + col];          // d2 -> d3
        const float e30 = -edge[72 + row * 9 + col];           // d3 -> d0
        sum += cv * fabsf(0.5f * (e01 + e12 + e23 + e30));
      }
    }
    __syncwarp();
  } else {
    for (int b = lane; b < kBins; b += 32) {
      const float cv = cov_j[32 * b];
      if (cv > 0.0f) sum += cv * clipped_bin_weight(c, n, b);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  return sum;
}

// The light a light cone's mask lets through (cone_irradiance_rect,
// :1286-1321: rect lights' Lambert bin weights, one cone at a time across the
// warp; sphere_open_share, :957-972), times the spot factor, and the lighting
// cache's ratio (vc_bake :3453-3510, static light). Warp-collective: every
// lane calls it. `cov` is the warp's coverage table (bin b of lane j at
// cov[32 b + j]); `scratch` holds 387 floats the warp may overwrite.
__device__ __forceinline__ void light_integral(const Cone& cone, f3 point, f3 normal, const DevLight& L, float spot,
                                               bool traced, const LightConeInfo& info, bool last_empty,
                                               bool last_full, const float* cov, float* scratch, int lane,
                                               float& value_out, float& ratio_out) {
  const float* mine = cov + lane;
  const bool rect_traced = traced && !is_sphere(L);
  bool all_above = true;
  float total = 0.0f;
  if (rect_traced) total = window_weight(cone, normal, &all_above);
  float blocked = 0.0f;
  uint32_t todo = __ballot_sync(0xffffffffu, rect_traced && !last_empty);
  while (todo) {
    const int j = __ffs(todo) - 1;
    todo &= todo - 1;
    const float b = warp_blocked(cone, normal, all_above, cov + j, scratch, j, lane);
    if (lane == j) blocked = b;
  }
  float value = 0.0f;
  if (traced) {
    if (is_sphere(L)) {
      // sphere_open_share (:957-972)
      float total_w = 0.0f, open_w = 0.0f;
      const float g = float(kGrid);
#pragma unroll 1
      for (int b = 0; b < kBins; ++b) {
        const float mfrac = info.wide_clipped ? 1.0f : c_disk[b];
        if (mfrac <= 0.0f) continue;
        f3 d = direction(cone, (float(b % kGrid) + 0.5f) / g, (float(b / kGrid) + 0.5f) / g);
        float l2 = dot(d, d);
        float w = mfrac * fmaxf(dot(normal, d), 0.0f) / (l2 * l2);
        total_w += w;
        open_w += w * (1.0f - mine[32 * b]);
      }
      const float share = total_w <= 0.0f ? 1.0f : open_w / total_w;
      value = sphere_unshadowed(point, normal, L) * share;
    } else {
      // cone_visible (:1244-1272) and wide_visible (:1070-1073)
      float visible = fmaxf(total - blocked, 0.0f);
      if (info.wide_clipped) visible = (total > 1e-9f ? visible / total : 1.0f) * rect_open(point, normal, L);
      value = visible;
    }
  }
  value *= spot;
  const float open = unshadowed(point, normal, L);
  float ratio = open > 0.0f ? clampf(value / open, 0.0f, 1.0f) : 1.0f;
  if (open > 0.0f && last_empty) ratio = 1.0f;
  if (open > 0.0f && last_full) ratio = 0.0f;
  value_out = value;
  ratio_out = ratio;
}

// The job of a batch that holds `key` (a packet or a cone number): the last
// job whose start is at most `key`. Warp-uniform.
__device__ __forceinline__ uint32_t find_job(const JobGpu* __restrict__ jobs, uint32_t njobs, uint64_t key,
                                             bool by_cone) {
  uint32_t lo = 0, hi = njobs;  // jobs[lo].start <= key < jobs[hi].start
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    const uint64_t start = by_cone ? __ldg(&jobs[mid].cone_start) : __ldg(&jobs[mid].packet_start);
    if (start <= key) lo = mid; else hi = mid;
  }
  return lo;
}

// kBatch: the cones of every job of a batch (BatchLaunch); each packet's job
// is looked up in the job table, and the redo list holds batch cone numbers.
// kInst: the scene's objects place shared geometry with transforms.
// kWide: 64-bit accumulator cells (the solo pass); else 32-bit ones (the
// packet pass), whose overflowed cones the solo pass walks again.
// kSky: sky cones, the six cube faces around each receiver in place of its
// lights (cone c = face * npoints + point).
// kSplat: prefiltering cones (q.prefilter bins), walking hierarchy level 2.
// kBack: cones may skip their receiver's own triangle (CC_BACK_FACING; the
// split path's plain cones of scenes without instancing).
// kFlat: the launch's cones may walk hierarchy levels 0 or 1 (else level 2).
template <bool kCount, bool kBatch, bool kInst, bool kWide, bool kSky, bool kSplat, bool kBack = false,
          bool kFlat = false>
// The blocks the shared memory fits per SM; saying so bounds the registers
// per thread the allocator may use without lowering occupancy.
__global__ void __launch_bounds__(kWarpsPerBlock * 32, resident_blocks<kWide, kSky, kSplat>())
    visibility_kernel(DevScene s_plain, DevQuery q_plain, DevOut o, BatchLaunch batch,
                      const uint32_t* __restrict__ list, const uint32_t* __restrict__ list_count, uint32_t pw) {
  using WS = KernelShared<kWide, kSky, kSplat, kBack, kInst>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  WS* ws = reinterpret_cast<WS*>(smem_raw) + wib;
  float cov_local[WS::kSmemCov ? 1 : kBins];  // the lane's cone's coverages, unless the warp's table holds them
  // The per-packet loops over the 64 bins stay rolled: unrolled, they are
  // a tenth of the kernel's code, which competes for the instruction caches
  // with the walk.
#pragma unroll 1
  for (int k = 0; k < kBins; ++k) ws->acc[32 * k + lane] = 0;
  if (lane == 0) ws->overflow[0] = 0u;
  leave_object(ws, lane);  // the world's weight until a placed object is entered
  ws->span_lo[lane] = 68u;
  ws->span_hi[lane] = 0u;

  // The split path (exact light cones): the walk takes each slot's cone from
  // its record, set up by cone_setup_kernel, and leaves its mask to
  // integrate_kernel. Slots are this chunk's: plain, slots slot_base ..;
  // batched, the cones of packets packet_base .. (from batch cone cone_base).
  constexpr bool kSplit = !kSky && !kSplat;
  const ConeRecord* __restrict__ records = kBatch ? batch.records : q_plain.records;
  uint64_t plain_cones = 0;  // unused when batched
  if constexpr (!kBatch && kSplit) {
    plain_cones = q_plain.slot_count;
    if (q_plain.cones) {
      const uint64_t listed_cones = *q_plain.cones_count;
      const uint64_t left = listed_cones > q_plain.slot_base ? listed_cones - q_plain.slot_base : 0;
      plain_cones = left < plain_cones ? left : plain_cones;
    }
  } else if constexpr (!kBatch) {
    plain_cones = q_plain.cones ? (uint64_t)*q_plain.cones_count : q_plain.npoints * (uint64_t)q_plain.nlights;
  }
  uint64_t npackets;
  if (list) npackets = (uint64_t)min(*list_count, o.redo_capacity);  // one cone per packet
  else npackets = kBatch ? batch.packet_count : (plain_cones + pw - 1) / pw;
  // Packets are taken from a shared counter as warps finish: their costs
  // differ by two orders of magnitude, so a fixed assignment leaves most
  // warps idle behind the slowest.
  uint32_t* next = list ? o.next_solo : o.next_packet;
  for (;;) {
    uint32_t packet = 0;
    if (lane == 0) packet = atomicAdd(next, 1u);
    packet = __shfl_sync(0xffffffffu, packet, 0);
    if (packet >= npackets) break;
    // The packet's job: its scene, query and outputs.
    DevScene s = s_plain;
    DevQuery q = q_plain;
    uint2* out_full = o.full;
    uint2* out_any = o.any;
    float* out_partial = o.partial;
    float* out_irradiance = o.irradiance;
    float* out_fraction = o.fraction;
    uint4* out_work = o.work;
    uint64_t cone_start = 0;  // the job's first cone in the batch's numbering
    uint64_t ncones = plain_cones;
    uint64_t wbase = (uint64_t)packet * pw;
    uint64_t listed = 0;
    // The solo pass (64-bit cells) takes the re-walk list from its end: the
    // packets that finish last, the heaviest, list their cones last, and
    // walked first they no longer set the pass's end (4.99 -> 3.87 ms for the
    // solo pass and integration on the plain workload at scale).
    if (list) listed = list[kWide ? npackets - 1 - packet : packet];
    if constexpr (kBatch) {
      // The packet's job; a listed slot's is in its record (split path), or
      // found from its batch cone number (the prefiltering kernel keeps no
      // records).
      const uint64_t packet_abs = batch.packet_base + packet;
      uint32_t j;
      if (list) j = kSplit ? records[listed].g.w : find_job(batch.jobs, batch.njobs, listed, true);
      else j = find_job(batch.jobs, batch.njobs, packet_abs, false);
      const JobGpu* J = batch.jobs + j;
      s = J->scene;
      q = J->query;
      q.order = batch.order ? batch.order + J->point_start : nullptr;
      out_full = J->full;
      out_any = J->any;
      out_partial = J->partial;
      out_irradiance = J->irradiance;
      out_fraction = J->fraction;
      out_work = J->work;
      cone_start = J->cone_start;
      ncones = q.npoints * (uint64_t)q.nlights;
      if (!list) wbase = (packet_abs - J->packet_start) * (uint64_t)pw;
    }
    const uint64_t slot = wbase + lane;
    bool valid = list ? lane == 0 : ((uint32_t)lane < pw && slot < ncones);
    uint64_t c = 0;
    [[maybe_unused]] uint64_t slot_local = 0;
    [[maybe_unused]] ConeRecord rec;
    if constexpr (kSplit) {
      if (valid) slot_local = list ? listed : (kBatch ? cone_start + slot - batch.cone_base : slot);
      rec = records[slot_local];
      // A batched job with a cone list (an update) has fewer cones than
      // slots: the setup marks the slots past its list.
      if constexpr (kBatch) valid = valid && !(rec.g.x == 0xffffffffu && rec.g.y == 0xffffffffu);
      c = valid ? ((uint64_t)rec.g.x | ((uint64_t)rec.g.y << 32)) : 0;
    } else if (valid) {
      if (list) {
        c = listed - cone_start;
      } else if (q.cones) {
        c = __ldg(&q.cones[slot]);
      } else if (q.order) {
        const uint64_t light_base = (slot / q.npoints) * q.npoints;
        c = light_base + __ldg(&q.order[slot - light_base]);
      } else {
        c = slot;
      }
    }
    const uint32_t l = (uint32_t)(c / q.npoints);
    const uint64_t p = c - (uint64_t)l * q.npoints;

    LaneState<WS> st;
    st.ws = ws;
    st.cov = WS::kSmemCov ? ws->cov + lane : cov_local;
    st.full = 0;
    st.queued = 0;
    st.cone_work = 0;
    st.status = 0;
    st.n_obj = st.n_blas = st.n_tris = 0;
    st.independent = false;
    st.skip = kNoneU;
    st.horizon = st.world_horizon = mk(0.f, 0.f, 0.f);
#pragma unroll 1
    for (int k = 0; k < kBins; ++k) st.cov_at(k) = 0.0f;

    const float4 pt4 = __ldg(&q.receivers[2 * (valid ? p : 0) + 0]);
    const float4 nm4 = __ldg(&q.receivers[2 * (valid ? p : 0) + 1]);
    const f3 point = xyz(pt4), normal = xyz(nm4);
    st.cone = Cone{};
    DevLight L{};
    float spot = 1.0f;
    LightConeInfo info{true, false, false};
    bool traced;
    if constexpr (kSplit) {
      // The cone as cone_setup_kernel set it up.
      st.cone.apex = mk(rec.a.x, rec.a.y, rec.a.z);
      st.cone.far_offset = rec.a.w;
      st.cone.right = mk(rec.b.x, rec.b.y, rec.b.z);
      st.cone.u0 = rec.b.w;
      st.cone.up = mk(rec.c.x, rec.c.y, rec.c.z);
      st.cone.v0 = rec.c.w;
      st.cone.fwd = mk(rec.d.x, rec.d.y, rec.d.z);
      st.cone.u1 = rec.d.w;
      st.cone.baxis = mk(rec.e.x, rec.e.y, rec.e.z);
      st.cone.v1 = rec.e.w;
      st.cone.bcos = rec.f.x;
      st.cone.bsin = rec.f.y;
      const uint32_t flags = __float_as_uint(rec.f.w);
      traced = valid && (flags & 1u);
      st.skip = valid ? (flags >> 4) - 1u : kNoneU;
      info.wide_window = (flags & 2u) != 0u;
      info.wide_clipped = (flags & 4u) != 0u;
      st.cap = rec.g.z;
    } else if constexpr (WS::kSky) {
      // Sky face l of the receiver (sky_face, :1444-1478); walked without a
      // cap (:1059, :1305). With kSkyObjectFrame the receiver's point.w holds
      // (as bits) the object it lies on, whose transform turns the faces
      // (sky_frame = meshes[m].w, :2286, :3602); objects without one, and
      // NONE, keep world axes.
      const float4* frame = nullptr;
      if ((q.sky & kSkyObjectFrame) && s.xforms) {
        const uint32_t m = __float_as_uint(pt4.w);
        if (m < s.nmeshes) {
          const uint32_t x = __ldg(&s.meshes[m]).w;
          if (x != kNoneU) frame = s.xforms + 4 * (size_t)x;
        }
      }
      traced = valid && sky_face(l, point, normal, st.cone, frame);
      st.cap = 0xffffffffu;
      st.independent = (q.sky & kSkyCombineMax) == 0u;
      st.horizon = (q.sky & kSkyNoHorizonCull) == 0u ? normal : mk(0.f, 0.f, 0.f);
      st.world_horizon = st.horizon;
    } else {
      L = load_light(q.lights, valid ? l : 0);
      // hit_irradiance_rect (:2125-2128): spot falloff and the facing test
      // gate the cone.
      spot = spot_falloff(L, normalize(point - light_center(L)));
      const bool on = valid && spot > 0.0f && faces_light(L, point, normal);
      info = light_cone(point, L, q.wide_extent, st.cone);
      traced = on && info.ok;
      st.cap = info.wide_window ? q.wide_cone_cap : q.light_cone_cap;
    }
    st.skips = __any_sync(0xffffffffu, st.skip != kNoneU);
    if (kInst) st.world = st.cone;
    store_cone(ws, st.cone, lane);
    store_horizon(ws, st.horizon, lane);
    __syncwarp();

    if constexpr (kSplat) scene_walk_splat<kCount, kInst>(s, q.prefilter, st, traced, lane);
    else scene_walk<kCount, kInst, kFlat>(s, q.hierarchy, st, traced, lane);

    // A grazing sliver stopped at its cap counts as blocked (:1295-1305).
    const bool capped = traced && st.cone_work >= st.cap;
    if (capped) st.status |= 1u;
    if (capped && info.wide_window && !info.wide_clipped) {
#pragma unroll 1
      for (int k = 0; k < kBins; ++k) st.cov_at(k) = 1.0f;
      st.full = kBins;
    }
    if (traced && st.full >= (uint32_t)kBins) st.status |= 16u;

    uint32_t fw0 = 0, fw1 = 0, aw0 = 0, aw1 = 0;
#pragma unroll 1
    for (int k = 0; k < kBins; ++k) {
      const float v = st.cov_at(k);
      const uint32_t bit = 1u << (k & 31);
      if (v >= 1.0f) { if (k < 32) fw0 |= bit; else fw1 |= bit; }
      if (v > 0.0f) { if (k < 32) aw0 |= bit; else aw1 |= bit; }
    }
    const bool last_empty = (aw0 | aw1) == 0u;
    const bool last_full = (fw0 & fw1) == 0xffffffffu;

    float value = 0.0f, ratio = 1.0f;
    if constexpr (WS::kSky) {
      // sky_face_light (:1489-1498): the face's window clipped to the
      // horizon, less its covered bins' clipped weights.
      if (traced) {
        float blocked = 0.0f;
#pragma unroll 1
        for (int b = 0; b < kBins; ++b) {
          const float cv = st.cov_at(b);
          if (cv > 0.0f) blocked += cv * clipped_bin_weight(st.cone, normal, b);
        }
        const float open = clipped_window_weight(st.cone, normal);
        value = fmaxf(open - blocked, 0.0f);
        ratio = open > 0.0f ? clampf(value / open, 0.0f, 1.0f) : 1.0f;
      }
    } else if constexpr (!kSplit) {
      // The cone table is free now: it is the integration's scratch.
      light_integral(st.cone, point, normal, L, spot, traced, info, last_empty, last_full, ws->cov, ws->cone, lane,
                     value, ratio);
    }

    // A walk again keeps the reasons its packet pass listed the cone for.
    if (valid && list && out_work) st.status |= out_work[c].w & (4u | kStatusAccOverflow);
    if (list) st.status |= 8u;
    const bool redo = !list && o.redo_list &&
                      (((st.status & 4u) && (st.status & (1u | 16u))) || (st.status & kStatusAccOverflow));
    if (redo) {
      const uint32_t at = atomicAdd(o.redo_count, 1u);
      if (at < o.redo_capacity) o.redo_list[at] = kSplit ? (uint32_t)slot_local : (uint32_t)(cone_start + c);
      else atomicOr(o.error, 1u);
    }
    if (st.status & 2u) atomicOr(o.error, 2u);
    if (valid && redo && out_work) out_work[c] = make_uint4(st.n_obj, st.n_blas, st.n_tris, st.status);
    if (valid && !redo) {
      if (out_full) out_full[c] = make_uint2(fw0, fw1);
      if (out_any) out_any[c] = make_uint2(aw0, aw1);
      if constexpr (kSplit) {
        // The mask, for the integration after the walk.
        float4* dst = reinterpret_cast<float4*>(o.cov_out + 64 * slot_local);
#pragma unroll 4
        for (int k = 0; k < 16; ++k)
          dst[k] = make_float4(st.cov_at(4 * k), st.cov_at(4 * k + 1), st.cov_at(4 * k + 2), st.cov_at(4 * k + 3));
      } else {
        if (out_irradiance) out_irradiance[c] = value;
        if (out_fraction) out_fraction[c] = ratio;
      }
      if (out_work) out_work[c] = make_uint4(st.n_obj, st.n_blas, st.n_tris, st.status);
      if (out_partial) {
        float4* dst = reinterpret_cast<float4*>(out_partial + 64 * c);
#pragma unroll 4
        for (int k = 0; k < 16; ++k)
          dst[k] = make_float4(st.cov_at(4 * k), st.cov_at(4 * k + 1), st.cov_at(4 * k + 2), st.cov_at(4 * k + 3));
      }
    }
    __syncwarp();
  }
}

// ---- launch templates ------------------------------------------------------------

// Whether the large dynamic shared memory size was allowed, per device and
// kernel variant (the attribute is set per device); per unit, for the
// variants it launches.
static uint64_t g_attr_set[256] = {};

template <bool kCount, bool kBatch, bool kInst, bool kWide, bool kSky, bool kSplat, bool kBack, bool kFlat>
static cudaError_t launch_variant(const DevScene& s, const DevQuery& q, const DevOut& o, const BatchLaunch& b,
                                  const uint32_t* list, const uint32_t* list_count, uint32_t pw, uint32_t blocks,
                                  cudaStream_t stream) {
  const size_t smem = (size_t)kWarpsPerBlock * sizeof(KernelShared<kWide, kSky, kSplat, kBack, kInst>);
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  const int variant = (kCount ? 1 : 0) + (kBatch ? 2 : 0) + (kInst ? 4 : 0) + (kWide ? 8 : 0) + (kSky ? 16 : 0) +
                      (kSplat ? 32 : 0) + (kBack ? 64 : 0) + (kFlat ? 128 : 0);
  if (!(g_attr_set[variant] & bit)) {
    cudaError_t e = cudaFuncSetAttribute(visibility_kernel<kCount, kBatch, kInst, kWide, kSky, kSplat, kBack, kFlat>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    g_attr_set[variant] |= bit;
  }
  visibility_kernel<kCount, kBatch, kInst, kWide, kSky, kSplat, kBack, kFlat>
      <<<blocks, kWarpsPerBlock * 32, smem, stream>>>(s, q, o, b, list, list_count, pw);
  return cudaGetLastError();
}

// The variant for the launch's hierarchy levels: levels 0 and 1 (a plain
// query's, or some job's of a batch) take the kernel that carries their code.
template <bool kCount, bool kBatch, bool kInst, bool kWide, bool kSky = false, bool kSplat = false,
          bool kBack = false>
static cudaError_t launch_one(const DevScene& s, const DevQuery& q, const DevOut& o, const BatchLaunch& b,
                              const uint32_t* list, const uint32_t* list_count, uint32_t pw, uint32_t blocks,
                              cudaStream_t stream) {
  if constexpr (!kSplat) {
    if (kBatch ? b.flat_levels != 0u : q.hierarchy < 2u)
      return launch_variant<kCount, kBatch, kInst, kWide, kSky, kSplat, kBack, true>(s, q, o, b, list, list_count,
                                                                                     pw, blocks, stream);
  }
  return launch_variant<kCount, kBatch, kInst, kWide, kSky, kSplat, kBack, false>(s, q, o, b, list, list_count, pw,
                                                                                  blocks, stream);
}

// A plain (not batched) pass of the variant the flags pick; q.back (the split
// path's exact cones of a scene without instancing) takes the variant that
// skips each cone's own triangle.
template <bool kWide, bool kSky, bool kSplat>
static cudaError_t plain_pass(bool count, bool inst, const DevScene& s, const DevQuery& q, const DevOut& o,
                              const uint32_t* list, const uint32_t* list_count, uint32_t pw, uint32_t blocks,
                              cudaStream_t stream) {
  const BatchLaunch none{};
  if constexpr (!kSky && !kSplat) {
    if (q.back && !inst)
      return count ? launch_one<true, false, false, kWide, false, false, true>(s, q, o, none, list, list_count, pw,
                                                                               blocks, stream)
                   : launch_one<false, false, false, kWide, false, false, true>(s, q, o, none, list, list_count, pw,
                                                                                blocks, stream);
  }
  if (inst)
    return count ? launch_one<true, false, true, kWide, kSky, kSplat>(s, q, o, none, list, list_count, pw, blocks,
                                                                      stream)
                 : launch_one<false, false, true, kWide, kSky, kSplat>(s, q, o, none, list, list_count, pw, blocks,
                                                                       stream);
  return count ? launch_one<true, false, false, kWide, kSky, kSplat>(s, q, o, none, list, list_count, pw, blocks,
                                                                     stream)
               : launch_one<false, false, false, kWide, kSky, kSplat>(s, q, o, none, list, list_count, pw, blocks,
                                                                      stream);
}

}  // namespace cc
