// The plain visibility kernel: one warp walks a packet of up to 32 cones
// (neighbouring points toward one light) through the scene hierarchy
// together; each lane tests, rasterizes and integrates its own cone.
//
// What the reference does per invocation (mask_cones.wgsl `main` :1513-1520
// -> hit_irradiance_rect :2125 -> cone_irradiance_rect :1286) is done here
// per lane, with the packet walk of the reference's PACKETS mode
// (packet_any, :666-711) built from warp votes:
//  * the traversal stack is warp-uniform and lives in registers spread over
//    the lanes (entry i in lane i % 32), so a push is one predicated move and
//    a pop one shuffle — no shared or local memory;
//  * each lane keeps a bit per stack entry saying whether its own walk needs
//    that entry (need_get/need_put, :694-711);
//  * node and triangle records are loaded by every lane from the same
//    address, which the load unit serves as one broadcast transaction.
// Results depend on the walk order only through the walk caps: the packet
// takes its child order from its first lane that descends; a lane whose own
// nearest-first order differs somewhere on its walk, and whose walk then
// stopped early (capped, or every bin full), is listed and walked again
// alone by a second launch, so every cone's result is the one its own walk
// gives (the reference's walk without packets, as its view-cache bakes run).
#include <cstdint>
#include <cuda_runtime.h>

#include "cone_device.cuh"
#include "kernels.h"

namespace cc {

__constant__ float c_disk[kBins];  // DISK (mask_cones.wgsl:888-897), uploaded by the host

constexpr int kStack = 64;         // entries; the reference's is 48 (mask_cones.wgsl:111)
// Shared memory per warp: the lanes' coverages (64 x 32), accumulators
// (64 x 32) and the cooperative integration's corners and edges (387).
constexpr int kScratchFloats = 416;
constexpr int kWarpFloats = 2 * kBins * 32 + kScratchFloats;

// A stack entry is a node reference packed in one word: the node's item
// count in the top 4 bits (0: interior) and its first item (leaf) or left
// child (interior) below. Each lane keeps two bits per entry: whether its
// own walk needs the entry, and whether its cone passed the entry's box
// test, which is done when the parent is visited (the two children of a
// node are adjacent, so one 64-byte load serves both tests and the
// nearest-first choice).
constexpr uint32_t kRefIndexBits = 28;
constexpr uint32_t kRefIndexMask = (1u << kRefIndexBits) - 1u;
__device__ __forceinline__ uint32_t node_ref(float4 a, float4 b) {
  return (__float_as_uint(b.w) << kRefIndexBits) | (__float_as_uint(a.w) & kRefIndexMask);
}

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

struct LaneState {
  Cone cone;
  f3 d00, d10, d01, d11;  // window corner directions
  float* cov;             // &cov[lane]; bin b at cov[32 * b]
  float* acc;             // &acc[lane]
  uint32_t full;
  uint32_t cone_work;
  uint32_t cap;
  uint32_t status;
  uint32_t n_obj, n_blas, n_tris;
};

__device__ __forceinline__ f3 node_lo(float4 a) { return mk(a.x, a.y, a.z); }

// The cheap tests of cover_triangle (:594-612): faces the apex, some window
// direction enters its plane, may touch the cone.
__device__ __forceinline__ bool cull_triangle(const LaneState& st, f3 v0, f3 v1, f3 v2) {
  const Cone& c = st.cone;
  f3 n = cross(v1 - v0, v2 - v0);
  if (dot(n, c.apex - v0) <= 0.0f) return false;  // faces away (:600)
  if (dot(n, st.d00) >= 0.f && dot(n, st.d10) >= 0.f && dot(n, st.d01) >= 0.f && dot(n, st.d11) >= 0.f)
    return false;  // every window direction leaves its plane (:601-606)
  return may_touch(c, v0, v1, v2);
}

// cover_triangle (:594-616): triangle slot t rasterized into `acc` if it
// faces the apex and may touch the cone.
template <bool kCount>
__device__ __forceinline__ bool cover_triangle(const DevScene& s, LaneState& st, LaneAcc& acc, uint32_t t) {
  if (kCount) st.n_tris++;
  f3 v0 = xyz(__ldg(&s.tris[3 * (size_t)t + 0]));
  f3 v1 = xyz(__ldg(&s.tris[3 * (size_t)t + 1]));
  f3 v2 = xyz(__ldg(&s.tris[3 * (size_t)t + 2]));
  if (!cull_triangle(st, v0, v1, v2)) return false;
  return rasterize(st.cone, acc, v0, v1, v2);
}

// add_mesh_coverage_if (:713-829) for the lanes with `on`; the others
// follow the packet's walk. The triangle hierarchy's stack entries start at
// `base`, above the object walk's. A node still counts toward the walk cap
// when it is popped, as in the reference, though its box was tested when its
// parent was visited. Triangles are stored in leaf order, so a leaf's items
// are the triangle slots themselves.
template <bool kCount>
__device__ __forceinline__ void add_mesh(const DevScene& s, uint32_t hierarchy, LaneState& st, WarpStack& stk,
                                         bool on, uint32_t m, int base, int lane) {
  if (!__any_sync(0xffffffffu, on)) return;
  const uint4 range = __ldg(&s.meshes[m]);
  LaneAcc acc{st.acc, 68u, 0u};
  bool touched = false;
  if (hierarchy == 2) {
    if (range.z != kNoneU) {
      const float4 ra = __ldg(&s.blas[2 * (size_t)range.z + 0]);
      const float4 rb = __ldg(&s.blas[2 * (size_t)range.z + 1]);
      const bool root_pass = on && may_touch_box(st.cone, node_lo(ra), node_lo(rb));
      int sp = base;
      stk.push(sp, node_ref(ra, rb), on, root_pass, lane);
      ++sp;
      while (sp > base) {
        --sp;
        const uint32_t ref = stk.get(sp);
        const bool mine = stk.need(sp) && st.cone_work < st.cap;
        if (mine) st.cone_work++;
        if (kCount && mine) st.n_blas++;
        const bool descend = mine && stk.pass(sp);
        if (!__any_sync(0xffffffffu, descend)) continue;
        const uint32_t ia = ref & kRefIndexMask, ib = ref >> kRefIndexBits;
        if (ib > 0) {
          if (descend) {
            st.cone_work += ib;
            for (uint32_t k = ia; k < ia + ib; ++k)
              if (cover_triangle<kCount>(s, st, acc, k)) touched = true;
          }
        } else {
          const float4 la = __ldg(&s.blas[2 * (size_t)ia + 0]);
          const float4 lb = __ldg(&s.blas[2 * (size_t)ia + 1]);
          const float4 xa = __ldg(&s.blas[2 * (size_t)ia + 2]);
          const float4 xb = __ldg(&s.blas[2 * (size_t)ia + 3]);
          bool pl = false, pr = false;
          if (descend) {
            pl = may_touch_box(st.cone, node_lo(la), node_lo(lb));
            pr = may_touch_box(st.cone, node_lo(xa), node_lo(xb));
          }
          if (sp + 2 > kStack) {
            if (descend) st.status |= 2u;
            continue;
          }
          // Right child popped first (:783-787).
          stk.push(sp, node_ref(la, lb), descend, pl, lane);
          stk.push(sp + 1, node_ref(xa, xb), descend, pr, lane);
          sp += 2;
        }
      }
    }
  } else if (on) {
    for (uint32_t t = range.x; t < range.x + range.y; ++t)
      if (cover_triangle<kCount>(s, st, acc, t)) touched = true;
  }
  // The mesh's coverage: running sum over the touched cells, snapped to
  // whole within 1e-5, combined into the cone's bins by max (:809-828).
  const uint32_t end = min(acc.span_hi, (uint32_t)kBins);
  if (touched) {
    float running = 0.0f;
    for (uint32_t b = acc.span_lo; b < end; ++b) {
      running += st.acc[32 * b];
      float covered = fabsf(running);
      if (covered >= 1.0f - 1e-5f) covered = 1.0f;
      if (covered > 1e-6f) {
        const float before = st.cov[32 * b];
        const float after = fmaxf(before, fminf(covered, 1.0f));
        st.cov[32 * b] = after;
        if (before < 1.0f && after >= 1.0f) st.full++;
      }
    }
  }
  for (uint32_t b = acc.span_lo; b < end; ++b) st.acc[32 * b] = 0.0f;
}

// scene_coverage_if (:1160-1227): the object hierarchy, nearest child first
// along the bounding cone's axis, until every bin is full or the cap.
template <bool kCount>
__device__ __forceinline__ void scene_walk(const DevScene& s, uint32_t hierarchy, LaneState& st, bool traced,
                                           int lane) {
  WarpStack stk;
  if (hierarchy >= 1) {
    const float4 ra = __ldg(&s.nodes[0]);
    const float4 rb = __ldg(&s.nodes[1]);
    const bool root_pass = traced && may_touch_box(st.cone, node_lo(ra), node_lo(rb));
    stk.push(0, node_ref(ra, rb), traced, root_pass, lane);
    int sp = 1;
    while (sp > 0) {
      --sp;
      const uint32_t ref = stk.get(sp);
      const bool mine = stk.need(sp) && st.full < (uint32_t)kBins && st.cone_work < st.cap;
      if (mine) st.cone_work++;
      if (kCount && mine) st.n_obj++;
      const bool descend = mine && stk.pass(sp);
      if (!__any_sync(0xffffffffu, descend)) continue;
      const uint32_t ia = ref & kRefIndexMask, ib = ref >> kRefIndexBits;
      if (ib > 0) {
        for (uint32_t k = ia; k < ia + ib; ++k)
          add_mesh<kCount>(s, hierarchy, st, stk, descend, __ldg(&s.items[k]), sp, lane);
      } else {
        const float4 la = __ldg(&s.nodes[2 * (size_t)ia + 0]);
        const float4 lb = __ldg(&s.nodes[2 * (size_t)ia + 1]);
        const float4 xa = __ldg(&s.nodes[2 * (size_t)ia + 2]);
        const float4 xb = __ldg(&s.nodes[2 * (size_t)ia + 3]);
        const Cone& c = st.cone;
        bool pl = false, pr = false;
        if (descend) {
          pl = may_touch_box(c, node_lo(la), node_lo(lb));
          pr = may_touch_box(c, node_lo(xa), node_lo(xb));
        }
        const float da = dot(c.baxis, (node_lo(la) + node_lo(lb)) * 0.5f - c.apex);
        const float db = dot(c.baxis, (node_lo(xa) + node_lo(xb)) * 0.5f - c.apex);
        const bool pref = db < da;  // this lane's own order: right child nearer
        const uint32_t voters = __ballot_sync(0xffffffffu, descend);
        const bool swap = __shfl_sync(0xffffffffu, pref, __ffs(voters) - 1);
        if (descend && pref != swap) st.status |= 4u;
        if (sp + 2 > kStack) {
          if (descend) st.status |= 2u;
          continue;
        }
        const uint32_t rl = node_ref(la, lb), rr = node_ref(xa, xb);
        // The far child below the near one: the near child is popped first.
        stk.push(sp, swap ? rl : rr, descend, swap ? pl : pr, lane);
        stk.push(sp + 1, swap ? rr : rl, descend, swap ? pr : pl, lane);
        sp += 2;
      }
    }
  } else {
    for (uint32_t m = 0; m < s.nmeshes; ++m)
      add_mesh<kCount>(s, hierarchy, st, stk, traced && st.full < (uint32_t)kBins, m, 0, lane);
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
__device__ __noinline__ float warp_blocked(const Cone& mine, f3 my_normal, bool my_all_above, const float* cov_j,
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

template <bool kCount>
// Three blocks per SM fit the shared memory (3 x 64 KB); saying so lets the
// register allocator use up to 170 registers a thread instead of spilling.
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kBlocksPerSm)
    visibility_kernel(DevScene s, DevQuery q, DevOut o, const uint32_t* __restrict__ list,
                      const uint32_t* __restrict__ list_count, uint32_t pw) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  float* cov_base = smem + (size_t)wib * kWarpFloats;
  float* acc_base = cov_base + kBins * 32;
  float* scratch = acc_base + kBins * 32;
  for (int k = 0; k < kBins; ++k) acc_base[32 * k + lane] = 0.0f;

  const uint64_t ncones = list ? (uint64_t)min(*list_count, o.redo_capacity) : q.npoints * (uint64_t)q.nlights;
  const uint64_t npackets = (ncones + pw - 1) / pw;
  // Packets are taken from a shared counter as warps finish: their costs
  // differ by two orders of magnitude, so a fixed assignment leaves most
  // warps idle behind the slowest.
  uint32_t* next = list ? o.next_solo : o.next_packet;
  for (;;) {
    uint32_t packet = 0;
    if (lane == 0) packet = atomicAdd(next, 1u);
    packet = __shfl_sync(0xffffffffu, packet, 0);
    if (packet >= npackets) break;
    const uint64_t wbase = (uint64_t)packet * pw;
    const uint64_t slot = wbase + lane;
    const bool valid = (uint32_t)lane < pw && slot < ncones;
    uint64_t c = 0;
    if (valid) {
      if (list) {
        c = list[slot];
      } else if (q.order) {
        const uint64_t light_base = (slot / q.npoints) * q.npoints;
        c = light_base + __ldg(&q.order[slot - light_base]);
      } else {
        c = slot;
      }
    }
    const uint32_t l = (uint32_t)(c / q.npoints);
    const uint64_t p = c - (uint64_t)l * q.npoints;

    LaneState st;
    st.cov = cov_base + lane;
    st.acc = acc_base + lane;
    st.full = 0;
    st.cone_work = 0;
    st.status = 0;
    st.n_obj = st.n_blas = st.n_tris = 0;
    for (int k = 0; k < kBins; ++k) st.cov[32 * k] = 0.0f;

    const DevLight L = load_light(q.lights, valid ? l : 0);
    const float4 pt4 = __ldg(&q.receivers[2 * (valid ? p : 0) + 0]);
    const float4 nm4 = __ldg(&q.receivers[2 * (valid ? p : 0) + 1]);
    const f3 point = xyz(pt4), normal = xyz(nm4);

    // hit_irradiance_rect (:2125-2128): spot falloff and the facing test gate
    // the cone.
    const float spot = spot_falloff(L, normalize(point - light_center(L)));
    const bool on = valid && spot > 0.0f && faces_light(L, point, normal);
    st.cone = Cone{};
    const LightConeInfo info = light_cone(point, L, q.wide_extent, st.cone);
    const bool traced = on && info.ok;
    st.cap = info.wide_window ? q.wide_cone_cap : q.light_cone_cap;
    st.d00 = direction(st.cone, 0.f, 0.f);
    st.d10 = direction(st.cone, 1.f, 0.f);
    st.d01 = direction(st.cone, 0.f, 1.f);
    st.d11 = direction(st.cone, 1.f, 1.f);

    scene_walk<kCount>(s, q.hierarchy, st, traced, lane);

    // A grazing sliver stopped at its cap counts as blocked (:1295-1305).
    const bool capped = traced && st.cone_work >= st.cap;
    if (capped) st.status |= 1u;
    if (capped && info.wide_window && !info.wide_clipped) {
      for (int k = 0; k < kBins; ++k) st.cov[32 * k] = 1.0f;
      st.full = kBins;
    }
    if (traced && st.full >= (uint32_t)kBins) st.status |= 16u;

    uint32_t fw0 = 0, fw1 = 0, aw0 = 0, aw1 = 0;
    for (int k = 0; k < kBins; ++k) {
      const float v = st.cov[32 * k];
      const uint32_t bit = 1u << (k & 31);
      if (v >= 1.0f) { if (k < 32) fw0 |= bit; else fw1 |= bit; }
      if (v > 0.0f) { if (k < 32) aw0 |= bit; else aw1 |= bit; }
    }
    const bool last_empty = (aw0 | aw1) == 0u;
    const bool last_full = (fw0 & fw1) == 0xffffffffu;

    // Rect light cones with coverage: the bins' Lambert weights, one cone at
    // a time across the warp.
    const bool rect_traced = traced && !is_sphere(L);
    bool all_above = true;
    float total = 0.0f;
    if (rect_traced) total = window_weight(st.cone, normal, &all_above);
    float blocked = 0.0f;
    uint32_t todo = __ballot_sync(0xffffffffu, rect_traced && !last_empty);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const float b = warp_blocked(st.cone, normal, all_above, cov_base + j, scratch, j, lane);
      if (lane == j) blocked = b;
    }
    float value = 0.0f;
    if (traced) {
      const Cone& cn = st.cone;
      if (is_sphere(L)) {
        // sphere_open_share (:957-972)
        float total = 0.0f, open = 0.0f;
        const float g = float(kGrid);
        for (int b = 0; b < kBins; ++b) {
          const float mfrac = info.wide_clipped ? 1.0f : c_disk[b];
          if (mfrac <= 0.0f) continue;
          f3 d = direction(cn, (float(b % kGrid) + 0.5f) / g, (float(b / kGrid) + 0.5f) / g);
          float l2 = dot(d, d);
          float w = mfrac * fmaxf(dot(normal, d), 0.0f) / (l2 * l2);
          total += w;
          open += w * (1.0f - st.cov[32 * b]);
        }
        const float share = total <= 0.0f ? 1.0f : open / total;
        value = sphere_unshadowed(point, normal, L) * share;
      } else {
        // cone_visible (:1244-1272) and wide_visible (:1070-1073)
        float visible = fmaxf(total - blocked, 0.0f);
        if (info.wide_clipped) visible = (total > 1e-9f ? visible / total : 1.0f) * rect_open(point, normal, L);
        value = visible;
      }
    }
    value *= spot;
    // The lighting cache's ratio (vc_bake :3453-3510, static light).
    const float open = unshadowed(point, normal, L);
    float ratio = open > 0.0f ? clampf(value / open, 0.0f, 1.0f) : 1.0f;
    if (open > 0.0f && last_empty) ratio = 1.0f;
    if (open > 0.0f && last_full) ratio = 0.0f;

    if (list) st.status |= 8u;
    const bool redo = !list && o.redo_list && (st.status & 4u) && (st.status & (1u | 16u));
    if (redo) {
      const uint32_t at = atomicAdd(o.redo_count, 1u);
      if (at < o.redo_capacity) o.redo_list[at] = (uint32_t)c;
      else atomicOr(o.error, 1u);
    }
    if (st.status & 2u) atomicOr(o.error, 2u);
    if (valid && !redo) {
      if (o.full) o.full[c] = make_uint2(fw0, fw1);
      if (o.any) o.any[c] = make_uint2(aw0, aw1);
      if (o.irradiance) o.irradiance[c] = value;
      if (o.fraction) o.fraction[c] = ratio;
      if (o.work) o.work[c] = make_uint4(st.n_obj, st.n_blas, st.n_tris, st.status);
      if (o.partial) {
        float4* dst = reinterpret_cast<float4*>(o.partial + 64 * c);
#pragma unroll 4
        for (int k = 0; k < 16; ++k)
          dst[k] = make_float4(st.cov[32 * (4 * k)], st.cov[32 * (4 * k + 1)], st.cov[32 * (4 * k + 2)],
                               st.cov[32 * (4 * k + 3)]);
      }
    }
  }
}

// ---- host-side launchers --------------------------------------------------------

cudaError_t upload_disk_table(const float* table64) {
  return cudaMemcpyToSymbol(c_disk, table64, kBins * sizeof(float));
}

// Whether the large dynamic shared memory size was allowed, per device and
// kernel variant (the attribute is set per device).
static uint64_t g_attr_set[2] = {0, 0};

template <bool kCount>
static cudaError_t launch_one(const DevScene& s, const DevQuery& q, const DevOut& o, const uint32_t* list,
                              const uint32_t* list_count, uint32_t pw, uint32_t blocks, cudaStream_t stream) {
  const size_t smem = (size_t)kWarpsPerBlock * kWarpFloats * sizeof(float);
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(g_attr_set[kCount] & bit)) {
    cudaError_t e = cudaFuncSetAttribute(visibility_kernel<kCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    g_attr_set[kCount] |= bit;
  }
  visibility_kernel<kCount><<<blocks, kWarpsPerBlock * 32, smem, stream>>>(s, q, o, list, list_count, pw);
  return cudaGetLastError();
}

cudaError_t launch_visibility(const DevScene& s, const DevQuery& q, const DevOut& o, uint32_t pw, bool count,
                              int sm_count, cudaStream_t stream, const cudaEvent_t* marks) {
  if (pw < 1) pw = 1;
  if (pw > 32) pw = 32;
  const uint64_t ncones = q.npoints * (uint64_t)q.nlights;
  if (marks) cudaEventRecord(marks[0], stream);
  if (ncones == 0) {
    if (marks) {
      cudaEventRecord(marks[1], stream);
      cudaEventRecord(marks[2], stream);
    }
    return cudaSuccess;
  }
  const uint64_t packets = (ncones + pw - 1) / pw;
  // Enough blocks to fill every SM several times over; each warp then strides
  // over packets.
  const uint64_t want = (packets + kWarpsPerBlock - 1) / kWarpsPerBlock;
  // One resident wave: warps take packets from the shared counter.
  const uint64_t cap = (uint64_t)sm_count * kBlocksPerSm;
  const uint32_t blocks = (uint32_t)(want < cap ? want : cap);
  cudaError_t e = count ? launch_one<true>(s, q, o, nullptr, nullptr, pw, blocks, stream)
                        : launch_one<false>(s, q, o, nullptr, nullptr, pw, blocks, stream);
  if (marks) cudaEventRecord(marks[1], stream);
  if (e != cudaSuccess) return e;
  if (o.redo_list) {
    // The listed cones, each walked alone (one lane per warp).
    const uint32_t solo_blocks = (uint32_t)sm_count * kBlocksPerSm;
    e = count ? launch_one<true>(s, q, o, o.redo_list, o.redo_count, 1, solo_blocks, stream)
              : launch_one<false>(s, q, o, o.redo_list, o.redo_count, 1, solo_blocks, stream);
  }
  if (marks) cudaEventRecord(marks[2], stream);
  return e;
}

}  // namespace cc
