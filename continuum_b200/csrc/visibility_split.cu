// The split path's kernels before and after the walk: each slot's light
// cone set up (cone_setup_kernel) and each walked mask integrated into the
// cone's light and the cache's ratio (integrate_kernel), with the same
// functions the fused kernels use, so every result is the same. Kept out of
// the walk kernel, whose speed follows the size of its code (instruction
// fetch): without them it is a third smaller.
#include "visibility_kernel.cuh"

namespace cc {

// The cone a slot walks: the listed cone, else its light's walk order.
__device__ __forceinline__ bool slot_cone(const DevQuery& q, uint64_t slot, uint64_t* c) {
  if (q.cones) {
    if (slot >= (uint64_t)*q.cones_count) return false;
    *c = __ldg(&q.cones[slot]);
    return true;
  }
  if (slot >= q.npoints * (uint64_t)q.nlights) return false;
  const uint64_t rank = slot / q.npoints;
  const uint64_t i = slot - rank * q.npoints;
  const uint64_t light = q.light_order ? (uint64_t)__ldg(&q.light_order[rank]) : rank;
  *c = light * q.npoints + (q.order ? (uint64_t)__ldg(&q.order[i]) : i);
  return true;
}

// A slot's record: the spot factor and facing test that gate its cone, and
// the cone itself (hit_irradiance_rect, :2125-2128; light_cone).
// vc_bake's `back` (:3476-3494): the light gives the receiver no unshadowed
// light, yet lies in front of a horizon facing it; the direction to the
// light's centre is that horizon's normal.
__device__ __forceinline__ bool back_facing(const DevLight& L, f3 point, f3 normal, f3& toward) {
  toward = normalize(light_center(L) - point);
  return unshadowed(point, normal, L) <= 0.0f && faces_light(L, point, toward);
}

__device__ __forceinline__ ConeRecord make_record(const DevQuery& q, bool valid, uint64_t c, uint32_t job) {
  const uint32_t l = valid ? (uint32_t)(c / q.npoints) : 0u;
  const uint64_t p = valid ? c - (uint64_t)l * q.npoints : 0u;
  const float4 normal4 = __ldg(&q.receivers[2 * p + 1]);
  const f3 point = xyz(__ldg(&q.receivers[2 * p + 0]));
  f3 normal = xyz(normal4);
  const DevLight L = load_light(q.lights, l);
  // CC_BACK_FACING: the cone of a light below the horizon is traced with a
  // horizon facing the light, past the receiver's own triangle (its slot + 1
  // goes in the flags' top bits).
  uint32_t back = 0u;
  const uint32_t own = __float_as_uint(normal4.w);  // the receiver's own triangle + 1 (0: none)
  if (q.back && valid && own != 0u) {
    f3 toward;
    if (back_facing(L, point, normal, toward)) {
      normal = toward;
      const uint32_t slot = own <= q.ntris ? __ldg(&q.tri_slot[own - 1u]) + 1u : 0u;
      back = 8u | (slot << 4);
    }
  }
  const float spot = spot_falloff(L, normalize(point - light_center(L)));
  const bool on = valid && spot > 0.0f && faces_light(L, point, normal);
  Cone cone{};
  const LightConeInfo info = light_cone(point, L, q.wide_extent, cone);
  const bool traced = on && info.ok;
  const uint32_t flags = (traced ? 1u : 0u) | (info.wide_window ? 2u : 0u) | (info.wide_clipped ? 4u : 0u) | back;
  ConeRecord r;
  r.a = make_float4(cone.apex.x, cone.apex.y, cone.apex.z, cone.far_offset);
  r.b = make_float4(cone.right.x, cone.right.y, cone.right.z, cone.u0);
  r.c = make_float4(cone.up.x, cone.up.y, cone.up.z, cone.v0);
  r.d = make_float4(cone.fwd.x, cone.fwd.y, cone.fwd.z, cone.u1);
  r.e = make_float4(cone.baxis.x, cone.baxis.y, cone.baxis.z, cone.v1);
  r.f = make_float4(cone.bcos, cone.bsin, spot, __uint_as_float(flags));
  // A slot past its cone list holds no cone (both words all ones).
  const uint64_t cn = valid ? c : ~0ull;
  r.g = make_uint4((uint32_t)cn, (uint32_t)(cn >> 32), info.wide_window ? q.wide_cone_cap : q.light_cone_cap, job);
  return r;
}

// One slot per thread. Plain: slots base .. base + n - 1 of q's walk.
// Batched: batch cones b.cone_base .. + b.cone_count, each in its job's walk.
template <bool kBatch>
__global__ void cone_setup_kernel(DevQuery q, BatchLaunch b, uint64_t base, uint64_t n,
                                  ConeRecord* __restrict__ records) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t c = 0;
  uint32_t j = 0;
  if constexpr (kBatch) {
    const uint64_t bc = base + i;
    j = find_job(b.jobs, b.njobs, bc, true);
    const JobGpu* J = b.jobs + j;
    q = J->query;
    q.order = b.order ? b.order + J->point_start : nullptr;
    const bool valid = slot_cone(q, bc - J->cone_start, &c);
    records[i] = make_record(q, valid, c, j);
  } else {
    const bool valid = slot_cone(q, base + i, &c);
    records[i] = make_record(q, valid, c, 0u);
  }
}

// Shared memory of one integrating warp: its 32 slots' masks (bin b of lane
// j at cov[32 b + j]) and the integration's scratch.
struct IntegrateShared {
  float cov[kBins * 32];
  float scratch[kConeFields * 32];
};

// One warp per 32 slots (n of them, from slot 0 of the chunk's records and
// masks; plain calls with a cone list stop at the list's end): each walked
// mask integrated as the fused kernels integrate it (light_integral), the
// results written at each slot's cone, in its job's outputs when batched.
template <bool kBatch>
__global__ void __launch_bounds__(64) integrate_kernel(DevQuery q, DevOut o, BatchLaunch b, uint64_t base,
                                                      uint64_t n, const ConeRecord* __restrict__ records) {
  __shared__ IntegrateShared sh[2];
  const int lane = threadIdx.x & 31;
  IntegrateShared* ws = sh + (threadIdx.x >> 5);
  const uint64_t first = ((uint64_t)blockIdx.x * 2 + (threadIdx.x >> 5)) * 32;
  if (first >= n) return;  // the whole warp leaves together
  uint64_t limit = n;
  if (!kBatch && q.cones) {
    const uint64_t listed = *q.cones_count;
    const uint64_t left = listed > base ? listed - base : 0;
    limit = left < limit ? left : limit;
  }
  const uint64_t slot = first + lane;
  const ConeRecord r = records[slot < limit ? slot : first];
  const uint64_t c = (uint64_t)r.g.x | ((uint64_t)r.g.y << 32);
  // Batched: a slot past its job's cone list holds no cone.
  const bool valid = slot < limit && (!kBatch || c != ~0ull);
  float* irradiance = o.irradiance;
  float* fraction = o.fraction;
  if constexpr (kBatch) {
    const JobGpu* J = b.jobs + r.g.w;
    q.receivers = J->query.receivers;
    q.lights = J->query.lights;
    q.npoints = J->query.npoints;
    irradiance = J->irradiance;
    fraction = J->fraction;
  }
  const uint32_t flags = __float_as_uint(r.f.w);
  const bool traced = valid && (flags & 1u);
  LightConeInfo info;
  info.ok = true;
  info.wide_window = (flags & 2u) != 0u;
  info.wide_clipped = (flags & 4u) != 0u;
  Cone cone{};
  cone.apex = mk(r.a.x, r.a.y, r.a.z);
  cone.far_offset = r.a.w;
  cone.right = mk(r.b.x, r.b.y, r.b.z);
  cone.u0 = r.b.w;
  cone.up = mk(r.c.x, r.c.y, r.c.z);
  cone.v0 = r.c.w;
  cone.fwd = mk(r.d.x, r.d.y, r.d.z);
  cone.u1 = r.d.w;
  cone.baxis = mk(r.e.x, r.e.y, r.e.z);
  cone.v1 = r.e.w;
  cone.bcos = r.f.x;
  cone.bsin = r.f.y;
  const uint64_t cv = valid ? c : 0;  // an invalid slot reads cone 0's inputs and writes nothing
  const uint32_t l = (uint32_t)(cv / q.npoints);
  const uint64_t p = cv - (uint64_t)l * q.npoints;
  const f3 point = xyz(__ldg(&q.receivers[2 * p + 0]));
  f3 normal = xyz(__ldg(&q.receivers[2 * p + 1]));
  const DevLight L = load_light(q.lights, l);
  // A cone traced toward a light below the receiver's horizon (CC_BACK_FACING)
  // is integrated with the horizon facing the light: its ratio is the share
  // seen past the receiver's own triangle, its light 0 (vc_bake :3476-3531).
  const bool back = (flags & 8u) != 0u;
  if (back) normal = normalize(light_center(L) - point);
  // The mask, and whether it is empty or whole.
  bool any = false, all = true;
  const float4* src = reinterpret_cast<const float4*>(o.cov_out + 64 * (valid ? slot : first));
#pragma unroll 4
  for (int k = 0; k < 16; ++k) {
    const float4 v = src[k];
    const float vs[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float x = valid ? vs[j] : 0.0f;
      ws->cov[32 * (4 * k + j) + lane] = x;
      any = any || x > 0.0f;
      all = all && x >= 1.0f;
    }
  }
  __syncwarp();
  float value, ratio;
  light_integral(cone, point, normal, L, r.f.z, traced, info, !any, all, ws->cov, ws->scratch, lane, value, ratio);
  if (valid) {
    if (irradiance) irradiance[c] = back ? 0.0f : value;
    if (fraction) fraction[c] = ratio;
  }
}

cudaError_t upload_disk_table_split(const float* table64) {
  return cudaMemcpyToSymbol(c_disk, table64, kBins * sizeof(float));
}

// One block: per light, the windows of its traced cones summed over the same
// sample of points (at most 1024, evenly strided), then the lights ranked
// by that sum, largest first (ties by index). Packet costs follow the
// cone's window (a wider cone meets more of the scene), and the packets of
// the light walked last end the pass.
__global__ void __launch_bounds__(256) light_order_kernel(DevQuery q, uint32_t* __restrict__ out) {
  __shared__ float sum[kMaxOrderedLights];
  __shared__ float part[8];
  const uint32_t L = q.nlights;
  const uint64_t samples = q.npoints < 1024 ? q.npoints : 1024;
  const uint64_t stride = samples ? q.npoints / samples : 1;
  for (uint32_t l = 0; l < L; ++l) {
    const DevLight light = load_light(q.lights, l);
    float acc = 0.0f;
    for (uint64_t k = threadIdx.x; k < samples; k += blockDim.x) {
      const uint64_t p = k * stride;
      const f3 point = xyz(__ldg(&q.receivers[2 * p + 0]));
      const f3 normal = xyz(__ldg(&q.receivers[2 * p + 1]));
      if (!(spot_falloff(light, normalize(point - light_center(light))) > 0.0f) || !faces_light(light, point, normal))
        continue;
      Cone cone{};
      if (light_cone(point, light, q.wide_extent, cone).ok) acc += (cone.u1 - cone.u0) * (cone.v1 - cone.v0);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      float total = 0.0f;
      for (int w = 0; w < 8; ++w) total += part[w];
      sum[l] = total;
    }
    __syncthreads();
  }
  for (uint32_t l = threadIdx.x; l < L; l += blockDim.x) {
    uint32_t rank = 0;
    for (uint32_t k = 0; k < L; ++k) rank += (sum[k] > sum[l] || (sum[k] == sum[l] && k < l)) ? 1u : 0u;
    out[rank] = l;
  }
}

cudaError_t launch_light_order(const DevQuery& q, uint32_t* out, cudaStream_t stream) {
  if (q.nlights == 0 || q.nlights > kMaxOrderedLights) return cudaErrorInvalidValue;
  light_order_kernel<<<1, 256, 0, stream>>>(q, out);
  return cudaGetLastError();
}

cudaError_t launch_cone_setup(const DevQuery& q, uint64_t base, uint64_t n, ConeRecord* records, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cone_setup_kernel<false><<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(q, BatchLaunch{}, base, n, records);
  return cudaGetLastError();
}

cudaError_t launch_integrate(const DevQuery& q, const DevOut& o, uint64_t base, uint64_t n,
                             const ConeRecord* records, cudaStream_t stream) {
  if (n == 0 || (!o.irradiance && !o.fraction)) return cudaSuccess;
  const uint64_t warps = (n + 31) / 32;
  integrate_kernel<false><<<(unsigned)((warps + 1) / 2), 64, 0, stream>>>(q, o, BatchLaunch{}, base, n, records);
  return cudaGetLastError();
}

cudaError_t launch_batch_setup(const BatchLaunch& b, cudaStream_t stream) {
  const uint64_t n = b.cone_count;
  if (n == 0) return cudaSuccess;
  cone_setup_kernel<true><<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(DevQuery{}, b, b.cone_base, n, b.records);
  return cudaGetLastError();
}

cudaError_t launch_batch_integrate(const BatchLaunch& b, const DevOut& o, cudaStream_t stream) {
  const uint64_t n = b.cone_count;
  if (n == 0) return cudaSuccess;
  const uint64_t warps = (n + 31) / 32;
  integrate_kernel<true><<<(unsigned)((warps + 1) / 2), 64, 0, stream>>>(DevQuery{}, o, b, b.cone_base, n, b.records);
  return cudaGetLastError();
}

std::vector<BatchChunk> batch_chunks(const std::vector<uint64_t>& cones, uint32_t pw, uint64_t max_slots) {
  std::vector<BatchChunk> out;
  BatchChunk cur{0, 0, 0, 0};
  for (const uint64_t c : cones) {
    const uint64_t packets = (c + pw - 1) / pw;
    uint64_t done = 0;  // the job's packets taken
    while (done < packets) {
      const uint64_t room = max_slots - cur.cone_count;
      if (room < pw) {
        out.push_back(cur);
        cur = BatchChunk{cur.packet_base + cur.packet_count, 0, cur.cone_base + cur.cone_count, 0};
        continue;
      }
      uint64_t take = room / pw;
      if (take > packets - done) take = packets - done;
      const uint64_t end = (done + take) * pw < c ? (done + take) * pw : c;  // a job's last packet may be short
      cur.packet_count += take;
      cur.cone_count += end - done * pw;
      done += take;
    }
  }
  if (cur.packet_count) out.push_back(cur);
  return out;
}

}  // namespace cc
