// The order in which receivers are walked: Morton order of their positions.
//
// A warp walks up to 32 cones together and visits the union of the nodes
// its cones need, so cones in a warp should see the same geometry. Callers
// list receivers in their own order (image rows, texels of many pages); here
// each receiver gets a 30-bit Morton code of its position quantized in the
// scene's bounds, and a device radix sort yields the walk order. Results do
// not depend on the order — only which cones share a warp.
#include <cub/device/device_radix_sort.cuh>

#include <cstdint>

#include "kernels.h"

namespace cc {

namespace {

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void morton_keys(const float4* __restrict__ receivers, uint64_t n, float3 lo, float3 scale,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ index) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = __ldg(&receivers[2 * i]);
  auto q = [](float x, float l, float s) {
    float t = (x - l) * s;
    t = fminf(fmaxf(t, 0.0f), 1023.0f);  // NaN clamps to 0
    return (uint32_t)t;
  };
  keys[i] = (spread10(q(p.x, lo.x, scale.x)) << 2) | (spread10(q(p.y, lo.y, scale.y)) << 1) |
            spread10(q(p.z, lo.z, scale.z));
  index[i] = (uint32_t)i;
}

// Batch keys: the job's index above the point's 30-bit code; values: the
// point's index within its job.
__global__ void batch_morton_keys(BatchLaunch b, unsigned long long* __restrict__ keys,
                                  uint32_t* __restrict__ index) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.points) return;
  uint32_t lo = 0, hi = b.njobs;  // jobs[lo].point_start <= i < jobs[hi].point_start
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(&b.jobs[mid].point_start) <= i) lo = mid; else hi = mid;
  }
  const JobGpu& J = b.jobs[lo];
  const uint64_t local = i - J.point_start;
  const float4 p = __ldg(&J.query.receivers[2 * local]);
  auto q = [](float x, float l, float h) {
    const float s = (h - l) > 0.0f ? 1023.0f / (h - l) : 0.0f;
    float t = (x - l) * s;
    t = fminf(fmaxf(t, 0.0f), 1023.0f);  // NaN clamps to 0
    return (uint32_t)t;
  };
  const uint32_t code = (spread10(q(p.x, J.lo[0], J.hi[0])) << 2) | (spread10(q(p.y, J.lo[1], J.hi[1])) << 1) |
                        spread10(q(p.z, J.lo[2], J.hi[2]));
  keys[i] = ((unsigned long long)lo << 30) | code;
  index[i] = (uint32_t)local;
}

int job_bits(uint32_t njobs) {
  int bits = 0;
  while ((1ull << bits) < njobs) ++bits;
  return bits;
}

}  // namespace

size_t batch_order_scratch_bytes(uint64_t points) {
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)points, 0, 62);
  return points * (2 * sizeof(unsigned long long) + sizeof(uint32_t)) + temp + 512;
}

cudaError_t batch_order(const BatchLaunch& b, void* scratch, size_t scratch_bytes, uint32_t* order,
                        cudaStream_t stream) {
  if (b.points == 0 || b.njobs == 0) return cudaSuccess;
  const uint64_t n = b.points;
  auto align = [](uint8_t* p) {
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
  };
  uint8_t* base = align(static_cast<uint8_t*>(scratch));
  unsigned long long* keys_in = reinterpret_cast<unsigned long long*>(base);
  unsigned long long* keys_out = keys_in + n;
  uint32_t* idx_in = reinterpret_cast<uint32_t*>(keys_out + n);
  uint8_t* temp = align(reinterpret_cast<uint8_t*>(idx_in + n));
  const size_t used = static_cast<size_t>(temp - static_cast<uint8_t*>(scratch));
  if (used > scratch_bytes) return cudaErrorInvalidValue;
  size_t temp_bytes = scratch_bytes - used;
  const unsigned threads = 256;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  batch_morton_keys<<<blocks, threads, 0, stream>>>(b, keys_in, idx_in);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, idx_in, order, (int)n, 0,
                                         30 + job_bits(b.njobs), stream);
}

size_t walk_order_scratch_bytes(uint64_t npoints) {
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)npoints, 0, 30);
  return 4 * npoints * sizeof(uint32_t) + temp + 256;
}

cudaError_t walk_order(const float4* receivers, uint64_t npoints, const float* scene_lo, const float* scene_hi,
                       void* scratch, size_t scratch_bytes, uint32_t* order, cudaStream_t stream) {
  if (npoints == 0) return cudaSuccess;
  uint32_t* keys_in = static_cast<uint32_t*>(scratch);
  uint32_t* keys_out = keys_in + npoints;
  uint32_t* idx_in = keys_out + npoints;
  uint8_t* temp = reinterpret_cast<uint8_t*>(idx_in + npoints);
  // 256-byte alignment for the sort's temporary storage.
  temp = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(temp) + 255) & ~uintptr_t(255));
  const size_t used = static_cast<size_t>(temp - static_cast<uint8_t*>(scratch));
  if (used > scratch_bytes) return cudaErrorInvalidValue;
  size_t temp_bytes = scratch_bytes - used;
  float3 lo = make_float3(scene_lo[0], scene_lo[1], scene_lo[2]);
  auto inv = [](float a, float b) { return (b - a) > 0.0f ? 1023.0f / (b - a) : 0.0f; };
  float3 scale = make_float3(inv(scene_lo[0], scene_hi[0]), inv(scene_lo[1], scene_hi[1]), inv(scene_lo[2], scene_hi[2]));
  const unsigned threads = 256;
  const unsigned blocks = (unsigned)((npoints + threads - 1) / threads);
  morton_keys<<<blocks, threads, 0, stream>>>(receivers, npoints, lo, scale, keys_in, idx_in);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, idx_in, order, (int)npoints, 0, 30,
                                         stream);
}

}  // namespace cc
