// The prefiltering cones' variants of the visibility kernel (kSplat), in a
// unit of their own so that the exact cones' kernels (visibility.cu) are
// compiled as they are without them.
#include "visibility_kernel.cuh"

namespace cc {

cudaError_t upload_disk_table_splat(const float* table64) {
  return cudaMemcpyToSymbol(c_disk, table64, kBins * sizeof(float));
}

cudaError_t launch_splat_pass(bool wide, bool count, bool inst, bool sky, const DevScene& s, const DevQuery& q,
                              const DevOut& o, const uint32_t* list, const uint32_t* list_count, uint32_t pw,
                              uint32_t blocks, cudaStream_t stream) {
  if (wide)
    return sky ? plain_pass<true, true, true>(count, inst, s, q, o, list, list_count, pw, blocks, stream)
               : plain_pass<true, false, true>(count, inst, s, q, o, list, list_count, pw, blocks, stream);
  return sky ? plain_pass<false, true, true>(count, inst, s, q, o, list, list_count, pw, blocks, stream)
             : plain_pass<false, false, true>(count, inst, s, q, o, list, list_count, pw, blocks, stream);
}

cudaError_t launch_batch_splat(const BatchLaunch& b0, const DevOut& o, bool count, int sm_count, int blocks_per_sm,
                               cudaStream_t stream) {
  if (b0.njobs == 0 || b0.packets == 0) return cudaSuccess;
  BatchLaunch b = b0;
  b.packet_base = 0;
  b.packet_count = b0.packets;
  const DevScene s{};
  const DevQuery q{};
  if (blocks_per_sm < 1) blocks_per_sm = 1;
  if (blocks_per_sm > kFusedBlocksPerSm) blocks_per_sm = kFusedBlocksPerSm;
  const uint64_t want = (b.packet_count + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const uint64_t cap = (uint64_t)sm_count * blocks_per_sm;
  const uint32_t blocks = (uint32_t)(want < cap ? want : cap);
  cudaError_t e;
  if (b.inst) {
    e = count ? launch_one<true, true, true, false, false, true>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream)
              : launch_one<false, true, true, false, false, true>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream);
  } else {
    e = count ? launch_one<true, true, false, false, false, true>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream)
              : launch_one<false, true, false, false, false, true>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream);
  }
  if (e != cudaSuccess || !o.redo_list) return e;
  const uint32_t solo = (uint32_t)sm_count * kFusedSoloBlocksPerSm;
  if (b.inst)
    return count ? launch_one<true, true, true, true, false, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo, stream)
                 : launch_one<false, true, true, true, false, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo, stream);
  return count ? launch_one<true, true, false, true, false, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo, stream)
               : launch_one<false, true, false, true, false, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo, stream);
}

}  // namespace cc
