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

}  // namespace cc
