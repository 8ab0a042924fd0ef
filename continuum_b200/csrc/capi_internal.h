// Host-side state shared by the C ABI's files: contexts, scenes, growable
// device buffers and the error helpers.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/continuum_cuda.h"
#include "bvh.h"
#include "kernels.h"

namespace cc_host {

// Records the calling thread's error message and returns `code`.
int fail(int code, const std::string& msg);
// The same for a failed CUDA call (CC_ERR_OOM for an allocation failure).
int cuda_fail(cudaError_t e, const char* what);

#define CC_CUDA(call, what)                      \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// A device allocation that grows on demand and is kept for reuse.
struct DevBuf {
  void* ptr = nullptr;
  size_t size = 0;
  cudaError_t reserve(size_t bytes) {
    if (bytes <= size) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    size = 0;
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) size = want;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    size = 0;
  }
};

int set_device(cc_context* ctx);

// cc_visibility's body (capi.cu): `sky` makes the cones sky faces (0: light
// cones); `cones` / `cones_count` (device, nullable) walk only listed cones.
int visibility_impl(cc_context* ctx, const cc_scene* scene, const float* receivers, uint64_t npoints,
                    const float* lights, uint32_t nlights, const cc_options* opt, const cc_outputs* out,
                    void* stream, uint32_t sky, const uint32_t* cones, const uint32_t* cones_count);

// The scene's prefiltered coverage samples on the device (built and uploaded
// on first use; capi.cu). The scene's device is current.
int scene_coverage(cc_scene* s);

}  // namespace cc_host

struct cc_context {
  using DevBuf = cc_host::DevBuf;
  int device = 0;
  int sm_count = 148;
  uint64_t split_chunk = cc::kSplitChunk;  // cones a split chunk holds at most
  cudaStream_t stream = nullptr;
  DevBuf receivers, lights, full, any, partial, irradiance, fraction, work;
  DevBuf sky_sum;   // sky irradiance per receiver before its download
  DevBuf redo;      // redo list
  DevBuf order;     // walk order of the points
  DevBuf light_order;  // the split path's light order
  DevBuf sort_scratch;
  // Moving frames' scratch, kept between frames: the movers' transforms, the
  // stale-cone tables, and the update's cone order, flags, list and count.
  DevBuf move_xforms, stale_tables, upd_perm, upd_flags, upd_list, upd_count, upd_order, upd_temp;
  DevBuf records;   // the split path's cone records, one chunk
  DevBuf masks;     // the split path's masks (64 floats a slot), one chunk
  DevBuf counters;  // [redo count, error word]
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Host-buffer calls download FULL/ANY on copy_stream once the walk is done
  // (walked), while the integration runs; copied marks that download's end.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t walked = nullptr, copied = nullptr;
  // Kernel timing: three events per visibility call (before the packet pass,
  // between the passes, after the solo pass) in a ring of kTimingRing calls.
  static constexpr int kTimingRing = 256;
  std::vector<cudaEvent_t> marks;  // 3 * kTimingRing
  int timed_first = 0;             // oldest unread call in the ring
  int timed_count = 0;             // unread calls
};

struct cc_scene {
  cc_context* ctx = nullptr;
  cc::FlatScene flat;  // host copy of the reference layouts
  float4* tris = nullptr;
  uint4* meshes = nullptr;
  float4* nodes = nullptr;
  uint32_t* items = nullptr;
  float4* blas = nullptr;
  float4* xforms = nullptr;  // instanced scenes: 4 per transform
  // Prefiltered cones' coverage samples, computed and uploaded on first use.
  float* blas_cov = nullptr;
  float* obj_cov = nullptr;
  bool coverage_ready = false;
  // CC_BACK_FACING: each triangle's slot on the device, uploaded on first use.
  uint32_t* tri_slot = nullptr;
  uint64_t bytes = 0;
  cc::DevScene dev() const {
    cc::DevScene s;
    s.tris = tris;
    s.meshes = meshes;
    s.nodes = nodes;
    s.items = items;
    s.blas = blas;
    s.nmeshes = flat.nmeshes;
    s.xforms = xforms;
    s.blas_cov = blas_cov;
    s.obj_cov = obj_cov;
    return s;
  }
};

