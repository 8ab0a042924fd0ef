// Scratch for cc_visibility_static: one file-scope device array per device,
// so that a call allocates nothing. Its address is looked up once per device
// with cudaGetSymbolAddress and cached.
#include <mutex>

#include "kernels.h"

namespace cc {

namespace {

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_address[kMaxDevices] = {};

}  // namespace

cudaError_t static_scratch(int device, void** ptr) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> guard(g_lock);
  if (!g_address[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_address[device] = p;
  }
  *ptr = g_address[device];
  return cudaSuccess;
}

}  // namespace cc
