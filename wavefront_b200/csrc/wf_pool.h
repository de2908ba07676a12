// wf_pool.h -- the per-device cache of the library's device allocations
// (wf_pool.cu): dev_alloc reuses a freed block of the same rounded size or
// calls cudaMalloc; dev_free waits for the device (as cudaFree does) and
// keeps the block for the next allocation.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace wf {

cudaError_t dev_alloc_bytes(void **p, size_t n);
template <typename T>
cudaError_t dev_alloc(T **p, size_t n) {
  return dev_alloc_bytes(reinterpret_cast<void **>(p), n);
}
void dev_free(void *p);
size_t dev_cached_bytes(int dev);
void dev_release(int dev);  // -1: every device
// Destroys the idle stream sets the fused step keeps per device (wf_engine.cu).
void release_idle_stream_sets(int dev);  // -1: every device

}  // namespace wf
