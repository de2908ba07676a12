// wf_pool.cu -- a per-device cache of the library's device allocations.
//
// Creating a handle allocates its two state buffers, the material ids and
// the CPML psi arrays: gigabytes at 512^3, whose cudaMalloc (page mapping)
// took from 7 to 800 ms on the GPUs this was measured on.  Blocks the
// library frees go into a cache keyed by device and rounded size instead of
// back to CUDA, so the next handle of the same shape (a sweep, a restart, a
// second run in the same process) gets them at once.
//
// Freeing keeps cudaFree's contract: it waits for the whole device first, so
// no kernel still in flight can touch a block that is handed out again.  The
// cache holds at most kCacheCap bytes per device; an allocation that fails
// for lack of memory releases the device's cache to CUDA and tries once more,
// and wf_release_cached_memory releases it on request.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <unordered_map>

#include "../../include/wavefront_gpu.h"
#include "wf_pool.h"

namespace wf {

namespace {

constexpr size_t kCacheCap = size_t(16) << 30;  // bytes cached per device at most

struct Block {
  int dev;
  size_t bytes;  // rounded size
};

std::mutex g_mu;
std::unordered_map<void *, Block> g_live;             // handed out
std::map<int, std::multimap<size_t, void *>> g_free;  // per device: rounded size -> block
std::map<int, size_t> g_cached;                       // bytes in g_free per device

size_t round_size(size_t n) {
  const size_t small = 512, large = size_t(2) << 20;
  const size_t q = n < (size_t(1) << 20) ? small : large;
  return (n + q - 1) / q * q;
}

// Returns the device's cached blocks to CUDA (g_mu held).
void release_locked(int dev) {
  auto it = g_free.find(dev);
  if (it == g_free.end()) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  for (auto &kv : it->second) cudaFree(kv.second);
  if (cur != dev && cur >= 0) cudaSetDevice(cur);
  it->second.clear();
  g_cached[dev] = 0;
}

}  // namespace

cudaError_t dev_alloc_bytes(void **p, size_t n) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const size_t r = round_size(n ? n : 1);
  std::lock_guard<std::mutex> lk(g_mu);
  auto &bins = g_free[dev];
  auto hit = bins.find(r);
  if (hit != bins.end()) {
    *p = hit->second;
    bins.erase(hit);
    g_cached[dev] -= r;
    g_live[*p] = Block{dev, r};
    return cudaSuccess;
  }
  e = cudaMalloc(p, r);
  if (e == cudaErrorMemoryAllocation && g_cached[dev] > 0) {
    cudaGetLastError();  // not sticky: clear it and retry with the cache released
    release_locked(dev);
    e = cudaMalloc(p, r);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  g_live[*p] = Block{dev, r};
  return cudaSuccess;
}

void dev_free(void *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) {  // not ours: hand it to CUDA as before
    cudaFree(p);
    return;
  }
  const Block b = it->second;
  g_live.erase(it);
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != b.dev) cudaSetDevice(b.dev);
  cudaDeviceSynchronize();  // cudaFree's implicit wait: nothing in flight uses p
  if (g_cached[b.dev] + b.bytes <= kCacheCap) {
    g_free[b.dev].emplace(b.bytes, p);
    g_cached[b.dev] += b.bytes;
  } else {
    cudaFree(p);
  }
  if (cur != b.dev && cur >= 0) cudaSetDevice(cur);
}

size_t dev_cached_bytes(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cached.find(dev);
  return it == g_cached.end() ? 0 : it->second;
}

void dev_release(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev >= 0) {
    release_locked(dev);
    return;
  }
  for (auto &kv : g_free) release_locked(kv.first);
}

}  // namespace wf

extern "C" {

wf_status wf_release_cached_memory(int device) {
  wf::dev_release(device);
  wf::release_idle_stream_sets(device);
  return WF_OK;
}

int64_t wf_cached_bytes(int device) { return static_cast<int64_t>(wf::dev_cached_bytes(device)); }

}  // extern "C"
