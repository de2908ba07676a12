// wf_slabs.cu -- the ghost-block copy of the z-slab decomposition.  A slab of
// z planes of one grid's state (the six field components and the x and y
// CPML psi of those planes) is a list of contiguous device segments; one
// launch moves every segment between the grid and a packed buffer, one
// blockIdx.y per segment, float4 accesses (every segment starts on a 16-byte
// boundary and holds a multiple of 4 floats: the planes hold nx*ny floats with
// nx, ny multiples of 8, and the x psi rows are padded to 4 positions).
#include <cuda_runtime.h>

#include "wf_launch.h"

namespace wf {

namespace {

__global__ void k_slab_copy(SlabSegments segs, float *buf, int unpack) {
  const SlabSegment sg = segs.seg[blockIdx.y];
  float4 *dev = reinterpret_cast<float4 *>(sg.dev);
  float4 *pk = reinterpret_cast<float4 *>(buf + sg.off);
  const long long n4 = sg.n / 4;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n4;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (unpack) dev[i] = pk[i];
    else pk[i] = dev[i];
  }
}

}  // namespace

cudaError_t launch_slab_copy(const SlabSegments &segs, float *buf, bool unpack, cudaStream_t s) {
  if (segs.n <= 0) return cudaSuccess;
  long long most = 0;
  for (int i = 0; i < segs.n; ++i) {
    const SlabSegment &sg = segs.seg[i];
    if ((sg.n & 3) || (sg.off & 3) || (reinterpret_cast<uintptr_t>(sg.dev) & 15))
      return cudaErrorInvalidValue;
    if (sg.n > most) most = sg.n;
  }
  if (reinterpret_cast<uintptr_t>(buf) & 15) return cudaErrorInvalidValue;
  // about 4 CTAs of 256 threads per SM over all segments
  const long long want = (most / 4 + 255) / 256;
  const long long cap = (148 * 4 + segs.n - 1) / segs.n;
  const dim3 grid(static_cast<unsigned>(want < cap ? (want > 0 ? want : 1) : cap),
                  static_cast<unsigned>(segs.n));
  k_slab_copy<<<grid, 256, 0, s>>>(segs, buf, unpack ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace wf
