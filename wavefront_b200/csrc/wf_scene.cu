// wf_scene.cu -- the scene voxelizer on the device (Scene::voxelize,
// src/scene.rs:149-230): the material id of every cell written straight into
// the handle's id array, one launch per primitive in file order so a later
// primitive overwrites an earlier one, each launch covering only the
// primitive's bounding box.  The sphere test is the reference's f32
// cell-centre test in its operation order (separate IEEE mul/add), so the ids
// equal the host voxelizer's bit for bit.
#include <cuda_runtime.h>

#include "wf_scene.h"

namespace wf {

namespace {

// op's z range is already clipped to the window; z_lo is the window's first
// plane, so the id of global plane z lands in row plane z - z_lo.
__global__ void k_raster(RasterOp op, uint8_t *ids, int nx, int ny, int pitch, long long z_lo) {
  const long long wx = op.x1 - op.x0, wy = op.y1 - op.y0, wz = op.z1 - op.z0;
  const long long n = wx * wy * wz;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long x = op.x0 + i % wx, y = op.y0 + (i / wx) % wy, z = op.z0 + i / (wx * wy);
    bool in = true;
    if (op.sphere) {
      const float ddx = __fsub_rn(__fadd_rn(static_cast<float>(x), 0.5f), op.cx);
      const float ddy = __fsub_rn(__fadd_rn(static_cast<float>(y), 0.5f), op.cy);
      const float ddz = __fsub_rn(__fadd_rn(static_cast<float>(z), 0.5f), op.cz);
      in = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz)) <= op.r2;
    }
    if (in) ids[((z - z_lo) * ny + y) * pitch + x] = op.id;
  }
  (void)nx;
}

}  // namespace

int launch_voxelize(const std::vector<RasterOp> &ops, uint8_t *ids, int nx, int ny, int nz,
                    int pitch, uint8_t fill, void *stream, int z_lo) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(ids, fill, static_cast<size_t>(pitch) * ny * nz, s);
  if (e != cudaSuccess) return e;
  for (RasterOp op : ops) {
    // keep the planes of the window [z_lo, z_lo + nz)
    if (op.z0 < z_lo) op.z0 = z_lo;
    if (op.z1 > static_cast<long long>(z_lo) + nz) op.z1 = static_cast<long long>(z_lo) + nz;
    if (op.x1 <= op.x0 || op.y1 <= op.y0 || op.z1 <= op.z0) continue;
    const long long n = (op.x1 - op.x0) * (op.y1 - op.y0) * (op.z1 - op.z0);
    const long long want = (n + 255) / 256;
    const unsigned blocks = static_cast<unsigned>(want < 148 * 64 ? want : 148 * 64);
    k_raster<<<blocks, 256, 0, s>>>(op, ids, nx, ny, pitch, z_lo);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace wf
