// wf_launch.h -- host-visible launch wrappers of the device kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "wf_internal.cuh"

namespace wf {

struct TailArgs {
  float *f;  // the new state (6*N)
  int nx, ny, nz;
  const SrcDev *src;
  int nsrc;
  const ProbeDev *probe;
  int nprobe;
  long long *step;  // device step counter (read, then incremented)
};

struct FusedArgs {
  GridArgs g;
  int tiles_x, tiles_y, zchunk;
  int has_pml;
  int prof_in_smem;  // every CPML axis has at most 64 slab positions
};

// Tiling of the fused kernel: TY rows per CTA (x width kTileX), z chunk and
// pipeline depth.  Only the instantiated combinations are accepted.
struct FusedConfig {
  int ty, zchunk, stages;
};

// TMA descriptors of one launch: E box, H box, ids box.
struct FusedMaps {
  CUtensorMap e, h, m;
};

cudaError_t launch_split(const GridArgs &g, bool fma, cudaStream_t s);
cudaError_t launch_tail(const TailArgs &t, cudaStream_t s);
cudaError_t launch_soa_to_blocks(const float *soa, float *blk, int nx, int ny, int nz,
                                 cudaStream_t s);
cudaError_t launch_blocks_to_soa(const float *blk, float *soa, int nx, int ny, int nz,
                                 cudaStream_t s);

// TMA boxes the fused kernel needs for a tiling (encoded by the host).
void fused_boxes(int ty, unsigned e_box[4], unsigned h_box[4], unsigned m_box[3]);
bool fused_supported(const FusedConfig &c);
int fused_smem_bytes(const FusedConfig &c);
// Sets the kernels' dynamic shared-memory limit (call outside graph capture).
cudaError_t fused_prepare(const FusedConfig &c);
// Kernel class of work item `item` (tile x, tile y, z chunk): 0 interior,
// 1 / 2 / 4 meets only the x / y / z CPML slab, 7 meets several.
int fused_item_class(const FusedArgs &a, int ty, int item);
constexpr int kFusedClasses[5] = {0, 1, 2, 4, 7};
// Launches the kernel of class `ax` over a device list of n_items items.
cudaError_t launch_fused(const FusedConfig &c, const FusedMaps &m, const FusedArgs &a,
                         const int *items, int n_items, int ax, bool fma, cudaStream_t s);

}  // namespace wf
