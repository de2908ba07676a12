// wf_launch.h -- host-visible launch wrappers of the device kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "wf_internal.cuh"

namespace wf {

struct TailArgs {
  float *f;  // the new state (6*N; 16-bit elements when prec != kPrecF32)
  int nx, ny, nz;
  const SrcDev *src;
  int nsrc;
  const ProbeDev *probe;
  int nprobe;
  long long *step;  // device step counter (read, then incremented)
  // 16-bit storage: shifts of the new state (sources and probes decode and
  // re-encode with them), its slab maxima, and the shifts the next step
  // writes with (computed here, into the buffer the step just read)
  int prec;
  const int *shift_f;
  unsigned *slab_max;
  int *shift_next;
  int nslab, periodic_z;
  float kh, ke;  // 8 * max |Db|, 8 * max |Cb| over the material table
  unsigned long long *ovf;
  int *err;  // device error word (bounds-checked builds latch kErrBounds)
};

struct FusedArgs {
  GridArgs g;
  int tiles_x, tiles_y, zchunk;
  // wide tiles cover x in [x_lo, x_hi): the whole grid, or [16, nx-16) when
  // the x-CPML slabs run as column tiles (tiles_x = 2 in a column launch:
  // the low and the high edge)
  int x_lo, x_hi;
  int has_pml;
  int prof_in_smem;  // every CPML axis has at most 64 slab positions
  int test_extra_tx;  // testing aid: bytes stage 0 expects beyond its copies (0 normally)
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

// One grid of a batched step, in device memory (64-byte aligned for the
// tensor maps): per parity of the state read, its TMA maps (E, H, ids) and
// fused-kernel arguments.
struct BatchScene {
  CUtensorMap maps[2][3];
  FusedArgs args[2];
};

cudaError_t launch_split(const GridArgs &g, bool fma, cudaStream_t s);
cudaError_t launch_tail(const TailArgs &t, cudaStream_t s);
cudaError_t launch_soa_to_blocks(const float *soa, float *blk, int nx, int ny, int nz,
                                 cudaStream_t s);
cudaError_t launch_blocks_to_soa(const float *blk, float *soa, int nx, int ny, int nz,
                                 cudaStream_t s);

// TMA boxes the fused kernel needs for a tiling and storage (encoded by the host).
void fused_boxes(int ty, int prec, unsigned e_box[4], unsigned h_box[4], unsigned m_box[3]);
bool fused_supported(const FusedConfig &c, int prec);
int fused_smem_bytes(const FusedConfig &c, int prec);
// Sets the kernels' dynamic shared-memory limit (call outside graph capture).
cudaError_t fused_prepare(const FusedConfig &c, int prec);
// Kernel class of work item `item` (tile x, tile y, z chunk): the mask of
// the CPML slabs it meets (1 x, 2 y, 4 z; 0 interior).
int fused_item_class(const FusedArgs &a, int ty, int item);
constexpr int kFusedClassCount = 8;
// x-CPML column tiles (16 cells wide, 32 rows; every lane holds graded
// cells): boxes, class of an item (always has the x bit: 1, 3, 5 or 7),
// kernel preparation and launch (any storage; FMA only for FP32).
constexpr int kColWidth = 16, kColTileRows = 32;
constexpr int kColClassCount = 4;  // classes 1, 3, 5, 7
void fused_col_boxes(int prec, unsigned e_box[4], unsigned h_box[4], unsigned m_box[3]);
int fused_col_item_class(const FusedArgs &a, int item);
cudaError_t fused_col_prepare(int prec);
cudaError_t launch_fused_col(const FusedMaps &m, const FusedArgs &a, const int *items,
                             int n_items, int ax, bool fma, cudaStream_t s);
// Launches the kernel of class `ax` over a device list of n_items items.
cudaError_t launch_fused(const FusedConfig &c, const FusedMaps &m, const FusedArgs &a,
                         const int *items, int n_items, int ax, bool fma, cudaStream_t s);
// Batched step (FP32 storage, exact arithmetic): one persistent launch per
// CPML class `ax` of `ctas` CTAs that take (grid, item) pairs of that class
// from *counter (zeroed by the caller before each launch) until n_items are
// done.
cudaError_t fused_batch_prepare(const FusedConfig &c);
cudaError_t launch_fused_batch(const FusedConfig &c, const BatchScene *scenes, const int2 *items,
                               int n_items, int *counter, int parity, int ctas, int ax,
                               cudaStream_t s);
// CTAs per SM the batched kernel of a tiling and class fits (for sizing `ctas`).
int fused_batch_ctas_per_sm(const FusedConfig &c, int ax);
// The narrow batched step (tile_rows == kColTileRows): every grid cut into
// kColWidth x kColTileRows tiles, all items in one persistent launch of the
// all-axes body.
bool fused_batch_narrow(const FusedConfig &c);
cudaError_t fused_batch_narrow_prepare();
cudaError_t launch_fused_batch_narrow(const BatchScene *scenes, const int2 *items, int n_items,
                                      int *counter, int parity, int ctas, cudaStream_t s);
int fused_batch_narrow_ctas_per_sm();
// The step tail of n grids at once: one CTA per grid, t[i] as for launch_tail.
cudaError_t launch_tail_batch(const TailArgs *t, int n, cudaStream_t s);

// 16-bit storage (wf_fused16.cu)
bool fused16_supported(const FusedConfig &c);
int fused16_smem_bytes(const FusedConfig &c, int prec);
cudaError_t fused16_prepare(const FusedConfig &c, int prec);
cudaError_t fused16_launch(const FusedConfig &c, const FusedMaps &m, const FusedArgs &a,
                           const int *items, int n_items, int ax, cudaStream_t s);
cudaError_t fused16_col_prepare(int prec);
cudaError_t fused16_col_launch(const FusedMaps &m, const FusedArgs &a, const int *items,
                               int n_items, int ax, cudaStream_t s);

// 16-bit storage helpers (wf_split.cu).
// Encodes FP32 values `in` (6*N) as the 16-bit state `out`: per slab and
// kind the shift of the slab's own maximum (written to `shift`); leaves the
// maxima of the encoded state in slab_max.
cudaError_t launch_encode_state(const float *in, void *out, int prec, int nx, int ny, int nz,
                                int *shift, unsigned *slab_max, unsigned long long *ovf,
                                cudaStream_t s);
cudaError_t launch_decode_state(const void *in, float *out, int prec, int nx, int ny, int nz,
                                const int *shift, cudaStream_t s);
// Slab maxima (bits of the largest decoded magnitude per slab and kind) of a
// 16-bit state, into slab_max.
cudaError_t launch_state_max(const void *in, int prec, int nx, int ny, int nz, const int *shift,
                             unsigned *slab_max, cudaStream_t s);
// Write shifts of the step with index `next` into t.shift_next (see k_tail).
cudaError_t launch_next_shifts(const TailArgs &t, long long next, cudaStream_t s);

// z-slab ghost blocks: contiguous device segments of a grid's state and their
// offsets in a packed buffer (floats; all multiples of 4, 16-byte aligned).
struct SlabSegment {
  float *dev;
  long long off, n;
};
constexpr int kSlabMaxSegments = 14;  // 6 field components + 4 x psi + 4 y psi
struct SlabSegments {
  SlabSegment seg[kSlabMaxSegments];
  int n;
};
// One launch: every segment copied into the packed buffer, or out of it.
cudaError_t launch_slab_copy(const SlabSegments &segs, float *buf, bool unpack, cudaStream_t s);

}  // namespace wf
