// wf_fused.cu -- FP32-storage instantiations of the fused step kernel
// (wf_fused_impl.cuh) and the host-side dispatch of every storage type:
// work-item classes, TMA box shapes, tiling support and launches.  The 16-bit
// instantiations live in wf_fused16.cu so the two compile in parallel.
#include "wf_fused_impl.cuh"

namespace wf {

// (tile rows, stages) combinations instantiated for FP32 storage
#define WF_FUSED_CONFIGS(X) X(4, 3) X(4, 4) X(8, 3) X(8, 4) X(16, 3)

void fused_boxes(int ty, int prec, unsigned e_box[4], unsigned h_box[4], unsigned m_box[3]) {
  const unsigned pad = prec == kPrecF32 ? 4u : 8u;  // 16 bytes of x
  e_box[0] = kTileX + 2 * pad; e_box[1] = ty + 2; e_box[2] = 1; e_box[3] = 3;
  h_box[0] = kTileX + pad; h_box[1] = ty + 1; h_box[2] = 1; h_box[3] = 3;
  m_box[0] = kTileX + 16; m_box[1] = ty + 1; m_box[2] = 1;
}

static int item_class(const FusedArgs &a, int ty, int item, bool col) {
  if (!a.has_pml) return 0;
  const int txi = item % a.tiles_x;
  const int tyi = (item / a.tiles_x) % a.tiles_y;
  const int zc = item / (a.tiles_x * a.tiles_y);
  const int x0 = col ? (txi == 0 ? 0 : a.g.nx - kColWidth) : a.x_lo + txi * kTileX;
  const int y0 = tyi * ty;
  const int k0 = zc * a.zchunk, k1 = std::min(k0 + a.zchunk, a.g.nz);
  const PmlAxis &X = a.g.pml[0], &Y = a.g.pml[1], &Z = a.g.pml[2];
  const int xh = col ? x0 + kColWidth - 1 : std::min(x0 + kTileX, a.x_hi) - 1;
  const int yh = std::min(y0 + ty, a.g.ny) - 1;
  // an axis's CPML code is needed if the CTA's cells, its -x/-y halo or its
  // warm-up plane (k0-1) meet that axis's graded slab
  int mask = 0;
  if (X.T > 0 && (x0 - 1 < X.T || xh >= a.g.nx - X.T)) mask |= 1;
  if (Y.T > 0 && (y0 - 1 < Y.T || yh >= a.g.ny - Y.T)) mask |= 2;
  if (Z.T > 0 && (k0 - 1 < Z.T || k1 - 1 >= a.g.nz - Z.T)) mask |= 4;
  return mask;
}

int fused_item_class(const FusedArgs &a, int ty, int item) { return item_class(a, ty, item, false); }

int fused_col_item_class(const FusedArgs &a, int item) {
  return item_class(a, kColTileRows, item, true) | 1;
}

void fused_col_boxes(int prec, unsigned e_box[4], unsigned h_box[4], unsigned m_box[3]) {
  const unsigned pad = prec == kPrecF32 ? 4u : 8u;  // 16 bytes of x
  e_box[0] = kColWidth + 2 * pad; e_box[1] = kColTileRows + 2; e_box[2] = 1; e_box[3] = 3;
  h_box[0] = kColWidth + pad; h_box[1] = kColTileRows + 1; h_box[2] = 1; h_box[3] = 3;
  m_box[0] = kColWidth + 32; m_box[1] = kColTileRows + 1; m_box[2] = 1;  // see Layout::MW
}

static_assert(kColWidth == 4 * kColLanes && kColTileRows == kColRows, "column tile shape");

cudaError_t fused_col_prepare(int prec) {
  if (prec != kPrecF32) return fused16_col_prepare(prec);
  cudaError_t e = col_prepare_t<false, float>();
  return e != cudaSuccess ? e : col_prepare_t<true, float>();
}

cudaError_t launch_fused_col(const FusedMaps &m, const FusedArgs &a, const int *items,
                             int n_items, int ax, bool fma, cudaStream_t s) {
  if (a.g.prec != kPrecF32) {
    if (fma) return cudaErrorInvalidValue;  // 16-bit storage runs the exact arithmetic
    return fused16_col_launch(m, a, items, n_items, ax, s);
  }
  return fma ? col_launch_t<true, float>(m, a, items, n_items, ax, s)
             : col_launch_t<false, float>(m, a, items, n_items, ax, s);
}

bool fused_supported(const FusedConfig &c, int prec) {
  if (c.zchunk < 1) return false;
  if (prec != kPrecF32) return fused16_supported(c);
#define X(T, S_) if (c.ty == T && c.stages == S_) return true;
  WF_FUSED_CONFIGS(X)
#undef X
  return false;
}

int fused_smem_bytes(const FusedConfig &c, int prec) {
  if (prec != kPrecF32) return fused16_smem_bytes(c, prec);
#define X(T, S_) if (c.ty == T && c.stages == S_) return Layout<T, S_, float>::BYTES;
  WF_FUSED_CONFIGS(X)
#undef X
  return -1;
}

cudaError_t fused_prepare(const FusedConfig &c, int prec) {
  if (prec != kPrecF32) return fused16_prepare(c, prec);
#define X(T, S_)                                                    \
  if (c.ty == T && c.stages == S_) {                                \
    cudaError_t e = prepare_t<T, S_, false, float>();               \
    return e != cudaSuccess ? e : prepare_t<T, S_, true, float>();  \
  }
  WF_FUSED_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t fused_batch_prepare(const FusedConfig &c) {
#define X(T, S_) if (c.ty == T && c.stages == S_) return batch_prepare_t<T, S_>();
  WF_FUSED_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t launch_fused_batch(const FusedConfig &c, const BatchScene *scenes, const int2 *items,
                               int n_items, int *counter, int parity, int ctas, int ax,
                               cudaStream_t s) {
#define X(T, S_)                                                                         \
  if (c.ty == T && c.stages == S_)                                                      \
    return batch_launch_t<T, S_>(scenes, items, n_items, counter, parity, ctas, ax, s);
  WF_FUSED_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

bool fused_batch_narrow(const FusedConfig &c) {
  return c.ty == kColTileRows && c.stages == kColStages && c.zchunk >= 1;
}

cudaError_t fused_batch_narrow_prepare() { return batch_narrow_prepare_t(); }

cudaError_t launch_fused_batch_narrow(const BatchScene *scenes, const int2 *items, int n_items,
                                      int *counter, int parity, int ctas, cudaStream_t s) {
  return batch_narrow_launch_t(scenes, items, n_items, counter, parity, ctas, s);
}

int fused_batch_narrow_ctas_per_sm() { return batch_narrow_ctas_per_sm_t(); }

int fused_batch_ctas_per_sm(const FusedConfig &c, int ax) {
#define X(T, S_) if (c.ty == T && c.stages == S_) return batch_ctas_per_sm_t<T, S_>(ax);
  WF_FUSED_CONFIGS(X)
#undef X
  return 0;
}

cudaError_t launch_fused(const FusedConfig &c, const FusedMaps &m, const FusedArgs &a,
                         const int *items, int n_items, int ax, bool fma, cudaStream_t s) {
  if (a.g.prec != kPrecF32) {
    if (fma) return cudaErrorInvalidValue;  // 16-bit storage runs the exact arithmetic
    return fused16_launch(c, m, a, items, n_items, ax, s);
  }
#define X(T, S_)                                                            \
  if (c.ty == T && c.stages == S_)                                         \
    return fma ? launch_t<T, S_, true, float>(m, a, items, n_items, ax, s) \
               : launch_t<T, S_, false, float>(m, a, items, n_items, ax, s);
  WF_FUSED_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

}  // namespace wf
