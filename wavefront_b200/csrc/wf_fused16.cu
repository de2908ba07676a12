// wf_fused16.cu -- 16-bit-storage instantiations of the fused step kernel
// (wf_fused_impl.cuh): binary16 and bfloat16 fields with per-slab
// power-of-two scales, FP32 arithmetic in the reference's exact operation
// order (no FMA variant).
#include "wf_fused_impl.cuh"

namespace wf {

// (tile rows, stages) combinations instantiated for 16-bit storage
#define WF_FUSED16_CONFIGS(X) X(4, 3) X(4, 4) X(4, 5) X(4, 6) X(8, 3) X(8, 4)

bool fused16_supported(const FusedConfig &c) {
#define X(T, S_) if (c.ty == T && c.stages == S_) return true;
  WF_FUSED16_CONFIGS(X)
#undef X
  return false;
}

int fused16_smem_bytes(const FusedConfig &c, int prec) {
  (void)prec;  // both 16-bit types have the same layout
#define X(T, S_) if (c.ty == T && c.stages == S_) return Layout<T, S_, __half>::BYTES;
  WF_FUSED16_CONFIGS(X)
#undef X
  return -1;
}

cudaError_t fused16_prepare(const FusedConfig &c, int prec) {
#define X(T, S_)                                                 \
  if (c.ty == T && c.stages == S_)                               \
    return prec == kPrecF16 ? prepare_t<T, S_, false, __half>()  \
                            : prepare_t<T, S_, false, __nv_bfloat16>();
  WF_FUSED16_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t fused16_launch(const FusedConfig &c, const FusedMaps &m, const FusedArgs &a,
                           const int *items, int n_items, int ax, cudaStream_t s) {
#define X(T, S_)                                                              \
  if (c.ty == T && c.stages == S_)                                           \
    return a.g.prec == kPrecF16                                              \
               ? launch_t<T, S_, false, __half>(m, a, items, n_items, ax, s) \
               : launch_t<T, S_, false, __nv_bfloat16>(m, a, items, n_items, ax, s);
  WF_FUSED16_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t fused16_col_prepare(int prec) {
  return prec == kPrecF16 ? col_prepare_t<false, __half>() : col_prepare_t<false, __nv_bfloat16>();
}

cudaError_t fused16_col_launch(const FusedMaps &m, const FusedArgs &a, const int *items,
                               int n_items, int ax, cudaStream_t s) {
  return a.g.prec == kPrecF16 ? col_launch_t<false, __half>(m, a, items, n_items, ax, s)
                              : col_launch_t<false, __nv_bfloat16>(m, a, items, n_items, ax, s);
}

}  // namespace wf
