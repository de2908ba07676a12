// wf_closure.h -- kernels of the learned thin-CPML boundary closure (see
// wf_closure.cu): the small 3D conv network's training and inference
// kernels, and the moves of a grid's boundary bands in and out of them.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace wf {

constexpr int kBandDepth = 8;  // cells from each face the closure sees and corrects
constexpr int kBandIn = 10;    // 6 fields + the 4 psi terms of the face's normal axis

struct BandPsi {
  int T, W, pitch;   // graded thickness, slab width, row pitch (x axis)
  float *p;          // [4][cells]
  long long cells;
};

// Raw view of one state buffer of a grid (fields component-major, x fastest).
struct BandGrid {
  int nx, ny, nz;
  long long N;
  float *fields;     // 6*N
  BandPsi psi[3];
};

// All return a cudaError_t value; every launch goes to `stream`.
int nn_conv_fwd(const float *in, const void *w_bf16, const int *face, float *z, float *a, int n,
                int ci, int co, int D, int H, int W, int act, void *stream);
int nn_conv_bwd_data(const float *dz, const void *w_bf16, const int *face, float *din, int n,
                     int ci, int co, int D, int H, int W, void *stream);
int nn_conv_bwd_weight(const float *in, const float *dz, const int *face, float *dw, int n, int ci,
                       int co, int D, int H, int W, int nface, void *stream);
int nn_gelu_bwd(const float *da, const float *z, float *dz, long long m, void *stream);
// The same forward and input-gradient convolutions on the tensor cores
// (tcgen05 implicit GEMMs, wf_conv_tc.cu); nn_conv_fwd / nn_conv_bwd_data
// dispatch to them unless nn_set_tensor_cores(0).
int nn_conv_fwd_tc(const float *in, const void *w_bf16, const int *face, float *z, float *a, int n,
                   int ci, int co, int D, int H, int W, int act, void *stream);
int nn_conv_bwd_data_tc(const float *dz, const void *w_bf16, const int *face, float *din, int n,
                        int ci, int co, int D, int H, int W, void *stream);
// The in-step closure on the tensor cores with its operands prepared once per
// layer (wf_closure_fast.cu): packed band tensors [face][6 arrays][P] of
// 16-byte words (the three bfloat16 parts of 16 channels), a 4-D TMA map over
// each, weights pre-arranged [face][9][2][48][8] bfloat16.
// Layer 1's packed input (the band cells times the gains, unscaled) straight
// from a cubic grid, and per CTA the sum of squares of its E values in
// part[f * closure_fast_parts(H, W) + CTA].
int closure_fast_gather(const BandGrid &g, void *packed, float *part, int H, int W, float ge,
                        float gh, void *stream);
// s[f] = sqrt(sum of face f's partial sums / 3P) + 1e-30 (fixed order)
int closure_fast_rms(const float *part, int H, int W, long long P, float *s, void *stream);
long long closure_fast_parts(int H, int W);  // partial sums per face (the largest axis's)
int closure_fast_pack_weights(const void *w, int co, int ci, void *wp, void *stream);
// One layer.  in_scale (layer 1): the accumulator is divided by in_scale[f]
// (times its reciprocal) before the activation, the network's input
// normalisation applied after the convolution.  last: out_y = FP32 output
// times s[f]; otherwise out_packed = the next layer's packed input.
int closure_fast_conv(const CUtensorMap &tm_in, const void *wp, void *out_packed, float *out_y,
                      const float *s, const float *in_scale, int nout, int D, int H, int W, bool last,
                      void *stream);
unsigned long long closure_fast_timeouts();
void nn_set_tensor_cores(int on);
int nn_tensor_cores();
unsigned long long nn_tc_timeouts();
int nn_mse(const float *y, const float *t, float *dy, float *loss, long long m, void *stream);
int nn_adam(float *w, void *w_bf16, const float *g, float *m1, float *m2, long long n, float lr,
            float b1, float b2, float eps, int t, void *stream);
// X[6][kBandIn][kBandDepth][H][W] from a cubic grid's bands (fields and psi
// scaled by the E / H gains).
int band_gather(const BandGrid &g, float *X, int H, int W, float ge, float gh, void *stream);
// fields += Y[6][6][kBandDepth][H][W] / gain, face by face.
int band_scatter_add(const BandGrid &g, const float *Y, int H, int W, float ge, float gh,
                     void *stream);
// s[f] = RMS of face f's E channels in X[6][C][P]; X[f] *= s[f] (or /=).
int face_rms(const float *X, int C, long long P, float *s, void *stream);
int face_scale(float *X, int C, long long P, const float *s, int divide, void *stream);
// Per face, the factor lam[f] in [0, 1] that keeps the correction Y from
// raising the energy of the band fields X * s[f] (see k_face_guard).
int face_guard(const float *X, int C, const float *Y, long long P, const float *s, float *lam,
               void *stream);
// student = teacher restricted at offset `off` (fields and each axis's psi).
int band_restrict(const BandGrid &teacher, const BandGrid &student, int off, void *stream);

}  // namespace wf
