// wf_closure.cu -- the learned thin-CPML boundary closure (no reference
// counterpart): a per-face 3-layer 3D convolutional network that corrects
// the fields in the 8-cell band next to each face of a grid with a thin
// (4-cell) CPML, so that it behaves like a thick one.
//
// Tensors are "band" tensors [N][C][D=8][H][W]: sample n (a face, or a crop
// of one), channel c, distance d from the outer face (0 = outermost cell),
// and the two tangential coordinates in increasing axis order.  Every conv
// is 3x3x3, stride 1, zero padding, no bias; weights are bfloat16
// [F][Co][Ci][27] (F = 6 faces; sample n uses face[n]) and every sum
// accumulates in FP32.  GELU is the erf form 0.5 z (1 + erf(z / sqrt 2)).
//
// Training runs on these kernels too: forward (keeping pre-activations),
// backward to the input and to the weights, GELU backward, the MSE loss and
// its gradient, and Adam on FP32 master weights with a bfloat16 copy for
// the forward pass.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "wf_band.cuh"
#include "wf_closure.h"

namespace wf {

namespace {

constexpr int kMaxC = 16;       // channels per layer at most
constexpr int kTaps = 27;
constexpr float kInvSqrt2 = 0.70710678118654752f;
constexpr float kInvSqrt2Pi = 0.39894228040143268f;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * kInvSqrt2)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * kInvSqrt2)) + z * kInvSqrt2Pi * expf(-0.5f * z * z);
}

// out[n][co][p] = sum_ci sum_tap w[face[n]][co][ci][tap] * in[n][ci][p + tap]
// (one thread per output voxel, all output channels in registers; the
// sample's weights staged in shared memory as FP32)
__global__ void k_conv_fwd(const float *in, const __nv_bfloat16 *w, const int *face, float *z,
                           float *a, int n, int ci, int co, int D, int H, int W, int act) {
  extern __shared__ float s_w[];  // [co][ci][27] of the block's sample
  const long long P = static_cast<long long>(D) * H * W;
  const int s = blockIdx.y;       // sample
  const int f = face ? face[s] : 0;
  const int nw = co * ci * kTaps;
  for (int i = threadIdx.x; i < nw; i += blockDim.x)
    s_w[i] = __bfloat162float(w[static_cast<long long>(f) * nw + i]);
  __syncthreads();
  const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= P || s >= n) return;
  const int x = static_cast<int>(p % W), y = static_cast<int>((p / W) % H), d = static_cast<int>(p / (static_cast<long long>(W) * H));
  float acc[kMaxC];
#pragma unroll
  for (int o = 0; o < kMaxC; ++o) acc[o] = 0.0f;
  const float *src = in + static_cast<long long>(s) * ci * P;
  for (int c = 0; c < ci; ++c) {
    const float *sc = src + c * P;
    for (int t = 0; t < kTaps; ++t) {
      const int dd = d + t / 9 - 1, yy = y + (t / 3) % 3 - 1, xx = x + t % 3 - 1;
      if (dd < 0 || dd >= D || yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
      const float v = sc[(static_cast<long long>(dd) * H + yy) * W + xx];
#pragma unroll
      for (int o = 0; o < kMaxC; ++o)
        if (o < co) acc[o] = __fmaf_rn(s_w[(o * ci + c) * kTaps + t], v, acc[o]);
    }
  }
  for (int o = 0; o < co; ++o) {
    const long long k = (static_cast<long long>(s) * co + o) * P + p;
    if (z) z[k] = acc[o];
    a[k] = act ? gelu(acc[o]) : acc[o];
  }
}

// The same convolution for the network's output-channel counts (CO = 16, 6),
// blocked for the FMA pipes: a thread computes 4 consecutive voxels of one
// row from 6 staged inputs per (channel, dz, dy), and the weights sit in
// shared memory output-channel fastest ([ci][27][CP], CP = CO rounded up to
// 4, zero padded) so that 128-bit loads feed CO FMAs for each of the 4
// voxels.  Every voxel still sums channel by channel and tap by tap in the
// order of k_conv_fwd, skipping the same out-of-range taps, so the results
// are identical.
template <int CO>
__global__ void __launch_bounds__(128) k_conv_fwd4(const float *in, const __nv_bfloat16 *w,
                                                   const int *face, float *z, float *a, int n,
                                                   int ci, int D, int H, int W, int act) {
  constexpr int CP = (CO + 3) / 4 * 4;
  extern __shared__ float s_w[];  // [ci][27][CP] of the block's sample
  const int s = blockIdx.y;
  const int f = face ? face[s] : 0;
  const int nw = ci * kTaps * CP;
  for (int i = threadIdx.x; i < nw; i += blockDim.x) {
    const int o = i % CP, ct = i / CP;  // ct = c * 27 + t
    const int c = ct / kTaps, t = ct % kTaps;
    s_w[i] = o < CO ? __bfloat162float(w[((static_cast<long long>(f) * CO + o) * ci + c) * kTaps + t])
                    : 0.0f;
  }
  __syncthreads();
  const int QW = (W + 3) / 4;
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= static_cast<long long>(D) * H * QW || s >= n) return;
  const int x0 = static_cast<int>(q % QW) * 4, y = static_cast<int>((q / QW) % H),
            d = static_cast<int>(q / (static_cast<long long>(QW) * H));
  bool ok[6];  // input column x0 - 1 + k inside the row
#pragma unroll
  for (int k = 0; k < 6; ++k) ok[k] = x0 - 1 + k >= 0 && x0 - 1 + k < W;
  float acc[4][CO];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int o = 0; o < CO; ++o) acc[v][o] = 0.0f;
  const long long P = static_cast<long long>(D) * H * W;
  const float *src = in + static_cast<long long>(s) * ci * P;
  for (int c = 0; c < ci; ++c) {
    const float *sc = src + c * P;
    for (int dz = -1; dz <= 1; ++dz) {
      const int dd = d + dz;
      if (dd < 0 || dd >= D) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= H) continue;
        const float *row = sc + (static_cast<long long>(dd) * H + yy) * W + x0 - 1;
        float r[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) r[k] = ok[k] ? __ldg(row + k) : 0.0f;
        const float *wt = s_w + (c * kTaps + (dz + 1) * 9 + (dy + 1) * 3) * CP;
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          float wv[CP];
#pragma unroll
          for (int o4 = 0; o4 < CP / 4; ++o4) {
            const float4 w4 = *reinterpret_cast<const float4 *>(wt + dx * CP + 4 * o4);
            wv[4 * o4] = w4.x;
            wv[4 * o4 + 1] = w4.y;
            wv[4 * o4 + 2] = w4.z;
            wv[4 * o4 + 3] = w4.w;
          }
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            if (!ok[v + dx]) continue;  // the tap k_conv_fwd skips
#pragma unroll
            for (int o = 0; o < CO; ++o) acc[v][o] = __fmaf_rn(wv[o], r[v + dx], acc[v][o]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    if (x0 + v >= W) break;
    const long long p = (static_cast<long long>(d) * H + y) * W + x0 + v;
#pragma unroll
    for (int o = 0; o < CO; ++o) {
      const long long k = (static_cast<long long>(s) * CO + o) * P + p;
      if (z) z[k] = acc[v][o];
      a[k] = act ? gelu(acc[v][o]) : acc[v][o];
    }
  }
}

// din[n][ci][p] = sum_co sum_tap w[co][ci][tap] * dz[n][co][p - tap]
__global__ void k_conv_bwd_data(const float *dz, const __nv_bfloat16 *w, const int *face, float *din,
                                int n, int ci, int co, int D, int H, int W) {
  extern __shared__ float s_w[];
  const long long P = static_cast<long long>(D) * H * W;
  const int s = blockIdx.y;
  const int f = face ? face[s] : 0;
  const int nw = co * ci * kTaps;
  for (int i = threadIdx.x; i < nw; i += blockDim.x)
    s_w[i] = __bfloat162float(w[static_cast<long long>(f) * nw + i]);
  __syncthreads();
  const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= P || s >= n) return;
  const int x = static_cast<int>(p % W), y = static_cast<int>((p / W) % H), d = static_cast<int>(p / (static_cast<long long>(W) * H));
  float acc[kMaxC];
#pragma unroll
  for (int c = 0; c < kMaxC; ++c) acc[c] = 0.0f;
  const float *src = dz + static_cast<long long>(s) * co * P;
  for (int o = 0; o < co; ++o) {
    const float *so = src + o * P;
    for (int t = 0; t < kTaps; ++t) {
      const int dd = d - (t / 9 - 1), yy = y - ((t / 3) % 3 - 1), xx = x - (t % 3 - 1);
      if (dd < 0 || dd >= D || yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
      const float g = so[(static_cast<long long>(dd) * H + yy) * W + xx];
#pragma unroll
      for (int c = 0; c < kMaxC; ++c)
        if (c < ci) acc[c] = __fmaf_rn(s_w[(o * ci + c) * kTaps + t], g, acc[c]);
    }
  }
  for (int c = 0; c < ci; ++c) din[(static_cast<long long>(s) * ci + c) * P + p] = acc[c];
}

// dw[face][co][ci][tap] += sum over samples of that face and voxels p of
// dz[n][co][p] * in[n][ci][p + tap]: one thread per weight entry, the
// samples split over blockIdx.y (partial sums added atomically)
__global__ void k_conv_bwd_weight(const float *in, const float *dz, const int *face, float *dw,
                                  int n, int ci, int co, int D, int H, int W, int nface) {
  const int nw = co * ci * kTaps;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nw) return;
  const int o = e / (ci * kTaps), c = (e / kTaps) % ci, t = e % kTaps;
  const int od = t / 9 - 1, oy = (t / 3) % 3 - 1, ox = t % 3 - 1;
  const long long P = static_cast<long long>(D) * H * W;
  float acc[8];
  for (int f = 0; f < 8; ++f) acc[f] = 0.0f;
  for (int s = blockIdx.y; s < n; s += gridDim.y) {
    const int f = face ? face[s] : 0;
    const float *g = dz + (static_cast<long long>(s) * co + o) * P;
    const float *v = in + (static_cast<long long>(s) * ci + c) * P;
    float sum = 0.0f;
    for (int d = 0; d < D; ++d) {
      const int dd = d + od;
      if (dd < 0 || dd >= D) continue;
      for (int y = 0; y < H; ++y) {
        const int yy = y + oy;
        if (yy < 0 || yy >= H) continue;
        const float *gr = g + (static_cast<long long>(d) * H + y) * W;
        const float *vr = v + (static_cast<long long>(dd) * H + yy) * W;
        for (int x = 0; x < W; ++x) {
          const int xx = x + ox;
          if (xx < 0 || xx >= W) continue;
          sum = __fmaf_rn(gr[x], vr[xx], sum);
        }
      }
    }
    if (f < 8) acc[f] += sum;
  }
  for (int f = 0; f < nface && f < 8; ++f)
    if (acc[f] != 0.0f) atomicAdd(dw + static_cast<long long>(f) * nw + e, acc[f]);
}

__global__ void k_gelu_bwd(const float *da, const float *z, float *dz, long long m) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < m) dz[i] = da[i] * gelu_grad(z[i]);
}

// loss += sum (y - t)^2 / m;  dy = 2 (y - t) / m
__global__ void k_mse(const float *y, const float *t, float *dy, float *loss, long long m) {
  __shared__ float s_sum[256];
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  float d = 0.0f;
  if (i < m) {
    d = y[i] - t[i];
    dy[i] = 2.0f * d / static_cast<float>(m);
  }
  s_sum[threadIdx.x] = d * d;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s_sum[threadIdx.x] += s_sum[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, s_sum[0] / static_cast<float>(m));
}

// Adam (Kingma & Ba) on FP32 master weights; the bfloat16 copy is what the
// forward pass reads.
__global__ void k_adam(float *w, __nv_bfloat16 *wb, const float *g, float *m1, float *m2, long long n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  const float wi = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
}

// ---- band gather / scatter on a grid's state --------------------------------

// X[f][10][8][H][W]: 6 fields scaled by gain (E by ge, H by gh), then the 4
// psi of the face's normal axis (terms of E differences by ge, of H by gh).
// One launch per axis covers its two faces.
template <int AX>
__global__ void __launch_bounds__(256) k_band_gather(BandGrid g, float *X, int H, int W, float ge,
                                                     float gh) {
  using T = BandTile<AX>;
  __shared__ float s[kBandIn][T::TO][T::TA][33];
  const int side = blockIdx.z / T::kZ, sub = blockIdx.z % T::kZ, f = 2 * AX + side;
  const int v0 = blockIdx.x * 32;
  const long long P = static_cast<long long>(kBandDepth) * H * W;
  const BandPsi &ps = g.psi[AX];
#pragma unroll
  for (int j = 0; j < T::kElems / 256; ++j) {  // grid side: a fastest
    const int e = threadIdx.x + 256 * j, al = e % T::TA, vl = (e / T::TA) % 32, ol = e / (T::TA * 32);
    int d, u;
    band_du<AX>(al, ol, blockIdx.y, sub, d, u);
    const int v = v0 + vl;
    if (d < kBandDepth && u < H && v < W) {
      int x, y, z;
      band_cell(g, f, d, u, v, x, y, z);
      const long long cell = (static_cast<long long>(z) * g.ny + y) * g.nx + x;
#pragma unroll
      for (int c = 0; c < 6; ++c) s[c][ol][al][vl] = g.fields[c * g.N + cell] * (c < 3 ? ge : gh);
      const long long k = psi_index(g, AX, x, y, z);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        s[6 + c][ol][al][vl] = k >= 0 ? ps.p[c * ps.cells + k] * (c < 2 ? ge : gh) : 0.0f;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < T::kElems / 256; ++j) {  // band side: v fastest
    const int e = threadIdx.x + 256 * j, vl = e % 32, al = (e / 32) % T::TA, ol = e / (32 * T::TA);
    int d, u;
    band_du<AX>(al, ol, blockIdx.y, sub, d, u);
    const int v = v0 + vl;
    if (d < kBandDepth && u < H && v < W) {
      float *out = X + static_cast<long long>(f) * kBandIn * P + (static_cast<long long>(d) * H + u) * W + v;
#pragma unroll
      for (int c = 0; c < kBandIn; ++c) out[c * P] = s[c][ol][al][vl];
    }
  }
}

// fields += Y / gain over the bands of faces f0 .. f0 + nf - 1 (both faces of
// axis AX in one launch when their bands are disjoint).  The axes go in
// order, so a cell in two bands gets both corrections, edges first by the
// lower face index.
template <int AX>
__global__ void __launch_bounds__(256) k_band_scatter_add(BandGrid g, const float *Y, int H, int W,
                                                          float ge, float gh, int f0) {
  using T = BandTile<AX>;
  __shared__ float s[6][T::TO][T::TA][33];
  const int f = f0 + blockIdx.z / T::kZ, sub = blockIdx.z % T::kZ, v0 = blockIdx.x * 32;
  const long long P = static_cast<long long>(kBandDepth) * H * W;
#pragma unroll
  for (int j = 0; j < T::kElems / 256; ++j) {  // band side: v fastest
    const int e = threadIdx.x + 256 * j, vl = e % 32, al = (e / 32) % T::TA, ol = e / (32 * T::TA);
    int d, u;
    band_du<AX>(al, ol, blockIdx.y, sub, d, u);
    const int v = v0 + vl;
    if (d < kBandDepth && u < H && v < W) {
      const float *in = Y + static_cast<long long>(f) * 6 * P + (static_cast<long long>(d) * H + u) * W + v;
#pragma unroll
      for (int c = 0; c < 6; ++c) s[c][ol][al][vl] = in[c * P];
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < T::kElems / 256; ++j) {  // grid side: a fastest
    const int e = threadIdx.x + 256 * j, al = e % T::TA, vl = (e / T::TA) % 32, ol = e / (T::TA * 32);
    int d, u;
    band_du<AX>(al, ol, blockIdx.y, sub, d, u);
    const int v = v0 + vl;
    if (d < kBandDepth && u < H && v < W) {
      int x, y, z;
      band_cell(g, f, d, u, v, x, y, z);
      const long long cell = (static_cast<long long>(z) * g.ny + y) * g.nx + x;
#pragma unroll
      for (int c = 0; c < 6; ++c) g.fields[c * g.N + cell] += s[c][ol][al][vl] / (c < 3 ? ge : gh);
    }
  }
}

// Student state (nx, ny, nz) = teacher state at offset `off` on every axis:
// the six fields, and on each axis the student's psi slab from the teacher's
// psi at the same physical cells.
__global__ void k_restrict(BandGrid t, BandGrid s, int off) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= s.N) return;
  const int x = static_cast<int>(i % s.nx), y = static_cast<int>((i / s.nx) % s.ny), z = static_cast<int>(i / (static_cast<long long>(s.nx) * s.ny));
  const int X = x + off, Y = y + off, Z = z + off;
  const long long ti = (static_cast<long long>(Z) * t.ny + Y) * t.nx + X;
  for (int c = 0; c < 6; ++c) s.fields[c * s.N + i] = t.fields[c * t.N + ti];
  for (int ax = 0; ax < 3; ++ax) {
    const long long ks = psi_index(s, ax, x, y, z);
    if (ks < 0) continue;
    const long long kt = psi_index(t, ax, X, Y, Z);
    for (int c = 0; c < 4; ++c)
      s.psi[ax].p[c * s.psi[ax].cells + ks] = kt >= 0 ? t.psi[ax].p[c * t.psi[ax].cells + kt] : 0.0f;
  }
}

// s[f] = RMS of the E channels (0..2) of face f's band tensor (a tiny floor
// keeps an all-zero band at zero after scaling).
__global__ void k_face_rms(const float *X, int C, long long P, float *s) {
  __shared__ float s_sum[256];
  const int f = blockIdx.x;
  const float *x = X + static_cast<long long>(f) * C * P;
  float acc = 0.0f;
  for (long long i = threadIdx.x; i < 3 * P; i += blockDim.x) acc += x[i] * x[i];
  s_sum[threadIdx.x] = acc;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s_sum[threadIdx.x] += s_sum[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) s[f] = sqrtf(s_sum[0] / static_cast<float>(3 * P)) + 1e-30f;
}

// Energy guard of a face's correction Y (field units times the gains) on its
// band fields F = X * s[f] (X normalised, channels 0-5 the fields): with
// a = <F, Y> and b = <Y, Y> over the six field channels, the band energy
// changes by 2a + b; if that is positive, lam[f] = clamp(-2a / b, 0, 1) is the
// largest factor that keeps it from growing, else lam[f] = 1.
__global__ void k_face_guard(const float *X, int C, const float *Y, long long P, const float *s,
                             float *lam) {
  __shared__ float s_a[256], s_b[256];
  const int f = blockIdx.x;
  const float *x = X + static_cast<long long>(f) * C * P;
  const float *y = Y + static_cast<long long>(f) * 6 * P;
  float a = 0.0f, b = 0.0f;
  for (long long i = threadIdx.x; i < 6 * P; i += blockDim.x) {
    a += x[i] * y[i];
    b += y[i] * y[i];
  }
  s_a[threadIdx.x] = a;
  s_b[threadIdx.x] = b;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) {
      s_a[threadIdx.x] += s_a[threadIdx.x + k];
      s_b[threadIdx.x] += s_b[threadIdx.x + k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float aa = s_a[0] * s[f], bb = s_b[0];
    float l = 1.0f;
    if (2.0f * aa + bb > 0.0f) l = (aa < 0.0f && bb > 0.0f) ? fminf(1.0f, -2.0f * aa / bb) : 0.0f;
    lam[f] = l;
  }
}

// X[f][c][p] *= s[f] (or / s[f])
__global__ void k_face_scale(float *X, int C, long long P, const float *s, int divide) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (i >= C * P) return;
  const float m = divide ? 1.0f / s[f] : s[f];
  X[static_cast<long long>(f) * C * P + i] *= m;
}

inline unsigned blocks_for(long long n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

// Which kernels run the forward and input-gradient convolutions: the
// tensor-core implicit GEMMs (wf_conv_tc.cu, the default) or the CUDA-core
// kernels above.
static int g_nn_tensor_cores = 1;
void nn_set_tensor_cores(int on) { g_nn_tensor_cores = on != 0; }
int nn_tensor_cores() { return g_nn_tensor_cores; }

int nn_conv_fwd(const float *in, const void *w_bf16, const int *face, float *z, float *a, int n,
                int ci, int co, int D, int H, int W, int act, void *stream) {
  if (ci > kMaxC || co > kMaxC || ci < 1 || co < 1 || n < 1) return cudaErrorInvalidValue;
  if (g_nn_tensor_cores) return nn_conv_fwd_tc(in, w_bf16, face, z, a, n, ci, co, D, H, W, act, stream);
  const long long P = static_cast<long long>(D) * H * W;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const __nv_bfloat16 *wb = static_cast<const __nv_bfloat16 *>(w_bf16);
  if (co == 16 || co == 6) {  // the network's layers: the blocked kernel
    const long long quads = static_cast<long long>(D) * H * ((W + 3) / 4);
    dim3 grid(blocks_for(quads, 128), n);
    const size_t sm = sizeof(float) * ci * kTaps * (co == 16 ? 16 : 8);
    if (co == 16)
      k_conv_fwd4<16><<<grid, 128, sm, st>>>(in, wb, face, z, a, n, ci, D, H, W, act);
    else
      k_conv_fwd4<6><<<grid, 128, sm, st>>>(in, wb, face, z, a, n, ci, D, H, W, act);
    return cudaGetLastError();
  }
  dim3 grid(blocks_for(P, 128), n);
  k_conv_fwd<<<grid, 128, sizeof(float) * co * ci * kTaps, st>>>(in, wb, face, z, a, n, ci, co, D,
                                                                  H, W, act);
  return cudaGetLastError();
}

int nn_conv_bwd_data(const float *dz, const void *w_bf16, const int *face, float *din, int n,
                     int ci, int co, int D, int H, int W, void *stream) {
  if (ci > kMaxC || co > kMaxC || ci < 1 || co < 1 || n < 1) return cudaErrorInvalidValue;
  if (g_nn_tensor_cores) return nn_conv_bwd_data_tc(dz, w_bf16, face, din, n, ci, co, D, H, W, stream);
  const long long P = static_cast<long long>(D) * H * W;
  dim3 grid(blocks_for(P, 128), n);
  k_conv_bwd_data<<<grid, 128, sizeof(float) * co * ci * kTaps, static_cast<cudaStream_t>(stream)>>>(
      dz, static_cast<const __nv_bfloat16 *>(w_bf16), face, din, n, ci, co, D, H, W);
  return cudaGetLastError();
}

int nn_conv_bwd_weight(const float *in, const float *dz, const int *face, float *dw, int n, int ci,
                       int co, int D, int H, int W, int nface, void *stream) {
  if (ci > kMaxC || co > kMaxC || nface > 8 || n < 1) return cudaErrorInvalidValue;
  const int nw = co * ci * kTaps;
  dim3 grid(blocks_for(nw, 128), n < 64 ? n : 64);
  k_conv_bwd_weight<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(in, dz, face, dw, n, ci, co,
                                                                         D, H, W, nface);
  return cudaGetLastError();
}

int nn_gelu_bwd(const float *da, const float *z, float *dz, long long m, void *stream) {
  k_gelu_bwd<<<blocks_for(m, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(da, z, dz, m);
  return cudaGetLastError();
}

int nn_mse(const float *y, const float *t, float *dy, float *loss, long long m, void *stream) {
  k_mse<<<blocks_for(m, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(y, t, dy, loss, m);
  return cudaGetLastError();
}

int nn_adam(float *w, void *w_bf16, const float *g, float *m1, float *m2, long long n, float lr,
            float b1, float b2, float eps, int t, void *stream) {
  const float c1 = 1.0f - powf(b1, static_cast<float>(t)), c2 = 1.0f - powf(b2, static_cast<float>(t));
  k_adam<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, static_cast<__nv_bfloat16 *>(w_bf16), g, m1, m2, n, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

int band_gather(const BandGrid &g, float *X, int H, int W, float ge, float gh, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned bx = blocks_for(W, 32);
  k_band_gather<0><<<dim3(bx, blocks_for(H, BandTile<0>::TO), 2 * BandTile<0>::kZ), 256, 0, st>>>(
      g, X, H, W, ge, gh);
  k_band_gather<1><<<dim3(bx, blocks_for(H, 32), 2 * BandTile<1>::kZ), 256, 0, st>>>(g, X, H, W, ge, gh);
  k_band_gather<2><<<dim3(bx, blocks_for(H, 32), 2 * BandTile<2>::kZ), 256, 0, st>>>(g, X, H, W, ge, gh);
  return cudaGetLastError();
}

int band_scatter_add(const BandGrid &g, const float *Y, int H, int W, float ge, float gh,
                     void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned bx = blocks_for(W, 32);
  const int extent[3] = {g.nx, g.ny, g.nz};
  for (int ax = 0; ax < 3; ++ax) {
    // the two faces' bands are disjoint when the axis holds two band depths
    const int nf = extent[ax] >= 2 * kBandDepth ? 2 : 1;
    for (int f = 2 * ax; f < 2 * ax + 2; f += nf) {
      if (ax == 0)
        k_band_scatter_add<0><<<dim3(bx, blocks_for(H, BandTile<0>::TO), nf * BandTile<0>::kZ), 256, 0,
                                st>>>(g, Y, H, W, ge, gh, f);
      else if (ax == 1)
        k_band_scatter_add<1><<<dim3(bx, blocks_for(H, 32), nf * BandTile<1>::kZ), 256, 0, st>>>(
            g, Y, H, W, ge, gh, f);
      else
        k_band_scatter_add<2><<<dim3(bx, blocks_for(H, 32), nf * BandTile<2>::kZ), 256, 0, st>>>(
            g, Y, H, W, ge, gh, f);
    }
  }
  return cudaGetLastError();
}

int face_rms(const float *X, int C, long long P, float *s, void *stream) {
  k_face_rms<<<6, 256, 0, static_cast<cudaStream_t>(stream)>>>(X, C, P, s);
  return cudaGetLastError();
}

int face_guard(const float *X, int C, const float *Y, long long P, const float *s, float *lam,
               void *stream) {
  k_face_guard<<<6, 256, 0, static_cast<cudaStream_t>(stream)>>>(X, C, Y, P, s, lam);
  return cudaGetLastError();
}

int face_scale(float *X, int C, long long P, const float *s, int divide, void *stream) {
  k_face_scale<<<dim3(blocks_for(C * P, 256), 6), 256, 0, static_cast<cudaStream_t>(stream)>>>(X, C, P, s, divide);
  return cudaGetLastError();
}

int band_restrict(const BandGrid &teacher, const BandGrid &student, int off, void *stream) {
  k_restrict<<<blocks_for(student.N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(teacher, student, off);
  return cudaGetLastError();
}

}  // namespace wf
