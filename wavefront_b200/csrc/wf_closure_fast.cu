// wf_closure_fast.cu -- the in-step closure network on the tensor cores with
// its operands prepared once per layer.
//
// The closure runs three 3x3x3 convolutions (10 -> 16 -> 16 -> 6 channels)
// over the six face bands after every step.  k_conv_tc (wf_conv_tc.cu) takes
// FP32 tensors: each CTA loads its halo'd tile voxel by voxel and splits every
// value into three bfloat16 parts, 3.2 times per voxel because of the halos,
// and stages its face's weights, which leaves the tensor pipe idle most of the
// time.  Here the band tensors are kept in the operand layout itself:
//
//   packed [face][array][d][y][x][8 channels] bfloat16, 16 bytes a voxel per
//   array, array = 2 * part + channel half (six arrays: three bfloat16 parts
//   of the FP32 value, channels 0-7 and 8-15)
//
// so that a CTA brings its whole A tile (4 planes x 6 rows x 32 columns of all
// six arrays) into shared memory with one 5-D TMA box, whose zero fill
// outside the band is the convolution's zero padding, and its face's
// pre-arranged weights with one bulk copy.  The epilogue applies GELU and
// writes the next layer's input already split; the last layer writes FP32
// times the face's RMS.  The operands, the MMA sequence and the FP32
// accumulation are those of k_conv_tc, so the results equal the FP32 path's.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "wf_closure.h"
#include "wf_internal.cuh"

namespace wf {

namespace {

constexpr int kFDT = 2, kFPlanes = 4, kFRows = 6, kFCols = 32, kFOutRows = 4, kFOutCols = 30;
constexpr int kFVox = kFPlanes * kFRows * kFCols;       // 768 voxels a tile
constexpr int kFArr = kFVox * 16;                        // bytes of one array of the tile
constexpr int kFABytes = 6 * kFArr;                      // the TMA box: 73 728 bytes
constexpr int kFAOff = 128;                              // guard before the box
constexpr int kFBOff = kFAOff + kFABytes + 128;          // weights, after a guard
constexpr int kFBBytes = 27 * 512;
constexpr int kFBarOff = kFBOff + kFBBytes;
constexpr int kFSmem = kFBarOff + 16 + 128;              // + base alignment slack
constexpr int kFThreads = 256;
constexpr int kFTmemCols = 32;

__device__ unsigned long long g_fast_timeouts;

constexpr float kInvSqrt2f = 0.70710678118654752f;
__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * kInvSqrt2f)); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16, BF16 A and B (K-major), FP32 D, M = 128, N = 16
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *tm, int c0, int c1,
                                            int c2, int c3, int c4, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
      : "memory");
}

// The three bfloat16 parts of 16 FP32 values, as six 16-byte words:
// out[2 * part + half] holds channels 8 * half .. 8 * half + 7 of `part`.
__device__ __forceinline__ void split16(float v[16], uint4 out[6]) {
#pragma unroll
  for (int part = 0; part < 3; ++part) {
    uint32_t q[8];
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
      const __nv_bfloat16 h0 = __float2bfloat16_rn(v[c]), h1 = __float2bfloat16_rn(v[c + 1]);
      q[c / 2] = static_cast<uint32_t>(__bfloat16_as_ushort(h0)) |
                 (static_cast<uint32_t>(__bfloat16_as_ushort(h1)) << 16);
      v[c] -= __bfloat162float(h0);
      v[c + 1] -= __bfloat162float(h1);
    }
    out[2 * part] = make_uint4(q[0], q[1], q[2], q[3]);
    out[2 * part + 1] = make_uint4(q[4], q[5], q[6], q[7]);
  }
}

}  // namespace

namespace {

constexpr int kRmsBlocks = 148;  // partial sums per face

// Sum of squares of the E channels (0..2) of each face band X[6][C][P]: a
// fixed grid of partial sums (deterministic order), then one CTA per face
// folds them: s[f] = sqrt(sum / 3P) + 1e-30, as face_rms computes it.
__global__ void k_face_sumsq(const float *X, int C, long long P, float *part) {
  __shared__ float s_sum[256];
  const int f = blockIdx.y;
  const float *x = X + static_cast<long long>(f) * C * P;
  float acc = 0.0f;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < 3 * P;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    acc += x[i] * x[i];
  s_sum[threadIdx.x] = acc;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s_sum[threadIdx.x] += s_sum[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[f * gridDim.x + blockIdx.x] = s_sum[0];
}

__global__ void k_face_rms_fold(const float *part, int nb, long long P, float *s) {
  __shared__ float s_sum[256];
  const int f = blockIdx.x;
  float acc = 0.0f;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += part[f * nb + i];
  s_sum[threadIdx.x] = acc;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s_sum[threadIdx.x] += s_sum[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) s[f] = sqrtf(s_sum[0] / static_cast<float>(3 * P)) + 1e-30f;
}

// packed[f][6][P] (16-byte words) from X[f][C][P] / s[f]; channels C..15 zero
__global__ void k_pack_band(const float *X, int C, long long P, const float *s, uint4 *packed) {
  const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (p >= P) return;
  const float *x = X + static_cast<long long>(f) * C * P + p;
  float v[16];
  const float m = 1.0f / s[f];  // as face_scale divides: times the reciprocal
#pragma unroll
  for (int c = 0; c < 16; ++c) v[c] = c < C ? x[c * P] * m : 0.0f;
  uint4 w[6];
  split16(v, w);
  uint4 *o = packed + static_cast<long long>(f) * 6 * P + p;
#pragma unroll
  for (int q = 0; q < 6; ++q) o[q * P] = w[q];
}

// Wp[f][27][half][n 16][k 8] bf16 from W[f][co][ci][27] (zero padded)
__global__ void k_pack_weights(const __nv_bfloat16 *w, int co, int ci, __nv_bfloat16 *wp) {
  const int f = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 27 * 256; i += gridDim.x * blockDim.x) {
    const int t = i >> 8, e = i & 255;
    const int half = e >> 7, n = (e >> 3) & 15, k = half * 8 + (e & 7);
    __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
    if (n < co && k < ci) v = w[((static_cast<long long>(f) * co + n) * ci + k) * 27 + t];
    wp[static_cast<long long>(f) * 27 * 256 + i] = v;
  }
}

}  // namespace

namespace {

// One layer of the in-step closure on face f's band: A tile by one TMA box of
// the packed input, the face's packed weights by one bulk copy, 2 planes x 27
// taps x 3 parts MMAs into tensor memory, then the epilogue: GELU and the
// next layer's packed input, or (LAST) the FP32 correction times s[f].
template <bool LAST>
__global__ void __launch_bounds__(kFThreads, 2)
    k_conv_fast(const __grid_constant__ CUtensorMap tm_in, const __nv_bfloat16 *wp,
                uint4 *out_packed, float *out_y, const float *s, int nout, int D, int H, int W,
                int ndt) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int f = blockIdx.z / ndt, dt = blockIdx.z % ndt;
  const int x0 = blockIdx.x * kFOutCols, y0 = blockIdx.y * kFOutRows, dp0 = dt * kFDT;
  const long long HW = static_cast<long long>(H) * W, P = HW * D;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t a0 = sbase + kFAOff, b0 = sbase + kFBOff;
  const uint32_t bar_in = sbase + kFBarOff, bar_mma = bar_in + 8;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(kFTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar_in, 1);
    mbar_init(bar_mma, 1);
    mbar_fence_init();
    mbar_expect_tx(bar_in, kFABytes + kFBBytes);
    tma_load_5d(a0, &tm_in, 0, x0 - 1, y0 - 1, dp0 - 1, f * 6, bar_in);
    bulk_load(b0, wp + static_cast<long long>(f) * 27 * 256, kFBBytes, bar_in);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int nplanes = min(kFDT, D - dp0);
  bool ok = mbar_wait(bar_in, 0);
  if (tid == 0 && ok) {
    for (int p = 0; p < nplanes; ++p) {
      const int f0 = ((p + 1) * kFRows + 1) * kFCols;  // first output row of plane p
      for (int t = 0; t < 27; ++t) {
        const int off = (t / 9 - 1) * kFRows * kFCols + ((t / 3) % 3 - 1) * kFCols + (t % 3 - 1);
        const uint64_t bd = smem_desc(b0 + t * 512, 256, 128);
#pragma unroll
        for (int part = 0; part < 3; ++part) {
          const uint32_t a_addr = a0 + (2 * part) * kFArr + (f0 + off) * 16;
          umma_bf16(tmem + p * 16, smem_desc(a_addr, kFArr, 128), bd, (t | part) != 0);
        }
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     bar_mma)
                 : "memory");
  }
  __syncwarp();  // warp 0's other lanes wait here while lane 0 issues
  ok = __syncthreads_and(ok ? 1 : 0) != 0;
  if (ok) ok = mbar_wait(bar_mma, 0);
  tc_fence_after();
  if (!ok) {
    if (tid == 0) atomicAdd(&g_fast_timeouts, 1ull);
  } else {
    // warp w: TMEM lanes 32(w%4).. of plane w/4 = output rows 32(w%4) + lane
    const int quarter = warp & 3, p = warp >> 2;
    const int y = y0 + quarter, x = x0 + lane - 1;
    const bool keep = lane >= 1 && lane <= kFOutCols && x < W && y < H && p < nplanes;
    if (p < nplanes) {
      float v[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + p * 16, v);
      if (keep) {
        const long long q = (dp0 + p) * HW + static_cast<long long>(y) * W + x;
        if (LAST) {
          const float sf = s[f];
#pragma unroll
          for (int o = 0; o < 16; ++o)
            if (o < nout) out_y[(static_cast<long long>(f) * nout + o) * P + q] = v[o] * sf;
        } else {
#pragma unroll
          for (int o = 0; o < 16; ++o) v[o] = o < nout ? gelu_f(v[o]) : 0.0f;
          uint4 w[6];
          split16(v, w);
          uint4 *o = out_packed + static_cast<long long>(f) * 6 * P + q;
#pragma unroll
          for (int a = 0; a < 6; ++a) o[a * P] = w[a];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFTmemCols)
                 : "memory");
  }
}

inline unsigned nblocks(long long n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

int closure_fast_rms(const float *X, int C, long long P, float *part, float *s, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_face_sumsq<<<dim3(kRmsBlocks, 6), 256, 0, st>>>(X, C, P, part);
  k_face_rms_fold<<<6, 256, 0, st>>>(part, kRmsBlocks, P, s);
  return cudaGetLastError();
}

int closure_fast_pack(const float *X, int C, long long P, const float *s, void *packed, void *stream) {
  k_pack_band<<<dim3(nblocks(P, 256), 6), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      X, C, P, s, static_cast<uint4 *>(packed));
  return cudaGetLastError();
}

int closure_fast_pack_weights(const void *w, int co, int ci, void *wp, void *stream) {
  k_pack_weights<<<dim3(8, 6), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16 *>(w), co, ci, static_cast<__nv_bfloat16 *>(wp));
  return cudaGetLastError();
}

int closure_fast_conv(const CUtensorMap &tm_in, const void *wp, void *out_packed, float *out_y,
                      const float *s, int nout, int D, int H, int W, bool last, void *stream) {
  static bool attr[2] = {false, false};
  const void *fn = last ? reinterpret_cast<const void *>(k_conv_fast<true>)
                        : reinterpret_cast<const void *>(k_conv_fast<false>);
  if (!attr[last]) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem);
    if (e != cudaSuccess) return e;
    attr[last] = true;
  }
  const int ndt = (D + kFDT - 1) / kFDT;
  const dim3 grid(nblocks(W, kFOutCols), nblocks(H, kFOutRows), 6 * ndt);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const __nv_bfloat16 *w = static_cast<const __nv_bfloat16 *>(wp);
  if (last)
    k_conv_fast<true><<<grid, kFThreads, kFSmem, st>>>(tm_in, w, nullptr, out_y, s, nout, D, H, W, ndt);
  else
    k_conv_fast<false><<<grid, kFThreads, kFSmem, st>>>(tm_in, w, static_cast<uint4 *>(out_packed),
                                                        nullptr, s, nout, D, H, W, ndt);
  return cudaGetLastError();
}

unsigned long long closure_fast_timeouts() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_fast_timeouts, sizeof(v));
  return v;
}

}  // namespace wf
