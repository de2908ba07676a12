// wf_conv_tc.cu -- the closure network's 3x3x3 convolutions on the sm_100a
// tensor cores (tcgen05.mma, accumulators in tensor memory), as implicit
// GEMMs: M = 128 output voxels, N = 16 output channels, K = 16 input channels
// per tap, 27 taps accumulated into the same tensor-memory tile.
//
// Numerics.  The weights are bfloat16 (exact operands).  An FP32 activation
// a is split into three bfloat16 parts, a1 = bf16(a), a2 = bf16(a - a1),
// a3 = bf16(a - a1 - a2) (each difference exact in FP32), and every part is
// multiplied by the weight (three MMAs per tap): the operand keeps 24
// significant bits, like FP32 itself (two parts would keep 16, a relative
// error up to 2^-16), every product is exact, and the tensor core
// accumulates in FP32.  Results agree with the FP32 CUDA-core kernels to
// about 1e-7 relative, not bit for bit (the summation order differs).
//
// Data layout in shared memory (no swizzle, K-major canonical layout: core
// matrices of 8 rows x 16 bytes):
//   A  [part 1..3][channel half][plane][row][col] x 8 channels (16 bytes a
//      voxel): a tile of DT+2 depth planes x 6 rows x 32 columns around the
//      CTA's DT x 4 x 30 output voxels.  Output voxels (plane p, rows 1..4,
//      columns 0..31) are 128 consecutive voxels, so one M tile of a plane is
//      one descriptor, and a tap (dz, dy, dx) only moves its start address by
//      (dz*192 + dy*32 + dx) voxels.  Columns 0 and 31 are the tile's x halo:
//      their rows are computed and discarded (30 of every 32 rows are kept).
//      SBO (8 rows) = 128 bytes; LBO (next 8 channels) = one channel-half array.
//   B  [tap][channel half][16 output channels][8 input channels]: 512 bytes a
//      tap, SBO 128, LBO 256.
// Tensor memory: DT tiles of 128 lanes x 16 FP32 columns (one per plane).
//
// One thread issues all MMAs of the CTA and commits them to an mbarrier;
// the wait is bounded (a timeout is counted, the epilogue is skipped and the
// tensor memory is still freed).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "wf_closure.h"
#include "wf_internal.cuh"

namespace wf {

namespace {

constexpr int kTcDT = 2;            // output depth planes per CTA
constexpr int kTcParts = 3;         // bfloat16 parts of an FP32 activation
constexpr int kTcPlanes = kTcDT + 2;
constexpr int kTcRows = 6;          // 4 output rows + halo
constexpr int kTcCols = 32;         // 30 output columns + halo
constexpr int kTcOutRows = 4, kTcOutCols = 30;
constexpr int kTcVox = kTcPlanes * kTcRows * kTcCols;            // 768
constexpr int kTcArr = (16 + kTcVox * 16 + 16 + 127) / 128 * 128;  // one [part][half] array, bytes
constexpr int kTcA = 2 * kTcParts * kTcArr;                        // parts x 2 channel halves
constexpr int kTcB = 27 * 512;
constexpr int kTcBar = kTcA + kTcB;
constexpr int kTcSmem = kTcBar + 16;
constexpr int kTcThreads = 256;  // 8 warps: two per TMEM lane quarter
constexpr int kTcCols32 = 32;  // tensor-memory columns allocated (kTcDT x 16, power of two)
static_assert(kTcDT * 16 <= kTcCols32, "accumulator tiles fit the allocation");

__device__ unsigned long long g_tc_timeouts;  // bounded-wait expiries (diagnostic)

constexpr float kInvSqrt2f = 0.70710678118654752f;
__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * kInvSqrt2f)); }

// Shared-memory matrix descriptor, no swizzle (sm_100 version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D,
// M = 128, N = 16.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
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

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo_elem));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi_elem));
  return a | (b << 16);
}

// out[s][co][p] = sum_ci sum_tap W[tap][co][ci] * in[s][ci][p + tap], with
// W from the bfloat16 weights [F][co][ci][27] (forward) or, for the
// gradient with respect to the input, [F][ci][co][27] transposed and with
// the taps flipped (BWD: in = dz with `kin` = co channels, out = ci).
template <bool BWD>
__global__ void __launch_bounds__(kTcThreads, 2)
    k_conv_tc(const float *in, const __nv_bfloat16 *w, const int *face, float *z, float *a,
              int kin, int nout, int D, int H, int W, int ndt, int act) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = blockIdx.z / ndt, dt = blockIdx.z % ndt;
  const int x0 = blockIdx.x * kTcOutCols, y0 = blockIdx.y * kTcOutRows, dp0 = dt * kTcDT;
  const int f = face ? face[s] : 0;
  const long long HW = static_cast<long long>(H) * W, P = HW * D;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar = sbase + kTcBar;

  if (warp == 0) {  // tensor memory for the DT accumulator tiles
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(kTcCols32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }

  // B: weights of the sample's face, [tap][half][n 16][k 8] bf16, zero padded.
  // The face's weights are one contiguous block: copied as it is (16-byte
  // vectors when it allows) into the A region, which is filled only after,
  // then rearranged from there.
  {
    __nv_bfloat16 *sb = reinterpret_cast<__nv_bfloat16 *>(smem + kTcA);
    __nv_bfloat16 *raw = reinterpret_cast<__nv_bfloat16 *>(smem);
    const int wn = BWD ? kin : nout;   // first index of the stored weights (co)
    const int wk = BWD ? nout : kin;   // second (ci)
    const int nraw = wn * wk * 27;
    const __nv_bfloat16 *wf = w + static_cast<long long>(f) * nraw;
    if ((nraw % 8) == 0 && (reinterpret_cast<uintptr_t>(wf) & 15) == 0) {
      const uint4 *src = reinterpret_cast<const uint4 *>(wf);
      uint4 *dst = reinterpret_cast<uint4 *>(raw);
      for (int i = tid; i < nraw / 8; i += kTcThreads) dst[i] = __ldg(src + i);
    } else {
      for (int i = tid; i < nraw; i += kTcThreads) raw[i] = wf[i];
    }
    __syncthreads();
    for (int i = tid; i < 27 * 256; i += kTcThreads) {
      const int t = i >> 8, e = i & 255;
      const int half = e >> 7, n = (e >> 3) & 15, k = half * 8 + (e & 7);
      __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
      if (n < nout && k < kin) v = BWD ? raw[(k * wk + n) * 27 + (26 - t)] : raw[(n * wk + k) * 27 + t];
      sb[i] = v;
    }
    __syncthreads();  // the raw copy in the A region is consumed
  }
  // A: the input tile as three bfloat16 parts, zero outside the tensor
  {
    constexpr int NA = 2 * kTcParts;
    uint4 *arr[NA];
#pragma unroll
    for (int q = 0; q < NA; ++q) arr[q] = reinterpret_cast<uint4 *>(smem + q * kTcArr + 16);
    if (tid < 2 * NA) {  // guards before and after each array
      const int q = tid % NA;
      uint4 *g = tid < NA ? arr[q] - 1 : arr[q] + kTcVox;
      *g = make_uint4(0u, 0u, 0u, 0u);
    }
    const int col = tid & 31;
    const float *src = in + static_cast<long long>(s) * kin * P;
    for (int pr = tid >> 5; pr < kTcPlanes * kTcRows; pr += kTcThreads / 32) {
      const int pl = pr / kTcRows, row = pr % kTcRows;
      const int d = dp0 - 1 + pl, y = y0 - 1 + row, x = x0 - 1 + col;
      const bool inside = d >= 0 && d < D && y >= 0 && y < H && x >= 0 && x < W;
      const long long off = d * HW + static_cast<long long>(y) * W + x;
      float v[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] = (inside && c < kin) ? __ldg(src + c * P + off) : 0.0f;
      const int vox = pr * kTcCols + col;
#pragma unroll
      for (int part = 0; part < kTcParts; ++part) {
        uint32_t q[8];
#pragma unroll
        for (int c = 0; c < 16; c += 2) {  // this part, and the residual left for the next
          const float h0 = __bfloat162float(__float2bfloat16_rn(v[c]));
          const float h1 = __bfloat162float(__float2bfloat16_rn(v[c + 1]));
          q[c / 2] = pack_bf16(h0, h1);
          v[c] -= h0;
          v[c + 1] -= h1;
        }
        arr[2 * part][vox] = make_uint4(q[0], q[1], q[2], q[3]);
        arr[2 * part + 1][vox] = make_uint4(q[4], q[5], q[6], q[7]);
      }
    }
  }
  fence_proxy_async();  // the operands above are read by the tensor core (async proxy)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int nplanes = min(kTcDT, D - dp0);

  if (tid == 0) {
    const uint32_t b0 = sbase + kTcA;
    for (int p = 0; p < nplanes; ++p) {
      const int f0 = ((p + 1) * kTcRows + 1) * kTcCols;  // first output row of plane p
      for (int t = 0; t < 27; ++t) {
        const int off = (t / 9 - 1) * kTcRows * kTcCols + ((t / 3) % 3 - 1) * kTcCols + (t % 3 - 1);
        const uint64_t bd = smem_desc(b0 + t * 512, 256, 128);
#pragma unroll
        for (int part = 0; part < kTcParts; ++part) {
          const uint32_t a_addr = sbase + (2 * part) * kTcArr + 16 + (f0 + off) * 16;
          umma_bf16(tmem + p * 16, smem_desc(a_addr, kTcArr, 128), bd, (t | part) != 0);
        }
      }
    }
    umma_commit(bar);
  }
  // warp 0's other lanes wait here, not in the mbarrier's try-wait loop: a
  // divergent warp alternates between its paths, and lanes suspended in the
  // try-wait would hold back the lane issuing the MMAs
  __syncwarp();
  const bool done = mbar_wait(bar, 0);
  tc_fence_after();
  if (!done) {
    if (tid == 0) atomicAdd(&g_tc_timeouts, 1ull);
  } else {
    // epilogue: warp w reads tensor-memory lanes 32(w%4)..+31 of plane w/4's
    // tile = output rows 32(w%4) + lane: voxel (row 1 + w%4, column lane)
    const int quarter = warp & 3;
    const int y = y0 + quarter, x = x0 + lane - 1;
    const bool keep = lane >= 1 && lane <= kTcOutCols && x < W && y < H;
    for (int p = warp >> 2; p < nplanes; p += kTcThreads / 128) {
      float v[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + p * 16, v);
      if (keep) {
        const long long q = (dp0 + p) * HW + static_cast<long long>(y) * W + x;
#pragma unroll
        for (int o = 0; o < 16; ++o) {
          if (o >= nout) break;
          const long long k = (static_cast<long long>(s) * nout + o) * P + q;
          if (z) z[k] = v[o];
          a[k] = act ? gelu_f(v[o]) : v[o];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols32)
                 : "memory");
  }
}

template <bool BWD>
int launch_tc(const float *in, const void *w, const int *face, float *z, float *a, int n, int kin,
              int nout, int D, int H, int W, int act, cudaStream_t st) {
  if (kin < 1 || kin > 16 || nout < 1 || nout > 16 || n < 1 || D < 1 || H < 1 || W < 1)
    return cudaErrorInvalidValue;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_tc<BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kTcSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int ndt = (D + kTcDT - 1) / kTcDT;
  const dim3 grid((W + kTcOutCols - 1) / kTcOutCols, (H + kTcOutRows - 1) / kTcOutRows, n * ndt);
  k_conv_tc<BWD><<<grid, kTcThreads, kTcSmem, st>>>(in, static_cast<const __nv_bfloat16 *>(w), face,
                                                     z, a, kin, nout, D, H, W, ndt, act);
  return cudaGetLastError();
}

}  // namespace

int nn_conv_fwd_tc(const float *in, const void *w_bf16, const int *face, float *z, float *a, int n,
                   int ci, int co, int D, int H, int W, int act, void *stream) {
  return launch_tc<false>(in, w_bf16, face, z, a, n, ci, co, D, H, W, act,
                          static_cast<cudaStream_t>(stream));
}

int nn_conv_bwd_data_tc(const float *dz, const void *w_bf16, const int *face, float *din, int n,
                        int ci, int co, int D, int H, int W, void *stream) {
  return launch_tc<true>(dz, w_bf16, face, nullptr, din, n, co, ci, D, H, W, 0,
                         static_cast<cudaStream_t>(stream));
}

unsigned long long nn_tc_timeouts() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_tc_timeouts, sizeof(v));
  return v;
}

}  // namespace wf
