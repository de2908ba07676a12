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
// so that a CTA brings each input plane of its tile (6 rows x 32 columns of
// all six arrays) into shared memory with one TMA box (x and the 8 channels of
// a word form the box's 512-byte rows), whose zero fill outside the band is
// the convolution's zero padding, and its face's pre-arranged weights with one
// bulk copy.  A tile spans the band's whole depth, so every input plane is
// loaded once, and one MMA of N = 48 applies the taps dz = -1, 0, +1 of an
// input plane to the three output planes it feeds: an M 128 x K 16 MMA costs
// the same for every N up to 64 (measured on B200), so this does the work of
// three N = 16 MMAs for the price of one.  The epilogue applies GELU and
// writes the next layer's input already split; the last layer writes FP32
// times the face's RMS.  The operands, the per-output tap order and the FP32
// accumulation are those of k_conv_tc, so the results equal the FP32 path's.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "wf_band.cuh"
#include "wf_closure.h"
#include "wf_internal.cuh"

namespace wf {

namespace {

// A tile is the band's whole depth (8 planes) x 4 rows x 30 columns of
// outputs; its input is 8 planes x 6 rows x 32 columns (zero outside the
// band), one 18 KB plane slot each.
constexpr int kFD = 8, kFRows = 6, kFCols = 32, kFOutRows = 4, kFOutCols = 30;
constexpr int kFPlaneVox = kFRows * kFCols;             // 192 voxels a plane
constexpr int kFArr = kFPlaneVox * 16;                   // 3072 B: one array of a plane
constexpr int kFPlaneBytes = 6 * kFArr;                  // 18 432 B: one plane slot
constexpr int kFN = 48;                                  // MMA N: three planes x 16 outputs
constexpr int kFWHalf = kFN * 16;                        // 768 B: one K half of a weight block
constexpr int kFWBlock = 2 * kFWHalf;                    // one (dy, dx) block
constexpr int kFWBytes = 9 * kFWBlock;                   // 13 824 B: one face's weights
// Shared memory: [guard][8 plane slots][guard][zero block][2 weight slots]
// [barriers].  The corner taps of a plane's first and last output rows read
// one voxel before or after the slot; those reads only feed the discarded
// halo lanes, and the guards keep the first and the last slot's inside the
// allocation.
constexpr int kFGuard = 128;
constexpr int kFAOff = kFGuard;
constexpr int kFZOff = kFAOff + kFD * kFPlaneBytes + kFGuard;
constexpr int kFZBytes = 4096;                           // A of zeros: clears an accumulator
constexpr int kFWOff = kFZOff + kFZBytes;
constexpr int kFBarOff = kFWOff + 2 * kFWBytes;
// full[8], empty[8], wfull[2], wempty[2], acc_full[2], acc_empty[2], done
constexpr int kFNumBars = 25;
constexpr int kFSmem = kFBarOff + kFNumBars * 8 + 128;  // + base alignment slack
constexpr int kFEpiWarps = 16;                           // 4 lane quarters x 4 plane pairs
constexpr int kFThreads = 64 + 32 * kFEpiWarps;          // TMA warp, MMA warp, epilogue
// Two accumulators of 160 columns: planes -1 .. 8 of 16 columns each (the
// outer two take the products of the first and last plane's out-of-band
// taps and are never read), 256 columns apart.
constexpr int kFAccCols = 256;
constexpr int kFTmemCols = 512;
static_assert(kFPlaneBytes % 128 == 0 && kFWOff % 128 == 0 && kFSmem <= 227 * 1024,
              "closure conv shared-memory layout");

__device__ unsigned long long g_fast_timeouts;

constexpr float kInvSqrt2f = 0.70710678118654752f;
__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * kInvSqrt2f)); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16, BF16 A and B (K-major), FP32 D, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_n(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum));
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

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}


}  // namespace

namespace {

// Layer 1's packed input straight from the grid: face f's band cells (the 6
// fields and the 4 psi of its normal axis, times the gains; channels 10-15
// zero) split into three bfloat16 parts, through the transposing tile of
// band_gather (grid side along x, band side along v).  Each CTA also writes
// the sum of squares of its E values to part[f * stride + CTA], summed in a
// fixed order.  One launch covers both faces of axis AX.
template <int AX>
__global__ void __launch_bounds__(256) k_band_gather_pack(BandGrid g, uint4 *packed, float *part,
                                                          long long stride, int H, int W, float ge,
                                                          float gh) {
  using T = BandTile<AX>;
  __shared__ float s[kBandIn][T::TO][T::TA][33];
  __shared__ float s_sum[256];
  const int side = blockIdx.z / T::kZ, sub = blockIdx.z % T::kZ, f = 2 * AX + side;
  const int v0 = blockIdx.x * 32;
  const long long P = static_cast<long long>(kBandDepth) * H * W;
  const BandPsi &ps = g.psi[AX];
  float acc = 0.0f;
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
      for (int c = 0; c < 6; ++c) {
        const float val = g.fields[c * g.N + cell] * (c < 3 ? ge : gh);
        s[c][ol][al][vl] = val;
        if (c < 3) acc += val * val;
      }
      const long long k = psi_index(g, AX, x, y, z);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        s[6 + c][ol][al][vl] = k >= 0 ? ps.p[c * ps.cells + k] * (c < 2 ? ge : gh) : 0.0f;
    }
  }
  s_sum[threadIdx.x] = acc;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < T::kElems / 256; ++j) {  // band side: v fastest
    const int e = threadIdx.x + 256 * j, vl = e % 32, al = (e / 32) % T::TA, ol = e / (32 * T::TA);
    int d, u;
    band_du<AX>(al, ol, blockIdx.y, sub, d, u);
    const int v = v0 + vl;
    if (d < kBandDepth && u < H && v < W) {
      float val[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) val[c] = c < kBandIn ? s[c][ol][al][vl] : 0.0f;
      uint4 w[6];
      split16(val, w);
      uint4 *o = packed + static_cast<long long>(f) * 6 * P + (static_cast<long long>(d) * H + u) * W + v;
#pragma unroll
      for (int q = 0; q < 6; ++q) o[q * P] = w[q];
    }
  }
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) s_sum[threadIdx.x] += s_sum[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    part[f * stride + (static_cast<long long>(sub) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] =
        s_sum[0];
}

// CTAs per face of k_band_gather_pack<AX>
__host__ __device__ inline long long gather_parts(int ax, int H, int W) {
  const long long bx = (W + 31) / 32;
  return ax == 0 ? bx * ((H + BandTile<0>::TO - 1) / BandTile<0>::TO)
                 : bx * ((H + 31) / 32) * BandTile<1>::kZ;
}

// s[f] = sqrt(sum / 3P) + 1e-30 from face f's partial sums, as face_rms
// computes it (fixed order: strided per thread, then a tree).
__global__ void k_face_rms_fold(const float *part, long long stride, int H, int W, long long P,
                                float *s) {
  __shared__ float s_sum[256];
  const int f = blockIdx.x;
  const long long nb = gather_parts(f >> 1, H, W);
  float acc = 0.0f;
  for (long long i = threadIdx.x; i < nb; i += blockDim.x) acc += part[f * stride + i];
  s_sum[threadIdx.x] = acc;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) s_sum[threadIdx.x] += s_sum[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) s[f] = sqrtf(s_sum[0] / static_cast<float>(3 * P)) + 1e-30f;
}

// Wp[f][r = 3 (dy + 1) + dx + 1][half][n 48][k 8] bf16 from W[f][co][ci][27]
// (tap (dz + 1) 9 + r, zero padded): rows n = 16 j + co hold the tap with
// dz = 1 - j, the three planes one input plane feeds.
__global__ void k_pack_weights(const __nv_bfloat16 *w, int co, int ci, __nv_bfloat16 *wp) {
  const int f = blockIdx.y;
  constexpr int kPer = 9 * 2 * kFN * 8;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kPer; i += gridDim.x * blockDim.x) {
    const int r = i / (2 * kFN * 8), e = i % (2 * kFN * 8);
    const int half = e / (kFN * 8), n = (e / 8) % kFN, k = half * 8 + (e & 7);
    const int j = n / 16, o = n % 16, t = (2 - j) * 9 + r;
    __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
    if (o < co && k < ci) v = w[((static_cast<long long>(f) * co + o) * ci + k) * 27 + t];
    wp[static_cast<long long>(f) * kPer + i] = v;
  }
}

}  // namespace

namespace {

// Tile t of a layer: x tiles fastest, then rows, then faces.
struct FastTile {
  int f, y0, x0;
};
__device__ __forceinline__ FastTile fast_tile(long long t, int txc, int tyc) {
  FastTile r;
  r.x0 = static_cast<int>(t % txc) * kFOutCols;
  t /= txc;
  r.y0 = static_cast<int>(t % tyc) * kFOutRows;
  r.f = static_cast<int>(t / tyc);
  return r;
}

// One layer of the in-step closure over all six face bands.  A persistent
// CTA per SM takes tiles blockIdx.x, + gridDim.x, ... (neighbouring tiles run
// together, so halo rows are read from L2), with three roles working on
// different tiles at once:
//   warp 0      TMA: the tile's eight input planes, one box each (x and the 8
//               channels of a word form the box's 512-byte rows; the zero
//               fill outside the band is the convolution's zero padding), into
//               eight plane slots, and its face's weights (one bulk copy) into
//               one of two weight slots;
//   warp 1      MMA: one MMA (A of zeros) clears the accumulator, then for each
//               input plane z, each in-plane tap (dy, dx) and each of the three
//               bfloat16 parts one MMA of M 128 x N 48 x K 16: the same input
//               rows feed output planes z + 1, z and z - 1 through the taps
//               dz = -1, 0, +1, whose weights are stacked along N.  A plane
//               slot is handed back as soon as its MMAs are done;
//   warps 2-17  epilogue: tensor memory to registers, the accumulator handed
//               back, then GELU and the next layer's packed input, or (LAST)
//               the FP32 correction times s[f].
// Per output the taps are summed in the order (dz, dy, dx, part), the order
// of the one-plane form.  Every wait is bounded; a wait that gives up counts
// a timeout and ends its role's loop, and the CTA waits (bounded) for its
// copies and MMAs in flight before it frees tensor memory and exits.
template <bool LAST>
__global__ void __launch_bounds__(kFThreads, 1)
    k_conv_fast(const __grid_constant__ CUtensorMap tm_in, const __nv_bfloat16 *wp,
                uint4 *out_packed, float *out_y, const float *s, const float *in_scale, int nout,
                int H, int W) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  __shared__ uint32_t s_tmem;
  __shared__ int s_pl_issued[kFD], s_pl_used[kFD], s_w_issued[2], s_w_used[2];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int txc = (W + kFOutCols - 1) / kFOutCols, tyc = (H + kFOutRows - 1) / kFOutRows;
  const long long ntot = 6LL * tyc * txc, t0 = blockIdx.x, tstep = gridDim.x;
  const int ntiles = static_cast<int>((ntot - t0 + tstep - 1) / tstep);
  const long long HW = static_cast<long long>(H) * W, P = HW * kFD;
  const uint32_t sbase = smem_u32(smem), bars = sbase + kFBarOff;
  const uint32_t a_base = sbase + kFAOff, z_base = sbase + kFZOff, w_base = sbase + kFWOff;
  auto full = [&](int z) { return bars + 8 * z; };
  auto empty = [&](int z) { return bars + 64 + 8 * z; };
  auto wfull = [&](int k) { return bars + 128 + 8 * k; };
  auto wempty = [&](int k) { return bars + 144 + 8 * k; };
  auto acc_full = [&](int k) { return bars + 160 + 8 * k; };
  auto acc_empty = [&](int k) { return bars + 176 + 8 * k; };
  const uint32_t done = bars + 192;

  for (int i = tid; i < kFZBytes / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(smem + kFZOff)[i] = make_uint4(0u, 0u, 0u, 0u);
  fence_proxy_async();  // the zero block is read by the tensor cores
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(kFTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int z = 0; z < kFD; ++z) {
      mbar_init(full(z), 1);
      mbar_init(empty(z), 1);
      s_pl_issued[z] = 0;
      s_pl_used[z] = 0;
    }
    for (int k = 0; k < 2; ++k) {
      mbar_init(wfull(k), 1);
      mbar_init(wempty(k), 1);
      mbar_init(acc_full(k), 1);
      mbar_init(acc_empty(k), kFEpiWarps);
      s_w_issued[k] = 0;
      s_w_used[k] = 0;
    }
    mbar_init(done, 1);
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  bool ok = true;

  if (warp == 0) {
    for (int i = 0; i < ntiles && ok; ++i) {
      const FastTile tl = fast_tile(t0 + i * tstep, txc, tyc);
      const int ws = i & 1;
      if (lane == 0) {
        ok = mbar_wait(wempty(ws), ((i >> 1) & 1) ^ 1);
        if (ok) {
          mbar_expect_tx(wfull(ws), kFWBytes);
          bulk_load(w_base + ws * kFWBytes, wp + static_cast<long long>(tl.f) * (kFWBytes / 2), kFWBytes,
                    wfull(ws));
          ++s_w_issued[ws];
        }
        for (int z = 0; z < kFD && ok; ++z) {
          ok = mbar_wait(empty(z), (i & 1) ^ 1);
          if (!ok) break;
          mbar_expect_tx(full(z), kFPlaneBytes);
          tma_load_4d(a_base + z * kFPlaneBytes, &tm_in, 8 * (tl.x0 - 1), tl.y0 - 1, z, tl.f * 6, full(z));
          ++s_pl_issued[z];
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    }
  } else if (warp == 1) {
    constexpr uint32_t kIdZero = idesc_n(160), kId48 = idesc_n(kFN);
    for (int i = 0; i < ntiles && ok; ++i) {
      const int ws = i & 1, acc = i & 1;
      if (lane == 0) {
        ok = mbar_wait(acc_empty(acc), ((i >> 1) & 1) ^ 1) && mbar_wait(wfull(ws), (i >> 1) & 1);
        if (ok) {
          ++s_w_used[ws];
          tc_fence_after();
          const uint32_t d0 = tmem + acc * kFAccCols;
          const uint32_t wb = w_base + ws * kFWBytes;
          // D = 0 x B: the accumulator's 160 columns start from zero
          umma_bf16(d0, smem_desc(z_base, 2048, 128), smem_desc(wb, kFWHalf, 128), kIdZero, 0u);
          // Descriptors of a slot's first row and of the first weight block;
          // a shifted operand adds its byte offset / 16 to the address field,
          // which stays below 2^14 (shared memory < 256 KB).
          const uint64_t ad0 = smem_desc(a_base, kFArr, 128), bd0 = smem_desc(wb, kFWHalf, 128);
          for (int z = 0; z < kFD && ok; ++z) {
            ok = mbar_wait(full(z), i & 1);
            if (!ok) break;
            ++s_pl_used[z];
            // (the TMA's complete_tx on full(z) orders the plane before these
            // MMAs, as in a TMA-to-UMMA pipeline: no tcgen05 fence here)
            const uint32_t d = d0 + 16 * z;  // planes z - 1, z, z + 1
#pragma unroll
            for (int r = 0; r < 9; ++r) {
              const int row = (r / 3) * kFCols + (r % 3 - 1);  // first A row: output row 1 + dy, dx
              const uint64_t bd = bd0 + static_cast<uint64_t>(r * kFWBlock / 16);
#pragma unroll
              for (int part = 0; part < 3; ++part) {
                const long long a_off =
                    (static_cast<long long>(z) * kFPlaneBytes + (2 * part) * kFArr + row * 16) / 16;
                umma_bf16(d, ad0 + static_cast<uint64_t>(a_off), bd, kId48, 1u);
              }
            }
            tc_commit(empty(z));  // the slot is free once these MMAs are done
          }
          if (ok) {
            tc_commit(wempty(ws));
            tc_commit(acc_full(acc));
          }
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    }
    // every MMA issued completes before the teardown frees tensor memory
    bool fin = true;
    if (lane == 0) {
      tc_commit(done);
      fin = mbar_wait(done, 0);
    }
    if (!(__shfl_sync(0xffffffffu, fin ? 1 : 0, 0) != 0)) ok = false;
  } else {
    // warp w reads TMEM lanes 32 (w % 4) ..: output rows 32 (w % 4) + lane of
    // planes 2 g and 2 g + 1, g = (w - 2) / 4
    const int quarter = warp & 3, g = (warp - 2) >> 2;
    for (int i = 0; i < ntiles; ++i) {
      const int acc = i & 1;
      if (lane == 0) ok = mbar_wait(acc_full(acc), (i >> 1) & 1);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      tc_fence_after();
      const FastTile tl = fast_tile(t0 + i * tstep, txc, tyc);
      float v[2][16];
      const uint32_t ta = tmem + (static_cast<uint32_t>(quarter * 32) << 16) + acc * kFAccCols;
      tmem_ld16(ta + 16 * (2 * g + 1), v[0]);  // plane p at column 16 (p + 1)
      tmem_ld16(ta + 16 * (2 * g + 2), v[1]);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty(acc));
      const int y = tl.y0 + quarter, x = tl.x0 + lane - 1;
      if (lane >= 1 && lane <= kFOutCols && x < W && y < H) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const long long q = (2 * g + h) * HW + static_cast<long long>(y) * W + x;
          if (LAST) {
            const float sf = s[tl.f];
#pragma unroll
            for (int o = 0; o < 16; ++o)
              if (o < nout) out_y[(static_cast<long long>(tl.f) * nout + o) * P + q] = v[h][o] * sf;
          } else {
            if (in_scale) {
              const float m = 1.0f / in_scale[tl.f];  // as face_scale divides: times the reciprocal
#pragma unroll
              for (int o = 0; o < 16; ++o) v[h][o] *= m;
            }
#pragma unroll
            for (int o = 0; o < 16; ++o) v[h][o] = o < nout ? gelu_f(v[h][o]) : 0.0f;
            uint4 wv[6];
            split16(v[h], wv);
            uint4 *op = out_packed + static_cast<long long>(tl.f) * 6 * P + q;
#pragma unroll
            for (int a = 0; a < 6; ++a) op[a * P] = wv[a];
          }
        }
      }
    }
  }
  if (!ok && lane == 0) atomicAdd(&g_fast_timeouts, 1ull);
  __syncthreads();
  // copies issued and never consumed (only after a wait gave up) land before exit
  if (tid == 0) {
    for (int z = 0; z < kFD; ++z)
      if (s_pl_issued[z] > s_pl_used[z]) mbar_wait(full(z), (s_pl_issued[z] - 1) & 1);
    for (int k = 0; k < 2; ++k)
      if (s_w_issued[k] > s_w_used[k]) mbar_wait(wfull(k), (s_w_issued[k] - 1) & 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFTmemCols)
                 : "memory");
  }
}

inline unsigned nblocks(long long n, int t) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

long long closure_fast_parts(int H, int W) {
  const long long a = gather_parts(0, H, W), b = gather_parts(1, H, W);
  return a > b ? a : b;
}

int closure_fast_gather(const BandGrid &g, void *packed, float *part, int H, int W, float ge,
                        float gh, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint4 *pk = static_cast<uint4 *>(packed);
  const long long stride = closure_fast_parts(H, W);
  const unsigned bx = nblocks(W, 32);
  k_band_gather_pack<0><<<dim3(bx, nblocks(H, BandTile<0>::TO), 2 * BandTile<0>::kZ), 256, 0, st>>>(
      g, pk, part, stride, H, W, ge, gh);
  k_band_gather_pack<1><<<dim3(bx, nblocks(H, 32), 2 * BandTile<1>::kZ), 256, 0, st>>>(
      g, pk, part, stride, H, W, ge, gh);
  k_band_gather_pack<2><<<dim3(bx, nblocks(H, 32), 2 * BandTile<2>::kZ), 256, 0, st>>>(
      g, pk, part, stride, H, W, ge, gh);
  return cudaGetLastError();
}

int closure_fast_rms(const float *part, int H, int W, long long P, float *s, void *stream) {
  k_face_rms_fold<<<6, 256, 0, static_cast<cudaStream_t>(stream)>>>(part, closure_fast_parts(H, W), H,
                                                                     W, P, s);
  return cudaGetLastError();
}

int closure_fast_pack_weights(const void *w, int co, int ci, void *wp, void *stream) {
  k_pack_weights<<<dim3(8, 6), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16 *>(w), co, ci, static_cast<__nv_bfloat16 *>(wp));
  return cudaGetLastError();
}

int closure_fast_conv(const CUtensorMap &tm_in, const void *wp, void *out_packed, float *out_y,
                      const float *s, const float *in_scale, int nout, int D, int H, int W, bool last,
                      void *stream) {
  if (D != kFD) return cudaErrorInvalidValue;
  static bool attr[2] = {false, false};
  const void *fn = last ? reinterpret_cast<const void *>(k_conv_fast<true>)
                        : reinterpret_cast<const void *>(k_conv_fast<false>);
  if (!attr[last]) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem);
    if (e != cudaSuccess) return e;
    attr[last] = true;
  }
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const long long ntot = 6LL * nblocks(H, kFOutRows) * nblocks(W, kFOutCols);
  const unsigned grid = static_cast<unsigned>(ntot < nsm ? ntot : nsm);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const __nv_bfloat16 *w = static_cast<const __nv_bfloat16 *>(wp);
  if (last)
    k_conv_fast<true><<<grid, kFThreads, kFSmem, st>>>(tm_in, w, nullptr, out_y, s, nullptr, nout, H, W);
  else
    k_conv_fast<false><<<grid, kFThreads, kFSmem, st>>>(tm_in, w, static_cast<uint4 *>(out_packed),
                                                        nullptr, s, in_scale, nout, H, W);
  return cudaGetLastError();
}

unsigned long long closure_fast_timeouts() {
  unsigned long long v = 0;
  cudaMemcpyFromSymbol(&v, g_fast_timeouts, sizeof(v));
  return v;
}

}  // namespace wf
