// wf_internal.cuh -- device-side state and the per-cell Yee/CPML arithmetic
// shared by every step kernel (split, fused, batched), so that all of them
// compute bit-identical results.
//
// The arithmetic restates src/fdtd.rs of the reference:
//   H = Da*H - Db*curl(E)       forward differences   (src/fdtd.rs:237-250)
//   E = Ca*E + Cb*curl(H)       backward differences  (src/fdtd.rs:412-425)
//   psi = b*psi + a*raw; d = raw*(1/kappa) + psi     (src/fdtd.rs:136-163)
// Exact mode uses __fmul_rn/__fadd_rn/__fsub_rn, which the compiler never
// contracts into an FMA, so results match the reference's AVX2 rows bit for
// bit.  FMA mode uses __fmaf_rn where a product feeds an add.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wf {

constexpr int kTileX = 128;          // cells per tile row: 32 lanes x float4
constexpr long long kWaitLimitCycles = 2000000000LL;  // ~1 s at B200 clocks

// Device error bits (latched in a device word, reported by wf_sync).
enum : int { kErrTimeout = 1, kErrBounds = 2 };

// One axis of the CPML: psi is kept only for cells whose coordinate on this
// axis lies in the graded slab [0,T) U [n-T,n), W = min(2T, n) positions.
struct PmlAxis {
  int T;                 // graded thickness in voxels (0: no CPML on axis)
  int W;                 // slab width
  int pitch;             // x axis: row pitch of the slab array (W rounded up to 4,
                         // so each row starts 16-byte aligned for TMA); y, z: W
  const float *prof;     // [3][W]: b, a, 1/kappa at slab positions
  const float *psi_cur;  // [4][cells]: H term 0, H term 1, E term 0, E term 1
  float *psi_nxt;
  long long cells;       // cells per psi component
};

// Per-axis psi components (slot order inside PmlAxis arrays):
//   x: ez_dx, ey_dx | hz_dx, hy_dx     y: ez_dy, ex_dy | hz_dy, hx_dy
//   z: ey_dz, ex_dz | hy_dz, hx_dz

struct SrcDev {
  int comp, mode, x, y, z, nvals;
  const float *vals;
};

struct ProbeDev {
  int comp, x, y, z, nfreq, nsteps, first_step, record;
  const double *cos_tab, *sin_tab;
  double *sc, *ss;
  unsigned long long *n;
  float *trace;
};

// Field storage of a handle (values match wf_precision of the C ABI).
enum : int { kPrecF32 = 0, kPrecBF16 = 1, kPrecF16 = 2 };
constexpr int kSlabPlanes = 8;  // z planes per storage-scale slab

struct GridArgs {
  int nx, ny, nz;
  long long N;           // nx*ny*nz
  int periodic[3];
  const float *cur;      // 6*N, component-major, x fastest (16-bit elements
  float *nxt;            // when prec != kPrecF32; the kernels cast)
  const uint8_t *mat;    // [nz][ny][mat_pitch]
  int mat_pitch;
  const float4 *coef;    // 256 x {ca, cb, da, db}
  PmlAxis pml[3];
  int *err;
  // 16-bit storage only: per slab (z / kSlabPlanes) and kind (0 E, 1 H)
  int prec;
  const int *shift_rd;   // [nslab][2] shifts of the state read
  const int *shift_wr;   // [nslab][2] shifts of the state written
  unsigned *slab_max;    // [nslab][2] max |decoded value| bits of the state written
  unsigned long long *ovf;  // binary16 saturations
  int nslab;
};

// Bounds-checked builds (compiled with -DWF_BOUNDS_CHECK, the library's
// debugging variant): each checked global access first tests its index
// against the extent of its buffer; a bad index latches kErrBounds in the
// grid's error word (reported by wf_sync) and the access is skipped, a load
// reading zero.  In the normal build the checks compile to nothing.
#ifdef WF_BOUNDS_CHECK
constexpr bool kBoundsCheck = true;
#else
constexpr bool kBoundsCheck = false;
#endif
__device__ __forceinline__ bool idx_ok(int *err, long long i, long long n) {
  if (!kBoundsCheck) return true;
  if (i >= 0 && i < n) return true;
  if (err) atomicOr(err, kErrBounds);
  return false;
}

__device__ __forceinline__ int slab_pos(int c, int n, int T, int W) {
  if (T <= 0) return -1;
  if (c < T) return c;
  if (c >= n - T) return c - (n - W);
  return -1;
}

template <bool FMA>
__device__ __forceinline__ float pml_corr(float raw, float b, float a, float ik, float &psi) {
  float pn, d;
  if (FMA) {
    pn = __fmaf_rn(b, psi, __fmul_rn(a, raw));
    d = __fmaf_rn(raw, ik, pn);
  } else {
    pn = __fadd_rn(__fmul_rn(b, psi), __fmul_rn(a, raw));
    d = __fadd_rn(__fmul_rn(raw, ik), pn);
  }
  psi = pn;
  return d;
}

template <bool FMA>
__device__ __forceinline__ float h_new(float da, float h, float db, float curl) {
  return FMA ? __fmaf_rn(da, h, -__fmul_rn(db, curl))
             : __fsub_rn(__fmul_rn(da, h), __fmul_rn(db, curl));
}

template <bool FMA>
__device__ __forceinline__ float e_new(float ca, float e, float cb, float curl) {
  return FMA ? __fmaf_rn(ca, e, __fmul_rn(cb, curl))
             : __fadd_rn(__fmul_rn(ca, e), __fmul_rn(cb, curl));
}

__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

// ---- mbarrier / TMA helpers (sm_90+ PTX) --------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint32_t bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false if the phase did not complete within
// kWaitLimitCycles, so a lost transfer becomes an error flag, not a hang.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kWaitLimitCycles) return false;
  }
  return true;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *tm, int c0, int c1,
                                            int c2, int c3, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *tm, int c0, int c1,
                                            int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

}  // namespace wf
