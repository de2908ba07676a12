// wf_store.cuh -- field storage formats of the step kernels.
//
// FP32 storage is the reference's own.  The mixed-precision forms store each
// field value as a 16-bit number (IEEE binary16 or bfloat16) of v * 2^-shift,
// where the power-of-two shift belongs to the value's z slab (8 planes) and
// kind (E or H); all arithmetic stays FP32.  Encoding is round to nearest
// even (binary16 saturates finite values at +-65504 and counts them);
// decoding multiplies by 2^shift, which is exact, so a kernel that rounds a
// value it has just computed ("round trip") sees exactly the value any later
// reader decodes.  The per-slab shifts are chosen between steps from the
// slab maxima (see k_tail in wf_split.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "wf_internal.cuh"

namespace wf {

__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }

template <typename ST>
struct Store;

template <>
struct Store<float> {
  static constexpr bool k16 = false;
  static constexpr int PAD = 4;  // 16 bytes of x in elements (TMA box x alignment)
  using Word = float4;
  __device__ static float4 ld4(const float *p, float) { return *reinterpret_cast<const float4 *>(p); }
  __device__ static float ld1(const float *p, float) { return *p; }
  __device__ static float rt(float v, float, float, unsigned long long *) { return v; }
  __device__ static Word enc4(float v[4], float, float, unsigned long long *) {
    return make_float4(v[0], v[1], v[2], v[3]);
  }
  __device__ static void st4(float *p, const Word &w) { *reinterpret_cast<float4 *>(p) = w; }
};

template <typename H>
struct Store16 {
  static constexpr bool k16 = true;
  static constexpr int PAD = 8;
  using Word = uint2;
  __device__ static unsigned short enc1(float u, unsigned long long *ovf);
  __device__ static float dec1(unsigned short b);
  // decoded values of 4 stored halves at p (8-byte aligned), times scale s
  __device__ static float4 ld4(const H *p, float s) {
    const uint2 w = *reinterpret_cast<const uint2 *>(p);
    return make_float4(__fmul_rn(dec1(w.x & 0xffffu), s), __fmul_rn(dec1(w.x >> 16), s),
                       __fmul_rn(dec1(w.y & 0xffffu), s), __fmul_rn(dec1(w.y >> 16), s));
  }
  __device__ static float ld1(const H *p, float s) {
    return __fmul_rn(dec1(*reinterpret_cast<const unsigned short *>(p)), s);
  }
  // the value a reader decodes after v is stored (inv = 2^-shift, s = 2^shift)
  __device__ static float rt(float v, float inv, float s, unsigned long long *ovf) {
    return __fmul_rn(dec1(enc1(__fmul_rn(v, inv), ovf)), s);
  }
  // encodes 4 values, replacing each by its decoded value; returns the word
  __device__ static Word enc4(float v[4], float inv, float s, unsigned long long *ovf) {
    unsigned short b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      b[i] = enc1(__fmul_rn(v[i], inv), ovf);
      v[i] = __fmul_rn(dec1(b[i]), s);
    }
    return make_uint2(b[0] | (static_cast<unsigned>(b[1]) << 16),
                      b[2] | (static_cast<unsigned>(b[3]) << 16));
  }
  __device__ static void st4(H *p, const Word &w) { *reinterpret_cast<uint2 *>(p) = w; }
};

// ovf may be null (values that are recomputed, not stored, are not counted)
template <>
__device__ __forceinline__ unsigned short Store16<__half>::enc1(float u, unsigned long long *ovf) {
  if (u > 65504.0f || u < -65504.0f) {
    if (ovf) atomicAdd(ovf, 1ull);
    u = u > 0.0f ? 65504.0f : -65504.0f;
  }
  return __half_as_ushort(__float2half_rn(u));
}
template <>
__device__ __forceinline__ float Store16<__half>::dec1(unsigned short b) {
  return __half2float(__ushort_as_half(b));
}
template <>
__device__ __forceinline__ unsigned short Store16<__nv_bfloat16>::enc1(float u, unsigned long long *) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(u));
}
template <>
__device__ __forceinline__ float Store16<__nv_bfloat16>::dec1(unsigned short b) {
  return __bfloat162float(__ushort_as_bfloat16(b));
}

template <>
struct Store<__half> : Store16<__half> {};
template <>
struct Store<__nv_bfloat16> : Store16<__nv_bfloat16> {};

// Shift mapping a bound into [2^13, 2^14): biased exponent of the bound minus
// 140, clamped to [-60, 60] (zero or subnormal bounds take -60).
__host__ __device__ __forceinline__ int store_shift_bits(unsigned bits) {
  const int e8 = static_cast<int>((bits >> 23) & 0xffu);
  const int sh = e8 == 0 ? -60 : e8 - 127 - 13;
  return sh < -60 ? -60 : (sh > 60 ? 60 : sh);
}

}  // namespace wf
