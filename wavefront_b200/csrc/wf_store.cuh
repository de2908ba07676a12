// wf_store.cuh -- field storage formats of the step kernels.
//
// FP32 storage is the reference's own.  The mixed-precision forms store each
// field value v as a 16-bit number u (IEEE binary16 or bfloat16) with
// v = u * 2^shift, where the power-of-two shift belongs to the value's z slab
// (8 planes) and is shared by E and H.  All arithmetic stays FP32 and runs
// in the units of the slab's write shift, so a stored value is its computed
// value rounded to 16 bits with no scaling, and a plane whose read and write
// shifts agree (the steady state) decodes with no scaling either.  Encoding
// is round to nearest even (binary16 saturates finite values at +-65504);
// decoding moves the 16 bits into an FP32 value, exactly, so a kernel that
// rounds a value it has just computed ("round trip") sees exactly the value
// any later reader decodes.  The per-slab shifts are chosen between steps
// from the slab maxima (see k_tail in wf_split.cu).
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
  template <bool SC>
  __device__ static float4 ld4(const float *p, float) { return *reinterpret_cast<const float4 *>(p); }
  template <bool SC>
  __device__ static float ld1(const float *p, float) { return *p; }
  __device__ static float rt(float v) { return v; }
  __device__ static Word enc4(const float v[4]) { return make_float4(v[0], v[1], v[2], v[3]); }
  __device__ static void st4(float *p, const Word &w) { *reinterpret_cast<float4 *>(p) = w; }
};

// Two values per conversion: cvt packs its first operand into the upper
// half of the word.  binary16 saturates finite values at +-65504
// (.satfinite); bfloat16 has FP32's range.
//
// Decoding: bfloat16 is the upper half of an FP32 pattern (a bit move);
// binary16 converts exactly in hardware.  SC: times a power-of-two factor f
// (another slab's or the previous step's units into this plane's).
template <typename H>
struct Store16 {
  static constexpr bool k16 = true;
  static constexpr int PAD = 8;
  using Word = uint2;  // 4 values, x ascending from the low half of .x
  // encode (lo, hi) -> one word (lo in bits 0-15)
  __device__ static unsigned enc2(float lo, float hi);
  // decoded low / high value of a word, and both
  __device__ static float dec_lo(unsigned w);
  __device__ static float dec_hi(unsigned w);
  __device__ static float2 dec2(unsigned w);
  __device__ static float4 dec4(const Word &w) {
    const float2 a = dec2(w.x), b = dec2(w.y);
    return make_float4(a.x, a.y, b.x, b.y);
  }
  // decoded values of 4 stored halves at p (8-byte aligned), times f if SC
  template <bool SC>
  __device__ static float4 ld4(const H *p, float f) {
    float4 v = dec4(*reinterpret_cast<const uint2 *>(p));
    if (SC) v = make_float4(__fmul_rn(v.x, f), __fmul_rn(v.y, f), __fmul_rn(v.z, f), __fmul_rn(v.w, f));
    return v;
  }
  template <bool SC>
  __device__ static float ld1(const H *p, float f) {
    const float v = dec_lo(*reinterpret_cast<const unsigned short *>(p));
    return SC ? __fmul_rn(v, f) : v;
  }
  // the value a reader decodes after v is stored
  __device__ static float rt(float v) { return dec_lo(enc2(v, v)); }
  // the stored word of 4 values
  __device__ static Word enc4(const float v[4]) { return make_uint2(enc2(v[0], v[1]), enc2(v[2], v[3])); }
  __device__ static void st4(H *p, const Word &w) { *reinterpret_cast<uint2 *>(p) = w; }
  // per-half magnitudes (sign bits cleared): non-negative 16-bit floats of
  // one shift order like these integers
  __device__ static unsigned mag(unsigned w) { return w & 0x7fff7fffu; }
};

template <>
__device__ __forceinline__ unsigned Store16<__half>::enc2(float lo, float hi) {
  unsigned r;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
template <>
__device__ __forceinline__ float Store16<__half>::dec_lo(unsigned w) {
  return __half2float(__ushort_as_half(static_cast<unsigned short>(w & 0xffffu)));
}
template <>
__device__ __forceinline__ float Store16<__half>::dec_hi(unsigned w) {
  return __half2float(__ushort_as_half(static_cast<unsigned short>(w >> 16)));
}
template <>
__device__ __forceinline__ float2 Store16<__half>::dec2(unsigned w) {
  return __half22float2(*reinterpret_cast<const __half2 *>(&w));  // one conversion per half
}
template <>
__device__ __forceinline__ unsigned Store16<__nv_bfloat16>::enc2(float lo, float hi) {
  unsigned r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
template <>
__device__ __forceinline__ float Store16<__nv_bfloat16>::dec_lo(unsigned w) {
  return __uint_as_float(w << 16);
}
template <>
__device__ __forceinline__ float Store16<__nv_bfloat16>::dec_hi(unsigned w) {
  return __uint_as_float(w & 0xffff0000u);
}
template <>
__device__ __forceinline__ float2 Store16<__nv_bfloat16>::dec2(unsigned w) {
  return make_float2(dec_lo(w), dec_hi(w));
}

template <>
struct Store<__half> : Store16<__half> {};
template <>
struct Store<__nv_bfloat16> : Store16<__nv_bfloat16> {};

// Shift mapping a bound into [2^13, 2^14): biased exponent of the bound minus
// 140, clamped to [-60, 15] (zero or subnormal bounds take -60), so every
// factor 2^(a - b) between two shifts is an FP32 normal.
__host__ __device__ __forceinline__ int store_shift_bits(unsigned bits) {
  const int e8 = static_cast<int>((bits >> 23) & 0xffu);
  const int sh = e8 == 0 ? -60 : e8 - 127 - 13;
  return sh < -60 ? -60 : (sh > 15 ? 15 : sh);
}

}  // namespace wf
