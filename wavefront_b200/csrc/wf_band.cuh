// wf_band.cuh -- device helpers shared by the closure's band kernels: the
// mapping between a face band's coordinates and the grid's cells, the tile
// of the transposing band copies, and the split of FP32 values into the
// three bfloat16 parts of the packed MMA operand.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "wf_closure.h"

namespace wf {

// Cell (x, y, z) of band coordinates (d, u, v) of face f (axis f/2, side f%2).
__device__ __forceinline__ void band_cell(const BandGrid &g, int f, int d, int u, int v, int &x,
                                          int &y, int &z) {
  const int ax = f >> 1;
  const int n = ax == 0 ? g.nx : (ax == 1 ? g.ny : g.nz);
  const int c = (f & 1) ? n - 1 - d : d;
  if (ax == 0) { x = c; y = u; z = v; }
  else if (ax == 1) { x = u; y = c; z = v; }
  else { x = u; y = v; z = c; }
}

// The psi slot index of cell (x, y, z) on axis `ax`, or -1 outside its slab.
__device__ __forceinline__ long long psi_index(const BandGrid &g, int ax, int x, int y, int z) {
  const BandPsi &P = g.psi[ax];
  if (P.T <= 0) return -1;
  const int n = ax == 0 ? g.nx : (ax == 1 ? g.ny : g.nz);
  const int c = ax == 0 ? x : (ax == 1 ? y : z);
  int s = -1;
  if (c < P.T) s = c;
  else if (c >= n - P.T) s = c - (n - P.W);
  if (s < 0) return -1;
  if (ax == 0) return (static_cast<long long>(z) * g.ny + y) * P.pitch + s;
  if (ax == 1) return (static_cast<long long>(z) * P.W + s) * g.nx + x;
  return (static_cast<long long>(s) * g.ny + y) * g.nx + x;
}

// The band copies move every cell between the grid (x fastest) and the band
// tensors (v fastest), two layouts whose unit-stride axes differ on every face:
// the grid's x is the band's depth d on the x faces and u on the y and z
// faces.  Each CTA therefore stages a tile in shared memory and reads and
// writes both sides along their own unit stride: TA cells along the band axis
// that is x in the grid, 32 along v, TO along the third band axis.
template <int AX>
struct BandTile {
  static constexpr int TA = AX == 0 ? kBandDepth : 32;  // along the grid's x
  static constexpr int TO = AX == 0 ? 4 : 1;            // along the third axis
  static constexpr int kElems = TA * 32 * TO;           // 1024: 4 per thread
  static constexpr int kZ = AX == 0 ? 1 : kBandDepth;   // CTAs along z per face
};
static_assert(BandTile<0>::kElems == 1024 && BandTile<1>::kElems == 1024, "band tile size");

// Band coordinates (d, u) of tile element (a, o) of CTA (by, sub).
template <int AX>
__device__ __forceinline__ void band_du(int al, int ol, int by, int sub, int &d, int &u) {
  if (AX == 0) {
    d = al;
    u = by * BandTile<0>::TO + ol;
  } else {
    d = sub;
    u = by * 32 + al;
  }
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

}  // namespace wf
