// wf_fused_impl.cuh -- one-pass fused H->E Yee step for sm_100a, templated on
// the field storage type (float; __half and __nv_bfloat16 for the
// mixed-precision forms, see wf_store.cuh).  wf_fused.cu and wf_fused16.cu
// instantiate it.
//
// Replaces, for zero-field boundaries, one whole step_all_slabs call of the
// reference (src/engine.rs:291-422: an H phase over every 8^3 block with
// update_h_field[_pml], a barrier, then an E phase with update_e_field[_pml])
// with a single kernel in which every field value crosses HBM once:
//
//  * a CTA owns a 128 x TY column of cells and marches it through a chunk of
//    z planes;
//  * plane p's E box (tile + 1-cell halo), H box (tile + -x/-y halo) and the
//    material-id box are staged into shared memory by TMA
//    (cp.async.bulk.tensor, no multicast) through an S-deep mbarrier ring;
//    out-of-domain box cells arrive as zeros, which is exactly the
//    reference's OUTER_ZERO_BLOCK (src/engine.rs:83);
//  * H of plane p is computed for the tile plus the -x column and -y row
//    the E update needs (recomputed, never exchanged between CTAs), E of
//    plane p follows at once from registers and a shared-memory H plane;
//    the -z neighbour H(p-1) rides along in registers (register-rotated z);
//  * the state is double-buffered: the kernel reads buffer `cur` and writes
//    buffer `nxt`, so halo recomputation never races a neighbour's writes;
//  * CPML: interior CTAs run a body with no CPML code.  CTAs whose tile,
//    halo or z chunk meets a graded slab treat each lane's 4 cells as one
//    vector: the y and z slab flags are uniform per warp and per plane, the
//    x slab flag per lane, psi moves as float4, and each phase's psi loads
//    are issued before the work that precedes their use (the H terms before
//    the stage wait, the E terms before the barrier) so their latency
//    overlaps it.
//
// All per-cell arithmetic goes through wf_internal.cuh, so results are
// bit-identical to the split kernels and to the reference.
//
// 16-bit storage: a plane computes in the units of its slab's write shift
// w.  Staged values are decoded into those units (a power-of-two factor only
// where the read shift differs: a slab whose shift changed, or plane p+1 in
// the next slab), H(p-1) is rescaled once when p enters a new slab, and psi
// stays in field units (raw differences enter the recursion times 2^w and
// leave it times 2^-w).  Every H value computed (tile, halo row and column,
// warm-up plane) is rounded through the storage format before any use,
// exactly as if it had been stored and re-read, and E values are rounded as
// they are stored.  Each warp keeps the largest stored magnitude per slab
// and kind and folds it into the slab maxima (one atomic per warp and slab).
#pragma once

#include <algorithm>
#include <type_traits>

#include "wf_internal.cuh"
#include "wf_launch.h"
#include "wf_store.cuh"

namespace wf {

namespace {

constexpr int kProfSmem = 3 * 3 * 64;  // floats: 3 axes x {b, a, 1/kappa} x 64 positions

// Box x extents start PAD elements left of the tile (PAD = 16 bytes, the TMA
// x alignment): E x0-PAD..x0+TW+PAD-1, H x0-PAD..x0+TW-1.  A tile is TW = 4*LX
// cells wide (LX lanes per row, 4 cells each) and TY rows tall: the wide
// tiles have LX = 32 (one row per warp), the x-CPML column tiles LX = 4
// (eight rows per warp).
template <int TY, int S, typename ST, int LX = 32>
struct Layout {
  static constexpr int PAD = Store<ST>::PAD;
  static constexpr int TW = 4 * LX;
  static constexpr int RW = 32 / LX;  // rows per tile warp
  static constexpr int EW = TW + 2 * PAD, EH = TY + 2;  // E box rows y0-1..y0+TY
  static constexpr int HW = TW + PAD, HH = TY + 1;      // H box rows y0-1..y0+TY-1
  // ids: the box starts at (x0-16) rounded down to 16 (u8 TMA x alignment):
  // x0-16 for the wide tiles (x0 a multiple of 16), x0-16 or x0-24 for a
  // column tile at nx-16 (nx a multiple of 8)
  static constexpr int MW = LX == 32 ? TW + 16 : TW + 32, MH = TY + 1;
  static constexpr int E_BYTES = 3 * EH * EW * static_cast<int>(sizeof(ST));
  static constexpr int H_BYTES = 3 * HH * HW * static_cast<int>(sizeof(ST));
  static constexpr int M_BYTES = MH * MW;
  static constexpr int al(int v) { return (v + 127) / 128 * 128; }
  static constexpr int H_OFF = al(E_BYTES);
  static constexpr int M_OFF = H_OFF + al(H_BYTES);
  static constexpr int STAGE = M_OFF + al(M_BYTES);
  static constexpr int STAGE_OFF = 4096;  // after the 256-entry float4 coefficient table
  static constexpr int PROWS = TY + 1;    // plane rows: 0 = y0-1, 1..TY = tile rows
  static constexpr int HALO = TY + 1 <= 32 ? 32 : 64;  // x-halo column entries (rows 1..TY)
  static constexpr int PLANE_FLOATS = 2 * PROWS * TW + 2 * HALO;  // hz, hx rows; x-halo hz, hy
  static constexpr int PLANE_OFF = STAGE_OFF + S * STAGE;
  static constexpr int PROF_OFF = PLANE_OFF + 2 * PLANE_FLOATS * 4;  // CPML profiles
  static constexpr int BAR_OFF = PROF_OFF + kProfSmem * 4;
  static constexpr int BYTES = BAR_OFF + S * 8 + 128;  // +128: base alignment slack
  static constexpr int THREADS = 32 * (TY / RW + 1);  // tile warps + the halo warp
  static_assert(TY % RW == 0, "whole tile warps");
  static_assert(TY <= 32, "x-halo column is handled by one warp");
};

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void stg4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float &el(float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ float comp(const float4 &v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

// CPML geometry of one lane's 4 cells at one plane.
struct LanePml {
  bool y, z;        // row in the y slab / plane in the z slab (warp / CTA uniform)
  int xmode;        // 0: no cell in the x slab; 1: all 4, aligned (vector); 2: per cell
  long long iy, iz, ix;  // psi index of the lane's first cell (y, z, x-vector)
  int sy, sz, sx;        // slab positions (x: of the first cell)
};

// The plane-independent part of a lane's CPML geometry (computed once per
// CTA): its x-slab mode and position, and its row's y-slab position.
struct LaneConst {
  int xmode, sx, sy;
};

// AX: bit mask of the CPML axes (1 x, 2 y, 4 z) the calling kernel handles.
template <int AX>
__device__ __forceinline__ LaneConst lane_const(const GridArgs &g, int xg, int y, bool cell_ok) {
  LaneConst c{0, -1, -1};
  if (!cell_ok) return c;
  const PmlAxis &X = g.pml[0], &Y = g.pml[1];
  if (AX & 2) c.sy = slab_pos(y, g.ny, Y.T, Y.W);
  if ((AX & 1) && X.T > 0) {
    const int s0 = slab_pos(xg, g.nx, X.T, X.W), s3 = slab_pos(xg + 3, g.nx, X.T, X.W);
    const int s1 = slab_pos(xg + 1, g.nx, X.T, X.W), s2 = slab_pos(xg + 2, g.nx, X.T, X.W);
    if (s0 >= 0 && s3 == s0 + 3 && (s0 & 3) == 0) {
      c.xmode = 1;
      c.sx = s0;
    } else if (s0 >= 0 || s1 >= 0 || s2 >= 0 || s3 >= 0) {
      c.xmode = 2;
    }
  }
  return c;
}

template <int AX>
__device__ __forceinline__ LanePml lane_pml(const GridArgs &g, const LaneConst &c, int xg, int y,
                                            int p) {
  LanePml L{};
  if (AX & 2) {
    L.sy = c.sy;
    L.y = c.sy >= 0;
    if (L.y) L.iy = (static_cast<long long>(p) * g.pml[1].W + c.sy) * g.nx + xg;
  }
  if (AX & 4) {
    const PmlAxis &Z = g.pml[2];
    L.sz = slab_pos(p, g.nz, Z.T, Z.W);
    L.z = L.sz >= 0;
    if (L.z) L.iz = (static_cast<long long>(L.sz) * g.ny + y) * g.nx + xg;
  }
  if (AX & 1) {
    L.xmode = c.xmode;
    L.sx = c.sx;
    if (c.xmode == 1) L.ix = (static_cast<long long>(p) * g.ny + y) * g.pml[0].pitch + c.sx;
  }
  return L;
}

// The two psi terms of one axis for a lane's 4 cells (float4 each).
struct Psi2 {
  float4 p0, p1;
};

// The H-term psi of the -x halo cell on each axis (slab position, or -1).
struct HaloPsi {
  int sx, sy, sz;
  float x0, x1, y0, y1, z0, z1;
};

__device__ __forceinline__ Psi2 load_psi2(const PmlAxis &P, int comp0, long long idx, int *err) {
  if (!idx_ok(err, idx + 3, P.cells)) return Psi2{};
  return Psi2{ldg4(P.psi_cur + comp0 * P.cells + idx), ldg4(P.psi_cur + (comp0 + 1) * P.cells + idx)};
}

// float4 store of psi components comp0 at idx (checked in bounds-checked builds)
__device__ __forceinline__ void store_psi4(const PmlAxis &P, int comp, long long idx, float4 v,
                                           int *err) {
  if (idx_ok(err, idx + 3, P.cells)) stg4(P.psi_nxt + comp * P.cells + idx, v);
}

// Computing units <-> field units of psi: 16-bit storage (U) computes in
// units of 2^w (su = 2^w, iu = 2^-w) and keeps psi in field units, so a raw
// difference enters the recursion times su and its result leaves times iu
// (both exact).
struct Units {
  float su, iu;
};
template <bool FMA, bool U>
__device__ __forceinline__ float corr_u(float raw, float b, float a, float ik, float &psi, Units u) {
  if (!U) return pml_corr<FMA>(raw, b, a, ik, psi);
  return __fmul_rn(pml_corr<FMA>(__fmul_rn(raw, u.su), b, a, ik, psi), u.iu);
}

// psi recursion of one axis over 4 cells with one coefficient set (y, z).
template <bool FMA, bool U>
__device__ __forceinline__ void corr4_uniform(float d0[4], float d1[4], Psi2 &q, float b, float a,
                                              float ik, Units u) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    d0[i] = corr_u<FMA, U>(d0[i], b, a, ik, el(q.p0, i), u);
    d1[i] = corr_u<FMA, U>(d1[i], b, a, ik, el(q.p1, i), u);
  }
}

// CPML profiles (b, a, 1/kappa at slab positions) as the body reads them:
// a shared-memory copy when every axis's slab fits kProfCap positions,
// otherwise the global arrays.
constexpr int kProfCap = kProfSmem / 9;
struct Prof {
  const float *p;  // shared memory: [3 axes][b, a, 1/kappa][kProfCap]
  __device__ __forceinline__ float b(int ax, int s) const { return p[ax * 3 * kProfCap + s]; }
  __device__ __forceinline__ float a(int ax, int s) const { return p[(ax * 3 + 1) * kProfCap + s]; }
  __device__ __forceinline__ float ik(int ax, int s) const { return p[(ax * 3 + 2) * kProfCap + s]; }
};

// x axis: per-cell coefficients at slab positions s0..s0+3.
template <bool FMA, bool U>
__device__ __forceinline__ void corr4_x(float d0[4], float d1[4], Psi2 &q, const Prof &pf, int s0,
                                        Units u) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float b = pf.b(0, s0 + i), a = pf.a(0, s0 + i), ik = pf.ik(0, s0 + i);
    d0[i] = corr_u<FMA, U>(d0[i], b, a, ik, el(q.p0, i), u);
    d1[i] = corr_u<FMA, U>(d1[i], b, a, ik, el(q.p1, i), u);
  }
}

// x axis, one cell at a time (lanes straddling a slab edge).
template <bool FMA, bool U>
__device__ __forceinline__ void corr_x_cell(const GridArgs &g, const Prof &pf, int comp0, int x,
                                            int y, int p, float &d0, float &d1, bool store, Units u) {
  const PmlAxis &P = g.pml[0];
  const int s = slab_pos(x, g.nx, P.T, P.W);
  if (s < 0) return;
  const long long idx = (static_cast<long long>(p) * g.ny + y) * P.pitch + s;
  if (!idx_ok(g.err, idx, P.cells)) return;
  float p0 = __ldg(P.psi_cur + comp0 * P.cells + idx), p1 = __ldg(P.psi_cur + (comp0 + 1) * P.cells + idx);
  const float b = pf.b(0, s), a = pf.a(0, s), ik = pf.ik(0, s);
  d0 = corr_u<FMA, U>(d0, b, a, ik, p0, u);
  d1 = corr_u<FMA, U>(d1, b, a, ik, p1, u);
  if (store) {
    P.psi_nxt[comp0 * P.cells + idx] = p0;
    P.psi_nxt[(comp0 + 1) * P.cells + idx] = p1;
  }
}

// AX: the CPML axes this body handles (bit 1 x, 2 y, 4 z; 0 = interior).
// The tile's cells are x in [x0, x_end), y in [y0, y0+TY), z in [k0, k1).
template <int TY, int S, bool FMA, int AX, typename ST, int LX = 32>
__device__ __forceinline__ void fused_body(const CUtensorMap *tmE, const CUtensorMap *tmH,
                                           const CUtensorMap *tmM, const FusedArgs &a,
                                           unsigned char *smem, int x0, int y0, int k0, int k1,
                                           int x_end) {
  using L = Layout<TY, S, ST, LX>;
  constexpr int TW = L::TW;
  using SD = Store<ST>;
  constexpr int PAD = L::PAD;
  constexpr bool PML = AX != 0;
  constexpr bool AXX = (AX & 1) != 0, AXY = (AX & 2) != 0, AXZ = (AX & 4) != 0;
  const GridArgs &g = a.g;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float4 *s_coef = reinterpret_cast<const float4 *>(smem);
  unsigned char *s_stage = smem + L::STAGE_OFF;
  float *s_plane = reinterpret_cast<float *>(smem + L::PLANE_OFF);
  uint64_t *s_bar = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);

  const int nx = g.nx, ny = g.ny;
  const long long N = g.N;
  const int moff = x0 - ((x0 - 16) & ~15);  // column of x0 in the ids box (16 or 24)
  const int kfirst = k0 > 0 ? k0 - 1 : 0;  // k0-1: warm-up plane for H(k0-1)
  const int np = k1 - kfirst + 1;          // planes staged; plane k1 brings only E

  auto issue = [&](int j) {
    const int p = kfirst + j;
    const int slot = j % S;
    unsigned char *st = s_stage + slot * L::STAGE;
    const uint32_t bar = smem_u32(&s_bar[slot]);
    const bool e_only = (p == k1);
    // (a nonzero test_extra_tx leaves stage 0's phase incomplete after its
    // copies land, so its bounded wait runs out: the timeout path, tested)
    mbar_expect_tx(bar, (e_only ? L::E_BYTES : (L::E_BYTES + L::H_BYTES + L::M_BYTES)) +
                            (j == 0 ? static_cast<uint32_t>(a.test_extra_tx) : 0u));
    tma_load_4d(smem_u32(st), tmE, x0 - PAD, y0 - 1, p, 0, bar);
    if (!e_only) {
      tma_load_4d(smem_u32(st + L::H_OFF), tmH, x0 - PAD, y0 - 1, p, 3, bar);
      tma_load_3d(smem_u32(st + L::M_OFF), tmM, x0 - moff, y0 - 1, p, bar);
    }
  };

  int issued = 0;
  if (tid == 0) {
    const int pro = np < S ? np : S;
    for (int j = 0; j < pro; ++j) issue(j);
    issued = pro;
  }
  bool ok = mbar_wait(smem_u32(&s_bar[0]), 0);
  int done = ok ? 1 : 0;  // stages [0, done) seen complete, in order

  // tile warps hold L::RW rows of LX lanes each; the halo warp computes the
  // -y halo row (every lane, col = lane % LX: lanes of the same col compute
  // the same cells) and the -x halo column (lanes 0..TY-1)
  const bool tile_warp = warp < TY / L::RW;
  const int col = lane % LX;
  const int r = tile_warp ? warp * L::RW + lane / LX + 1 : 0;  // smem row: 0 is y0-1
  const int y = y0 - 1 + r;
  const int xg = x0 + 4 * col;
  const bool row_in = (y >= 0) && (y < ny);
  const bool x_in = xg < x_end;  // x_end % 4 == 0: a lane's 4 cells are all in or all out
  const bool cell_ok = row_in && x_in;
  const int cE = PAD + 4 * col;
  float4 hxp = make_float4(0.f, 0.f, 0.f, 0.f), hyp = hxp;  // H(p-1), own cells
  // E(p+1) of the own row as decoded for plane p's z differences: plane p+1's
  // own ex, ey when the warp worked on plane p and p+1 is in the same slab
  float4 ex_nx = hxp, ey_nx = hxp;
  bool have_nx = false;
  ST *const nxt = reinterpret_cast<ST *>(g.nxt);
  // 16-bit storage: this thread's largest stored E, H magnitudes in slab
  // sl_c (two 16-bit lanes each, compared as integers: one shift per slab),
  // that slab's write shift w_c, and the unit factors of the plane: fC
  // (plane p's stored values into units of 2^w_c), fN (plane p+1's) and su,
  // iu (field units <-> computing units)
  unsigned mxE = 0, mxH = 0;
  int sl_c = -1, w_c = 0;
  float fC = 1.0f, fN = 1.0f;
  Units un{1.0f, 1.0f};
  auto flush_max = [&]() {
    if constexpr (SD::k16) {
      const unsigned e = __reduce_max_sync(0xffffffffu, max(mxE & 0xffffu, mxE >> 16));
      const unsigned h = __reduce_max_sync(0xffffffffu, max(mxH & 0xffffu, mxH >> 16));
      if (lane == 0 && e)
        atomicMax(g.slab_max + 2 * sl_c, __float_as_uint(__fmul_rn(SD::dec_lo(e), un.su)));
      if (lane == 0 && h)
        atomicMax(g.slab_max + 2 * sl_c + 1, __float_as_uint(__fmul_rn(SD::dec_lo(h), un.su)));
      mxE = mxH = 0;
    }
  };

  const Prof pf{reinterpret_cast<const float *>(smem + L::PROF_OFF)};
  const LaneConst lc = lane_const<AX>(g, xg, y, cell_ok);
  // CPML: each plane's H-term psi is loaded one plane ahead (the first plane's
  // here), so its latency hides behind a whole plane of work.
  LanePml lp_n{};
  Psi2 qx_n{}, qy_n{}, qz_n{};
  auto prefetch = [&](int pp) {
    lp_n = lane_pml<AX>(g, lc, xg, y, pp);
    if (AXY && lp_n.y) qy_n = load_psi2(g.pml[1], 0, lp_n.iy, g.err);
    if (AXZ && lp_n.z) qz_n = load_psi2(g.pml[2], 0, lp_n.iz, g.err);
    if (AXX && lp_n.xmode == 1) qx_n = load_psi2(g.pml[0], 0, lp_n.ix, g.err);
  };
  // ... and so is the H-term psi of the -x halo cell (x0-1, y0+lane) that
  // lanes 0..TY-1 of the halo warp update.
  const bool xhalo = PML && !tile_warp && lane < TY && x0 > 0 && y0 + lane < ny;
  HaloPsi hh_n{-1, -1, -1, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  auto prefetch_halo = [&](int pp) {
    const int xh = x0 - 1, yh = y0 + lane;
    if (AXX) {
      const PmlAxis &P = g.pml[0];
      hh_n.sx = slab_pos(xh, nx, P.T, P.W);
      if (hh_n.sx >= 0) {
        const long long i = (static_cast<long long>(pp) * ny + yh) * P.pitch + hh_n.sx;
        if (idx_ok(g.err, i, P.cells)) {
          hh_n.x0 = __ldg(P.psi_cur + i);
          hh_n.x1 = __ldg(P.psi_cur + P.cells + i);
        }
      }
    }
    if (AXY) {
      const PmlAxis &P = g.pml[1];
      hh_n.sy = slab_pos(yh, ny, P.T, P.W);
      if (hh_n.sy >= 0) {
        const long long i = (static_cast<long long>(pp) * P.W + hh_n.sy) * nx + xh;
        if (idx_ok(g.err, i, P.cells)) {
          hh_n.y0 = __ldg(P.psi_cur + i);
          hh_n.y1 = __ldg(P.psi_cur + P.cells + i);
        }
      }
    }
    if (AXZ) {
      const PmlAxis &P = g.pml[2];
      hh_n.sz = slab_pos(pp, g.nz, P.T, P.W);
      if (hh_n.sz >= 0) {
        const long long i = (static_cast<long long>(hh_n.sz) * ny + yh) * nx + xh;
        if (idx_ok(g.err, i, P.cells)) {
          hh_n.z0 = __ldg(P.psi_cur + i);
          hh_n.z1 = __ldg(P.psi_cur + P.cells + i);
        }
      }
    }
  };
  if (PML && cell_ok) prefetch(kfirst);
  if (xhalo) prefetch_halo(kfirst);

  for (int j = 0; j < np - 1; ++j) {
    const int p = kfirst + j;
    const bool warm = p < k0;
    const bool active = tile_warp || !warm;  // the halo warp idles on the warm-up plane
    const LanePml lp = lp_n;
    Psi2 qx = qx_n, qy = qy_n, qz = qz_n;
    HaloPsi hh = hh_n;  // (pml_corr updates its psi argument in place)

    if constexpr (SD::k16) {
      const int sl = p / kSlabPlanes;
      if (sl != sl_c) {
        const int w = __ldg(g.shift_wr + 2 * sl);
        if (sl_c >= 0) {
          flush_max();
          if (w != w_c) {  // H(p-1), computed in the previous slab's units
            const float f = pow2f(w_c - w);
            hxp = make_float4(__fmul_rn(hxp.x, f), __fmul_rn(hxp.y, f), __fmul_rn(hxp.z, f),
                              __fmul_rn(hxp.w, f));
            hyp = make_float4(__fmul_rn(hyp.x, f), __fmul_rn(hyp.y, f), __fmul_rn(hyp.z, f),
                              __fmul_rn(hyp.w, f));
          }
        }
        sl_c = sl;
        w_c = w;
        un = Units{pow2f(w), pow2f(-w)};
        fC = pow2f(__ldg(g.shift_rd + 2 * sl) - w);
      }
      const int sln = min((p + 1) / kSlabPlanes, g.nslab - 1);
      fN = sln == sl ? fC : pow2f(__ldg(g.shift_rd + 2 * sln) - w_c);
    }

    const bool arrived = mbar_wait(smem_u32(&s_bar[(j + 1) % S]), ((j + 1) / S) & 1);
    if (arrived && done == j + 1) done = j + 2;
    ok = arrived && ok;
    const unsigned char *stc = s_stage + (j % S) * L::STAGE;
    const ST *Ec = reinterpret_cast<const ST *>(stc);
    const ST *En = reinterpret_cast<const ST *>(s_stage + ((j + 1) % S) * L::STAGE);
    const ST *Hc = reinterpret_cast<const ST *>(stc + L::H_OFF);
    const uint8_t *Mc = stc + L::M_OFF;
    float *pl = s_plane + (p & 1) * L::PLANE_FLOATS;
    float *pl_hz = pl, *pl_hx = pl + L::PROWS * TW;
    float *pl_hzh = pl + 2 * L::PROWS * TW, *pl_hyh = pl_hzh + L::HALO;

    // ---------------- H phase (update_h_field[_pml], src/fdtd.rs:194-345) ----
    float ha[4], hb[4], hc[4];  // new hx, hy, hz of this lane's 4 cells
    float4 ex4, ey4, ez4;
    uchar4 m4;
    Psi2 ex_{}, ey_{}, ez_{};  // E-term psi (x, y, z axes), loaded before the barrier
    if (active) {
      // the staged values in computing units (SC: times fC / fN)
      float4 ex_py, ez_py, ex_pz, ey_pz, hx4, hy4, hz4;
      auto load = [&](auto sc) {
        constexpr bool SC = decltype(sc)::value;
        auto E4 = [&](const ST *B, int c, int row, float f) {
          return SD::template ld4<SC>(B + (c * L::EH + row) * L::EW + cE, f);
        };
        if (have_nx && (!SD::k16 || p % kSlabPlanes != 0)) {
          ex4 = ex_nx;
          ey4 = ey_nx;
        } else {
          ex4 = E4(Ec, 0, r, fC);
          ey4 = E4(Ec, 1, r, fC);
        }
        ez4 = E4(Ec, 2, r, fC);
        ex_py = E4(Ec, 0, r + 1, fC);
        ez_py = E4(Ec, 2, r + 1, fC);
        ex_pz = E4(En, 0, r, fN);
        ey_pz = E4(En, 1, r, fN);
        hx4 = SD::template ld4<SC>(Hc + (0 * L::HH + r) * L::HW + cE, fC);
        hy4 = SD::template ld4<SC>(Hc + (1 * L::HH + r) * L::HW + cE, fC);
        hz4 = SD::template ld4<SC>(Hc + (2 * L::HH + r) * L::HW + cE, fC);
      };
      if constexpr (SD::k16) {
        if (fC != 1.0f || fN != 1.0f)
          load(std::true_type{});
        else
          load(std::false_type{});
      } else {
        load(std::false_type{});
      }
      ex_nx = ex_pz;
      ey_nx = ey_pz;
      float ez_n = __shfl_down_sync(0xffffffffu, ez4.x, 1);
      float ey_n = __shfl_down_sync(0xffffffffu, ey4.x, 1);
      if (col == LX - 1) {
        ez_n = SD::template ld1<SD::k16>(Ec + (2 * L::EH + r) * L::EW + PAD + TW, fC);
        ey_n = SD::template ld1<SD::k16>(Ec + (1 * L::EH + r) * L::EW + PAD + TW, fC);
      }
      m4 = *reinterpret_cast<const uchar4 *>(Mc + r * L::MW + moff + 4 * col);

      float d_ez_dy[4], d_ex_dy[4], d_ey_dz[4], d_ex_dz[4], d_ez_dx[4], d_ey_dx[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        d_ez_dy[q] = sub(comp(ez_py, q), comp(ez4, q));
        d_ex_dy[q] = sub(comp(ex_py, q), comp(ex4, q));
        d_ey_dz[q] = sub(comp(ey_pz, q), comp(ey4, q));
        d_ex_dz[q] = sub(comp(ex_pz, q), comp(ex4, q));
        d_ez_dx[q] = sub(q < 3 ? comp(ez4, q + 1) : ez_n, comp(ez4, q));
        d_ey_dx[q] = sub(q < 3 ? comp(ey4, q + 1) : ey_n, comp(ey4, q));
      }
      if (PML && cell_ok) {  // CPML on the H terms (pml_correct_*, src/fdtd.rs:136-163)
        const bool wpsi = tile_warp && !warm;
        if (AXX && lp.xmode == 1) {
          corr4_x<FMA, SD::k16>(d_ez_dx, d_ey_dx, qx, pf, lp.sx, un);
          if (wpsi) {
            store_psi4(g.pml[0], 0, lp.ix, qx.p0, g.err);
            store_psi4(g.pml[0], 1, lp.ix, qx.p1, g.err);
          }
        } else if (AXX && lp.xmode == 2) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            corr_x_cell<FMA, SD::k16>(g, pf, 0, xg + q, y, p, d_ez_dx[q], d_ey_dx[q], wpsi, un);
        }
        if (AXY && lp.y) {
          corr4_uniform<FMA, SD::k16>(d_ez_dy, d_ex_dy, qy, pf.b(1, lp.sy), pf.a(1, lp.sy),
                                      pf.ik(1, lp.sy), un);
          if (wpsi) {
            store_psi4(g.pml[1], 0, lp.iy, qy.p0, g.err);
            store_psi4(g.pml[1], 1, lp.iy, qy.p1, g.err);
          }
        }
        if (AXZ && lp.z) {
          corr4_uniform<FMA, SD::k16>(d_ey_dz, d_ex_dz, qz, pf.b(2, lp.sz), pf.a(2, lp.sz),
                                      pf.ik(2, lp.sz), un);
          if (wpsi) {
            store_psi4(g.pml[2], 0, lp.iz, qz.p0, g.err);
            store_psi4(g.pml[2], 1, lp.iz, qz.p1, g.err);
          }
        }
        if (wpsi) {  // the E terms' psi: in flight across the barrier
          if (AXX && lp.xmode == 1) ex_ = load_psi2(g.pml[0], 2, lp.ix, g.err);
          if (AXY && lp.y) ey_ = load_psi2(g.pml[1], 2, lp.iy, g.err);
          if (AXZ && lp.z) ez_ = load_psi2(g.pml[2], 2, lp.iz, g.err);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const unsigned char id = q == 0 ? m4.x : (q == 1 ? m4.y : (q == 2 ? m4.z : m4.w));
        const float4 cf = s_coef[id];
        ha[q] = h_new<FMA>(cf.z, comp(hx4, q), cf.w, sub(d_ez_dy[q], d_ey_dz[q]));
        hb[q] = h_new<FMA>(cf.z, comp(hy4, q), cf.w, sub(d_ex_dz[q], d_ez_dx[q]));
        hc[q] = h_new<FMA>(cf.z, comp(hz4, q), cf.w, sub(d_ey_dx[q], d_ex_dy[q]));
      }
      if (!row_in) {  // outside the domain in y: zero field (OUTER_ZERO_BLOCK)
#pragma unroll
        for (int q = 0; q < 4; ++q) ha[q] = hb[q] = hc[q] = 0.0f;
      }
      // every H value is used as stored (16-bit: rounded here, in place)
      const bool hstore = !warm && tile_warp && cell_ok;
      const typename SD::Word wa = SD::enc4(ha);
      const typename SD::Word wb = SD::enc4(hb);
      const typename SD::Word wc = SD::enc4(hc);
      if constexpr (SD::k16) {
        const float4 da = SD::dec4(wa), db = SD::dec4(wb), dc = SD::dec4(wc);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ha[q] = comp(da, q);
          hb[q] = comp(db, q);
          hc[q] = comp(dc, q);
        }
      }
      if (!warm) {
        stg4(pl_hz + r * TW + 4 * col, make_float4(hc[0], hc[1], hc[2], hc[3]));
        stg4(pl_hx + r * TW + 4 * col, make_float4(ha[0], ha[1], ha[2], ha[3]));
        const long long hcell = (static_cast<long long>(p) * ny + y) * nx + xg;
        if (hstore && idx_ok(g.err, hcell + 3, N)) {
          ST *Hn = nxt + 3 * N + hcell;
          SD::st4(Hn, wa);
          SD::st4(Hn + N, wb);
          SD::st4(Hn + 2 * N, wc);
          if constexpr (SD::k16) {
            mxH = __vmaxu2(mxH, __vmaxu2(__vmaxu2(SD::mag(wa.x), SD::mag(wa.y)),
                                         __vmaxu2(__vmaxu2(SD::mag(wb.x), SD::mag(wb.y)),
                                                  __vmaxu2(SD::mag(wc.x), SD::mag(wc.y)))));
          }
        }
      }
      // -x halo column (x0-1, y0..y0+TY-1): Hz and Hy for the E update at x0
      if (!tile_warp && !warm && lane < TY) {
        const int rh = lane + 1, yh = y0 + lane;
        float hzv = 0.0f, hyv = 0.0f;
        if (x0 > 0 && yh < ny) {
          auto Ev = [&](const ST *B, int c, int row, int col, float f) {
            return SD::template ld1<SD::k16>(B + (c * L::EH + row) * L::EW + col, f);
          };
          const float ex = Ev(Ec, 0, rh, PAD - 1, fC);
          const float ey = Ev(Ec, 1, rh, PAD - 1, fC);
          const float ez = Ev(Ec, 2, rh, PAD - 1, fC);
          float d_ez_dx1 = sub(Ev(Ec, 2, rh, PAD, fC), ez);
          float d_ey_dx1 = sub(Ev(Ec, 1, rh, PAD, fC), ey);
          float d_ex_dz1 = sub(Ev(En, 0, rh, PAD - 1, fN), ex);
          float d_ey_dz1 = sub(Ev(En, 1, rh, PAD - 1, fN), ey);
          float d_ex_dy1 = sub(Ev(Ec, 0, rh + 1, PAD - 1, fC), ex);
          float d_ez_dy1 = sub(Ev(Ec, 2, rh + 1, PAD - 1, fC), ez);
          constexpr bool U = SD::k16;
          if (AXX && hh.sx >= 0) {
            const float b = pf.b(0, hh.sx), a_ = pf.a(0, hh.sx), ik = pf.ik(0, hh.sx);
            d_ez_dx1 = corr_u<FMA, U>(d_ez_dx1, b, a_, ik, hh.x0, un);
            d_ey_dx1 = corr_u<FMA, U>(d_ey_dx1, b, a_, ik, hh.x1, un);
          }
          if (AXY && hh.sy >= 0) {
            const float b = pf.b(1, hh.sy), a_ = pf.a(1, hh.sy), ik = pf.ik(1, hh.sy);
            d_ez_dy1 = corr_u<FMA, U>(d_ez_dy1, b, a_, ik, hh.y0, un);
            d_ex_dy1 = corr_u<FMA, U>(d_ex_dy1, b, a_, ik, hh.y1, un);
          }
          if (AXZ && hh.sz >= 0) {
            const float b = pf.b(2, hh.sz), a_ = pf.a(2, hh.sz), ik = pf.ik(2, hh.sz);
            d_ey_dz1 = corr_u<FMA, U>(d_ey_dz1, b, a_, ik, hh.z0, un);
            d_ex_dz1 = corr_u<FMA, U>(d_ex_dz1, b, a_, ik, hh.z1, un);
          }
          const float4 cf = s_coef[Mc[rh * L::MW + moff - 1]];
          auto Hv = [&](int c) {
            return SD::template ld1<SD::k16>(Hc + (c * L::HH + rh) * L::HW + PAD - 1, fC);
          };
          hyv = SD::rt(h_new<FMA>(cf.z, Hv(1), cf.w, sub(d_ex_dz1, d_ez_dx1)));
          hzv = SD::rt(h_new<FMA>(cf.z, Hv(2), cf.w, sub(d_ey_dx1, d_ex_dy1)));
        }
        pl_hzh[rh] = hzv;
        pl_hyh[rh] = hyv;
      }
    }
    have_nx = active;
    if (PML && cell_ok && j + 1 < np - 1) prefetch(p + 1);  // next plane's H terms
    if (xhalo && j + 1 < np - 1) prefetch_halo(p + 1);

    ok = __syncthreads_or(ok ? 0 : 1) == 0;
    if (!ok) break;
    if (tid == 0 && issued < np) {  // stage j is consumed: refill its slot
      fence_proxy_async();
      issue(issued);
      ++issued;
    }

    // ---------------- E phase (update_e_field[_pml], src/fdtd.rs:369-509) ----
    if (tile_warp) {
      if (!warm) {
        const float4 hz_my = lds4(pl_hz + (r - 1) * TW + 4 * col);
        const float4 hx_my = lds4(pl_hx + (r - 1) * TW + 4 * col);
        float hz_w = __shfl_up_sync(0xffffffffu, hc[3], 1);
        float hy_w = __shfl_up_sync(0xffffffffu, hb[3], 1);
        if (col == 0) {
          hz_w = pl_hzh[r];
          hy_w = pl_hyh[r];
        }
        float d_hz_dy[4], d_hx_dy[4], d_hy_dz[4], d_hx_dz[4], d_hz_dx[4], d_hy_dx[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          d_hz_dy[q] = sub(hc[q], comp(hz_my, q));
          d_hx_dy[q] = sub(ha[q], comp(hx_my, q));
          d_hy_dz[q] = sub(hb[q], comp(hyp, q));
          d_hx_dz[q] = sub(ha[q], comp(hxp, q));
          d_hz_dx[q] = sub(hc[q], q == 0 ? hz_w : hc[q - 1]);
          d_hy_dx[q] = sub(hb[q], q == 0 ? hy_w : hb[q - 1]);
        }
        if (PML && cell_ok) {
          if (AXX && lp.xmode == 1) {
            corr4_x<FMA, SD::k16>(d_hz_dx, d_hy_dx, ex_, pf, lp.sx, un);
            store_psi4(g.pml[0], 2, lp.ix, ex_.p0, g.err);
            store_psi4(g.pml[0], 3, lp.ix, ex_.p1, g.err);
          } else if (AXX && lp.xmode == 2) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              corr_x_cell<FMA, SD::k16>(g, pf, 2, xg + q, y, p, d_hz_dx[q], d_hy_dx[q], true, un);
          }
          if (AXY && lp.y) {
            corr4_uniform<FMA, SD::k16>(d_hz_dy, d_hx_dy, ey_, pf.b(1, lp.sy), pf.a(1, lp.sy),
                                        pf.ik(1, lp.sy), un);
            store_psi4(g.pml[1], 2, lp.iy, ey_.p0, g.err);
            store_psi4(g.pml[1], 3, lp.iy, ey_.p1, g.err);
          }
          if (AXZ && lp.z) {
            corr4_uniform<FMA, SD::k16>(d_hy_dz, d_hx_dz, ez_, pf.b(2, lp.sz), pf.a(2, lp.sz),
                                        pf.ik(2, lp.sz), un);
            store_psi4(g.pml[2], 2, lp.iz, ez_.p0, g.err);
            store_psi4(g.pml[2], 3, lp.iz, ez_.p1, g.err);
          }
        }
        const long long ecell = (static_cast<long long>(p) * ny + y) * nx + xg;
        if (cell_ok && idx_ok(g.err, ecell + 3, N)) {
          float eo[3][4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const unsigned char id = q == 0 ? m4.x : (q == 1 ? m4.y : (q == 2 ? m4.z : m4.w));
            const float4 cf = s_coef[id];
            eo[0][q] = e_new<FMA>(cf.x, comp(ex4, q), cf.y, sub(d_hz_dy[q], d_hy_dz[q]));
            eo[1][q] = e_new<FMA>(cf.x, comp(ey4, q), cf.y, sub(d_hx_dz[q], d_hz_dx[q]));
            eo[2][q] = e_new<FMA>(cf.x, comp(ez4, q), cf.y, sub(d_hy_dx[q], d_hx_dy[q]));
          }
          ST *Ep = nxt + ecell;
          const typename SD::Word w0 = SD::enc4(eo[0]), w1 = SD::enc4(eo[1]), w2 = SD::enc4(eo[2]);
          SD::st4(Ep, w0);
          SD::st4(Ep + N, w1);
          SD::st4(Ep + 2 * N, w2);
          if constexpr (SD::k16) {
            mxE = __vmaxu2(mxE, __vmaxu2(__vmaxu2(SD::mag(w0.x), SD::mag(w0.y)),
                                         __vmaxu2(__vmaxu2(SD::mag(w1.x), SD::mag(w1.y)),
                                                  __vmaxu2(SD::mag(w2.x), SD::mag(w2.y)))));
          }
        }
      }
      hxp = make_float4(ha[0], ha[1], ha[2], ha[3]);
      hyp = make_float4(hb[0], hb[1], hb[2], hb[3]);
    }
  }

  flush_max();
  if (!ok) {
    // A staged plane never arrived within the wait limit: latch the error and
    // wait (again bounded) for this CTA's copies still in flight before its
    // shared memory is released.
    if (tid == 0) {
      atomicOr(g.err, kErrTimeout);
      for (int jj = done; jj < issued; ++jj) mbar_wait(smem_u32(&s_bar[jj % S]), (jj / S) & 1);
    }
  }
}

// One launch handles one class of work items, named by the mask of the CPML
// slabs its items meet (1 x, 2 y, 4 z): interior items (AX = 0: no CPML
// code, lean registers) and one instantiation per combination, so that each
// item runs only the psi code of its own axes.  The host lists each class's
// items (tile x, tile y, z chunk); the launches partition the grid.
// CTAs per SM at 4 tile rows: three, except for items on two or three CPML
// axes, whose psi registers (prefetched H terms, in-flight E terms) need
// more than a third of the register file (two there, without spills), and
// the 16-bit interior, which fits 96 registers without spills and gains
// from a fourth CTA (its shared memory allows four at 3 stages).
template <int AX>
constexpr int kMultiAxis = (AX & (AX - 1)) != 0;
template <int AX, typename ST>
constexpr int kCtasPerSm4 = kMultiAxis<AX> ? 2 : (sizeof(ST) == 2 && AX == 0 ? 4 : 3);
// five-warp CTAs (four tile warps + the halo warp) follow the rule above
template <int TY, int LX, int AX, typename ST>
constexpr int kCtasPerSm = Layout<TY, 3, ST, LX>::THREADS <= 160 ? kCtasPerSm4<AX, ST> : 1;

// Column tiles of the x-CPML slabs: 16 cells (4 lanes) wide, 32 rows tall,
// so that every lane of the CTA holds graded cells and the wide tiles hold
// none (their x range is [x_lo, x_hi) = [16, nx-16)).
constexpr int kColLanes = 4, kColRows = 32, kColStages = 3;

template <int TY, int S, bool FMA, int AX, typename ST, int LX = 32>
__global__ void __launch_bounds__(Layout<TY, S, ST, LX>::THREADS, kCtasPerSm<TY, LX, AX, ST>)
    k_fused(const __grid_constant__ CUtensorMap tmE, const __grid_constant__ CUtensorMap tmH,
            const __grid_constant__ CUtensorMap tmM, const FusedArgs a, const int *items) {
  using L = Layout<TY, S, ST, LX>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  int item = items[blockIdx.x];
  const int txi = item % a.tiles_x;
  item /= a.tiles_x;
  const int tyi = item % a.tiles_y;
  const int zc = item / a.tiles_y;
  // wide tiles step through [x_lo, x_hi); a column tile is the low (txi 0)
  // or the high (txi 1) x edge of the grid
  const int x0 = LX == 32 ? a.x_lo + txi * kTileX : (txi == 0 ? 0 : a.g.nx - L::TW);
  const int x_end = LX == 32 ? min(x0 + kTileX, a.x_hi) : x0 + L::TW;
  const int y0 = tyi * TY;
  const int k0 = zc * a.zchunk;
  const int k1 = min(k0 + a.zchunk, a.g.nz);

  float4 *s_coef = reinterpret_cast<float4 *>(smem);
  for (int i = threadIdx.x; i < 256; i += blockDim.x) s_coef[i] = a.g.coef[i];
  if (AX != 0) {  // CPML profiles at slab positions (every W <= kProfCap here)
    float *s_prof = reinterpret_cast<float *>(smem + L::PROF_OFF);
    for (int i = threadIdx.x; i < kProfSmem; i += blockDim.x) {
      const int cap = kProfSmem / 9;
      const int ax = i / (3 * cap), k = (i / cap) % 3, s = i % cap;
      const PmlAxis &P = a.g.pml[ax];
      s_prof[i] = (P.T > 0 && s < P.W) ? P.prof[k * P.W + s] : 0.0f;
    }
  }
  if (threadIdx.x == 0) {
    uint64_t *s_bar = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    for (int s = 0; s < S; ++s) mbar_init(smem_u32(&s_bar[s]), 1);
    mbar_fence_init();
  }
  __syncthreads();
  fused_body<TY, S, FMA, AX, ST, LX>(&tmE, &tmH, &tmM, a, smem, x0, y0, k0, k1, x_end);
}

// Batched step: one persistent launch per CPML class AX.  A CTA takes
// (grid, item) pairs of its class from that class's counter and runs the
// class's body for each, with that grid's arguments copied to shared memory
// and its TMA maps read from global memory.  The mbarrier ring is
// re-initialised per item (every copy of the previous item has completed:
// the body consumes or drains all it issued).
// LX < 32: the tiles are 4*LX cells wide (x0 = txi * 4*LX), as the x-CPML
// column tiles of the single-grid step, so that narrow grids keep their
// lanes busy.
template <int TY, int S, int AX, int LX = 32>
__global__ void __launch_bounds__(Layout<TY, S, float, LX>::THREADS, kCtasPerSm<TY, LX, AX, float>)
    k_fused_batch(const BatchScene *scenes, const int2 *items, int n_items, int *counter,
                  int parity) {
  using L = Layout<TY, S, float, LX>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  __shared__ int s_item;
  __shared__ FusedArgs s_args;
  uint64_t *s_bar = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
  bool first = true;
  for (;;) {
    __syncthreads();  // the previous item is done with shared memory
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const int2 si = items[it];
    const BatchScene *sc = scenes + si.x;
    {
      const int *src = reinterpret_cast<const int *>(&sc->args[parity]);
      int *dst = reinterpret_cast<int *>(&s_args);
      for (int i = threadIdx.x; i < static_cast<int>(sizeof(FusedArgs) / 4); i += blockDim.x)
        dst[i] = src[i];
    }
    __syncthreads();
    const FusedArgs &a = s_args;
    int item = si.y;
    const int txi = item % a.tiles_x;
    item /= a.tiles_x;
    const int tyi = item % a.tiles_y;
    const int zc = item / a.tiles_y;
    const int x0 = txi * L::TW, y0 = tyi * TY;
    const int k0 = zc * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.g.nz);
    float4 *s_coef = reinterpret_cast<float4 *>(smem);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_coef[i] = a.g.coef[i];
    float *s_prof = reinterpret_cast<float *>(smem + L::PROF_OFF);
    for (int i = threadIdx.x; i < kProfSmem; i += blockDim.x) {
      const int cap = kProfSmem / 9;
      const int ax = i / (3 * cap), k = (i / cap) % 3, s = i % cap;
      const PmlAxis &P = a.g.pml[ax];
      s_prof[i] = (P.T > 0 && s < P.W) ? P.prof[k * P.W + s] : 0.0f;
    }
    if (threadIdx.x == 0) {
      for (int s = 0; s < S; ++s) {
        if (!first) mbar_inval(smem_u32(&s_bar[s]));
        mbar_init(smem_u32(&s_bar[s]), 1);
      }
      mbar_fence_init();
    }
    first = false;
    __syncthreads();
    fused_body<TY, S, false, AX, float, LX>(&sc->maps[parity][0], &sc->maps[parity][1],
                                            &sc->maps[parity][2], a, smem, x0, y0, k0, k1,
                                            min(x0 + L::TW, a.g.nx));
  }
}

// The batched step in one launch: every item of every grid on 16-wide,
// 32-row tiles, all through the body that carries the psi code of all three
// axes (its slab flags are per lane and per plane).
using BatchNarrowL = Layout<kColRows, kColStages, float, kColLanes>;

cudaError_t batch_narrow_prepare_t() {
  return cudaFuncSetAttribute(k_fused_batch<kColRows, kColStages, 7, kColLanes>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, BatchNarrowL::BYTES);
}

cudaError_t batch_narrow_launch_t(const BatchScene *scenes, const int2 *items, int n_items,
                                  int *counter, int parity, int ctas, cudaStream_t s) {
  k_fused_batch<kColRows, kColStages, 7, kColLanes>
      <<<ctas, BatchNarrowL::THREADS, BatchNarrowL::BYTES, s>>>(scenes, items, n_items, counter,
                                                               parity);
  return cudaGetLastError();
}

int batch_narrow_ctas_per_sm_t() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, k_fused_batch<kColRows, kColStages, 7, kColLanes>, BatchNarrowL::THREADS,
          BatchNarrowL::BYTES) != cudaSuccess)
    return 0;
  return n;
}

#define WF_AX_CLASSES(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7)

template <int TY, int S>
cudaError_t batch_prepare_t() {
  const void *fns[] = {
#define X(A) (const void *)k_fused_batch<TY, S, A>,
      WF_AX_CLASSES(X)
#undef X
  };
  for (const void *f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Layout<TY, S, float>::BYTES);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <int TY, int S>
cudaError_t batch_launch_t(const BatchScene *scenes, const int2 *items, int n_items, int *counter,
                           int parity, int ctas, int ax, cudaStream_t s) {
  using L = Layout<TY, S, float>;
  switch (ax) {
#define X(A)                                                                                    \
  case A:                                                                                      \
    k_fused_batch<TY, S, A><<<ctas, L::THREADS, L::BYTES, s>>>(scenes, items, n_items, counter, \
                                                               parity);                        \
    break;
    WF_AX_CLASSES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int TY, int S>
int batch_ctas_per_sm_t(int ax) {
  using L = Layout<TY, S, float>;
  const void *f = nullptr;
  switch (ax) {
#define X(A)                                 \
  case A:                                    \
    f = (const void *)k_fused_batch<TY, S, A>; \
    break;
    WF_AX_CLASSES(X)
#undef X
    default:
      return 0;
  }
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, L::THREADS, L::BYTES) != cudaSuccess)
    return 0;
  return n;
}


template <int TY, int S, bool FMA, typename ST>
cudaError_t prepare_t() {
  using L = Layout<TY, S, ST>;
  const void *fns[] = {
#define X(A) (const void *)k_fused<TY, S, FMA, A, ST>,
      WF_AX_CLASSES(X)
#undef X
  };
  for (const void *f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// x-CPML column tiles: classes with the x bit only (1, 3, 5, 7)
#define WF_COL_CLASSES(X) X(1) X(3) X(5) X(7)

template <bool FMA, typename ST>
cudaError_t col_prepare_t() {
  using L = Layout<kColRows, kColStages, ST, kColLanes>;
  const void *fns[] = {
#define X(A) (const void *)k_fused<kColRows, kColStages, FMA, A, ST, kColLanes>,
      WF_COL_CLASSES(X)
#undef X
  };
  for (const void *f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <bool FMA, typename ST>
cudaError_t col_launch_t(const FusedMaps &m, const FusedArgs &a, const int *items, int n_items,
                         int ax, cudaStream_t s) {
  using L = Layout<kColRows, kColStages, ST, kColLanes>;
  if (n_items <= 0) return cudaSuccess;
  switch (ax) {
#define X(A)                                                                                \
  case A:                                                                                  \
    k_fused<kColRows, kColStages, FMA, A, ST, kColLanes>                                   \
        <<<n_items, L::THREADS, L::BYTES, s>>>(m.e, m.h, m.m, a, items);                    \
    break;
    WF_COL_CLASSES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int TY, int S, bool FMA, typename ST>
cudaError_t launch_t(const FusedMaps &m, const FusedArgs &a, const int *items, int n_items,
                     int ax, cudaStream_t s) {
  using L = Layout<TY, S, ST>;
  if (n_items <= 0) return cudaSuccess;
  switch (ax) {
#define X(A)                                                                                     \
  case A:                                                                                       \
    k_fused<TY, S, FMA, A, ST><<<n_items, L::THREADS, L::BYTES, s>>>(m.e, m.h, m.m, a, items); \
    break;
    WF_AX_CLASSES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace
}  // namespace wf
