// wf_split.cu -- the two-kernel step (H kernel, then E kernel), the step-tail
// kernel (sources, then probes), and layout conversion kernels.
//
// The split step is the general path: one thread per cell, any boundary on
// any axis (zero-field as OUTER_ZERO_BLOCK, src/engine.rs:83, or periodic as
// the validation studies' Y/Z wrap, examples/convergence_study.rs:121-149).
// It reads the current state and writes the next state buffer, exactly like
// the fused kernel, so either path can continue a run the other started.
#include "wf_internal.cuh"
#include "wf_launch.h"
#include "wf_store.cuh"

namespace wf {

namespace {

__device__ __forceinline__ void cell_xyz(long long i, int nx, int ny, int &x, int &y, int &z) {
  x = static_cast<int>(i % nx);
  const long long yz = i / nx;
  y = static_cast<int>(yz % ny);
  z = static_cast<int>(yz / ny);
}

// psi slot of the cell on one axis; returns false outside that axis's slab
__device__ __forceinline__ bool pml_slot(const PmlAxis &P, int axis, int x, int y, int z, int nx,
                                         int ny, int nz, long long &idx, float &b, float &a,
                                         float &ik) {
  const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
  const int c = axis == 0 ? x : (axis == 1 ? y : z);
  const int s = slab_pos(c, n, P.T, P.W);
  if (s < 0) return false;
  if (axis == 0) idx = (static_cast<long long>(z) * ny + y) * P.pitch + s;
  else if (axis == 1) idx = (static_cast<long long>(z) * P.W + s) * nx + x;
  else idx = (static_cast<long long>(s) * ny + y) * nx + x;
  b = P.prof[s];
  a = P.prof[P.W + s];
  ik = P.prof[2 * P.W + s];
  return true;
}

// value i of a component array of n cells, zero when a bounds-checked build
// finds i outside it
__device__ __forceinline__ float ld_chk(const float *p, long long i, long long n, int *err) {
  return idx_ok(err, i, n) ? p[i] : 0.0f;
}

// update_h_field[_pml] for one cell (src/fdtd.rs:194-345)
template <bool FMA>
__global__ void k_split_h(GridArgs g) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int x, y, z;
  cell_xyz(i, g.nx, g.ny, x, y, z);
  const long long N = g.N, sy = g.nx, sz = static_cast<long long>(g.nx) * g.ny;
  const float *E = g.cur;
  const long long ixp = x + 1 < g.nx ? i + 1 : (g.periodic[0] ? i - (g.nx - 1) : -1);
  const long long iyp = y + 1 < g.ny ? i + sy : (g.periodic[1] ? i - (g.ny - 1) * sy : -1);
  const long long izp = z + 1 < g.nz ? i + sz : (g.periodic[2] ? i - (g.nz - 1) * sz : -1);
  int *err = g.err;
  const float ex = E[i], ey = E[N + i], ez = E[2 * N + i];
  const float ez_py = iyp >= 0 ? ld_chk(E + 2 * N, iyp, N, err) : 0.0f;
  const float ex_py = iyp >= 0 ? ld_chk(E, iyp, N, err) : 0.0f;
  const float ey_pz = izp >= 0 ? ld_chk(E + N, izp, N, err) : 0.0f;
  const float ex_pz = izp >= 0 ? ld_chk(E, izp, N, err) : 0.0f;
  const float ez_px = ixp >= 0 ? ld_chk(E + 2 * N, ixp, N, err) : 0.0f;
  const float ey_px = ixp >= 0 ? ld_chk(E + N, ixp, N, err) : 0.0f;
  float d_ez_dy = sub(ez_py, ez), d_ex_dy = sub(ex_py, ex);
  float d_ey_dz = sub(ey_pz, ey), d_ex_dz = sub(ex_pz, ex);
  float d_ez_dx = sub(ez_px, ez), d_ey_dx = sub(ey_px, ey);
  long long idx;
  float b, a, ik;
  if (pml_slot(g.pml[0], 0, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik) &&
      idx_ok(err, idx, g.pml[0].cells)) {
    const PmlAxis &P = g.pml[0];
    float p0 = P.psi_cur[idx], p1 = P.psi_cur[P.cells + idx];
    d_ez_dx = pml_corr<FMA>(d_ez_dx, b, a, ik, p0);
    d_ey_dx = pml_corr<FMA>(d_ey_dx, b, a, ik, p1);
    P.psi_nxt[idx] = p0;
    P.psi_nxt[P.cells + idx] = p1;
  }
  if (pml_slot(g.pml[1], 1, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik) &&
      idx_ok(err, idx, g.pml[1].cells)) {
    const PmlAxis &P = g.pml[1];
    float p0 = P.psi_cur[idx], p1 = P.psi_cur[P.cells + idx];
    d_ez_dy = pml_corr<FMA>(d_ez_dy, b, a, ik, p0);
    d_ex_dy = pml_corr<FMA>(d_ex_dy, b, a, ik, p1);
    P.psi_nxt[idx] = p0;
    P.psi_nxt[P.cells + idx] = p1;
  }
  if (pml_slot(g.pml[2], 2, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik) &&
      idx_ok(err, idx, g.pml[2].cells)) {
    const PmlAxis &P = g.pml[2];
    float p0 = P.psi_cur[idx], p1 = P.psi_cur[P.cells + idx];
    d_ey_dz = pml_corr<FMA>(d_ey_dz, b, a, ik, p0);
    d_ex_dz = pml_corr<FMA>(d_ex_dz, b, a, ik, p1);
    P.psi_nxt[idx] = p0;
    P.psi_nxt[P.cells + idx] = p1;
  }
  const float curl_hx = sub(d_ez_dy, d_ey_dz);
  const float curl_hy = sub(d_ex_dz, d_ez_dx);
  const float curl_hz = sub(d_ey_dx, d_ex_dy);
  const float4 cf = g.coef[g.mat[(static_cast<long long>(z) * g.ny + y) * g.mat_pitch + x]];
  const float *H = g.cur + 3 * N;  // (i < N: all indices below are in range)
  float *Hn = g.nxt + 3 * N;
  Hn[i] = h_new<FMA>(cf.z, H[i], cf.w, curl_hx);
  Hn[N + i] = h_new<FMA>(cf.z, H[N + i], cf.w, curl_hy);
  Hn[2 * N + i] = h_new<FMA>(cf.z, H[2 * N + i], cf.w, curl_hz);
}

// update_e_field[_pml] for one cell (src/fdtd.rs:369-509); H is the new H
template <bool FMA>
__global__ void k_split_e(GridArgs g) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int x, y, z;
  cell_xyz(i, g.nx, g.ny, x, y, z);
  const long long N = g.N, sy = g.nx, sz = static_cast<long long>(g.nx) * g.ny;
  const float *H = g.nxt + 3 * N;
  const long long ixm = x > 0 ? i - 1 : (g.periodic[0] ? i + (g.nx - 1) : -1);
  const long long iym = y > 0 ? i - sy : (g.periodic[1] ? i + (g.ny - 1) * sy : -1);
  const long long izm = z > 0 ? i - sz : (g.periodic[2] ? i + (g.nz - 1) * sz : -1);
  int *err = g.err;
  const float hx = H[i], hy = H[N + i], hz = H[2 * N + i];
  const float hz_my = iym >= 0 ? ld_chk(H + 2 * N, iym, N, err) : 0.0f;
  const float hx_my = iym >= 0 ? ld_chk(H, iym, N, err) : 0.0f;
  const float hy_mz = izm >= 0 ? ld_chk(H + N, izm, N, err) : 0.0f;
  const float hx_mz = izm >= 0 ? ld_chk(H, izm, N, err) : 0.0f;
  const float hz_mx = ixm >= 0 ? ld_chk(H + 2 * N, ixm, N, err) : 0.0f;
  const float hy_mx = ixm >= 0 ? ld_chk(H + N, ixm, N, err) : 0.0f;
  float d_hz_dy = sub(hz, hz_my), d_hx_dy = sub(hx, hx_my);
  float d_hy_dz = sub(hy, hy_mz), d_hx_dz = sub(hx, hx_mz);
  float d_hz_dx = sub(hz, hz_mx), d_hy_dx = sub(hy, hy_mx);
  long long idx;
  float b, a, ik;
  if (pml_slot(g.pml[0], 0, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik) &&
      idx_ok(err, idx, g.pml[0].cells)) {
    const PmlAxis &P = g.pml[0];
    float p2 = P.psi_cur[2 * P.cells + idx], p3 = P.psi_cur[3 * P.cells + idx];
    d_hz_dx = pml_corr<FMA>(d_hz_dx, b, a, ik, p2);
    d_hy_dx = pml_corr<FMA>(d_hy_dx, b, a, ik, p3);
    P.psi_nxt[2 * P.cells + idx] = p2;
    P.psi_nxt[3 * P.cells + idx] = p3;
  }
  if (pml_slot(g.pml[1], 1, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik) &&
      idx_ok(err, idx, g.pml[1].cells)) {
    const PmlAxis &P = g.pml[1];
    float p2 = P.psi_cur[2 * P.cells + idx], p3 = P.psi_cur[3 * P.cells + idx];
    d_hz_dy = pml_corr<FMA>(d_hz_dy, b, a, ik, p2);
    d_hx_dy = pml_corr<FMA>(d_hx_dy, b, a, ik, p3);
    P.psi_nxt[2 * P.cells + idx] = p2;
    P.psi_nxt[3 * P.cells + idx] = p3;
  }
  if (pml_slot(g.pml[2], 2, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik) &&
      idx_ok(err, idx, g.pml[2].cells)) {
    const PmlAxis &P = g.pml[2];
    float p2 = P.psi_cur[2 * P.cells + idx], p3 = P.psi_cur[3 * P.cells + idx];
    d_hy_dz = pml_corr<FMA>(d_hy_dz, b, a, ik, p2);
    d_hx_dz = pml_corr<FMA>(d_hx_dz, b, a, ik, p3);
    P.psi_nxt[2 * P.cells + idx] = p2;
    P.psi_nxt[3 * P.cells + idx] = p3;
  }
  const float curl_ex = sub(d_hz_dy, d_hy_dz);
  const float curl_ey = sub(d_hx_dz, d_hz_dx);
  const float curl_ez = sub(d_hy_dx, d_hx_dy);
  const float4 cf = g.coef[g.mat[(static_cast<long long>(z) * g.ny + y) * g.mat_pitch + x]];
  const float *E = g.cur;
  float *En = g.nxt;
  En[i] = e_new<FMA>(cf.x, E[i], cf.y, curl_ex);
  En[N + i] = e_new<FMA>(cf.x, E[N + i], cf.y, curl_ey);
  En[2 * N + i] = e_new<FMA>(cf.x, E[2 * N + i], cf.y, curl_ez);
}

// One stored value of a 16-bit state in field units: decode / encode with a
// shift.
__device__ __forceinline__ float dec16(const void *f, long long i, int prec, int shift) {
  const unsigned b = static_cast<const unsigned short *>(f)[i];
  return __fmul_rn(prec == kPrecF16 ? Store<__half>::dec_lo(b) : Store<__nv_bfloat16>::dec_lo(b),
                   pow2f(shift));
}
// stores v; returns the decoded stored value
__device__ __forceinline__ float enc16(void *f, long long i, int prec, int shift, float v) {
  const float u = __fmul_rn(v, pow2f(-shift));
  const unsigned w = prec == kPrecF16 ? Store16<__half>::enc2(u, u) : Store16<__nv_bfloat16>::enc2(u, u);
  static_cast<unsigned short *>(f)[i] = static_cast<unsigned short>(w & 0xffffu);
  return dec16(f, i, prec, shift);
}

// Write shifts of the step with index `next`, from the slab maxima of the
// state it reads (then cleared): a slab's bound takes its neighbour slabs'
// maxima (one step moves information one plane), the E/H cross-coupling
// through the largest Cb/Db times 8 (four raw differences, each at most
// doubled by the CPML correction), and the soft-source amplitudes that
// step adds:  bh = 2*NH + kh*NE,  be = 2*NE + ke*bh + src  (f32, this
// order); the slab's shift (E and H alike) = store_shift_bits(max(be, bh)).
// Whole CTA; s_src >= nslab.
// count_sat (after a step, binary16): every slab and kind whose maximum is
// binary16's largest finite magnitude (where .satfinite puts overflowing
// values) adds one to *ovf.
__device__ void next_shifts(const TailArgs &t, long long next, float *s_src, bool count_sat) {
  if (count_sat && t.prec == kPrecF16) {
    for (int k = threadIdx.x; k < 2 * t.nslab; k += blockDim.x)
      if (t.slab_max[k] == __float_as_uint(__fmul_rn(65504.0f, pow2f(t.shift_f[k]))))
        atomicAdd(t.ovf, 1ull);
  }
  for (int b = threadIdx.x; b < t.nslab; b += blockDim.x) s_src[b] = 0.0f;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < t.nsrc; ++i) {
      const SrcDev q = t.src[i];
      const float v = next < q.nvals ? fabsf(q.vals[next]) : 0.0f;
      if (q.mode == 0) {
        const int b = q.z / kSlabPlanes;
        s_src[b] = __fadd_rn(s_src[b], v);
      } else {
        for (int b = 0; b < t.nslab; ++b) s_src[b] = __fadd_rn(s_src[b], v);
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < t.nslab; b += blockDim.x) {
    unsigned me = t.slab_max[2 * b], mh = t.slab_max[2 * b + 1];
    for (int d = -1; d <= 1; d += 2) {
      int n = b + d;
      if (n < 0 || n >= t.nslab) {
        if (!t.periodic_z) continue;
        n = (n + t.nslab) % t.nslab;
      }
      me = max(me, t.slab_max[2 * n]);
      mh = max(mh, t.slab_max[2 * n + 1]);
    }
    const float ne = __uint_as_float(me), nh = __uint_as_float(mh);
    const float bh = __fadd_rn(__fmul_rn(2.0f, nh), __fmul_rn(t.kh, ne));
    const float be = __fadd_rn(__fadd_rn(__fmul_rn(2.0f, ne), __fmul_rn(t.ke, bh)), s_src[b]);
    const int sh = store_shift_bits(__float_as_uint(fmaxf(be, bh)));
    t.shift_next[2 * b] = sh;
    t.shift_next[2 * b + 1] = sh;
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 2 * t.nslab; b += blockDim.x) t.slab_max[b] = 0u;
}

constexpr int kMaxSlabs = 1024;  // nz <= 8192 for 16-bit storage

// Sources in list order (src/engine.rs:769-772, Source::inject
// src/source.rs:79-95), then probes (src/probe.rs:126-138).  One CTA; the
// step index lives in device memory so captured graphs stay replayable.
// 16-bit storage: sources re-encode the cells they change (their magnitudes
// join the slab maxima), probes decode, and the CTA then picks the shifts
// the next step writes with.
__device__ void tail_body(const TailArgs &t, float *s_src);

__global__ void k_tail(TailArgs t) {
  __shared__ float s_src[kMaxSlabs];
  tail_body(t, s_src);
}

// one CTA per grid of a batch (FP32 storage: no slab scales)
__global__ void k_tail_batch(const TailArgs *ts) {
  const TailArgs t = ts[blockIdx.x];
  tail_body(t, nullptr);
}

__device__ void tail_body(const TailArgs &t, float *s_src) {
  __shared__ long long s_step;
  if (threadIdx.x == 0) s_step = *t.step;
  __syncthreads();
  const long long st = s_step;
  const long long N = static_cast<long long>(t.nx) * t.ny * t.nz;
  const bool f16 = t.prec != kPrecF32;
  for (int s = 0; s < t.nsrc; ++s) {
    const SrcDev q = t.src[s];
    const float v = st < q.nvals ? q.vals[st] : 0.0f;
    if (q.mode == 0) {
      const long long i = q.comp * N + (static_cast<long long>(q.z) * t.ny + q.y) * t.nx + q.x;
      if (threadIdx.x == 0 && idx_ok(t.err, i, 6 * N)) {
        if (f16) {
          const int b = q.z / kSlabPlanes, sh = t.shift_f[2 * b];
          const float d = enc16(t.f, i, t.prec, sh, __fadd_rn(dec16(t.f, i, t.prec, sh), v));
          t.slab_max[2 * b] = max(t.slab_max[2 * b], __float_as_uint(fabsf(d)));
        } else {
          t.f[i] = __fadd_rn(t.f[i], v);
        }
      }
    } else {
      const long long m = static_cast<long long>(t.ny) * t.nz;
      for (long long c = threadIdx.x; c < m; c += blockDim.x) {
        const long long yy = c % t.ny, zz = c / t.ny;
        const long long i = q.comp * N + (zz * t.ny + yy) * t.nx + q.x;
        if (!idx_ok(t.err, i, 6 * N)) continue;
        if (f16) {
          const int b = static_cast<int>(zz) / kSlabPlanes;
          const float d = enc16(t.f, i, t.prec, t.shift_f[2 * b], v);
          atomicMax(t.slab_max + 2 * b, __float_as_uint(fabsf(d)));
        } else {
          t.f[i] = v;
        }
      }
    }
    __syncthreads();
  }
  for (int p = threadIdx.x; p < t.nprobe; p += blockDim.x) {
    const ProbeDev q = t.probe[p];
    const long long i = q.comp * N + (static_cast<long long>(q.z) * t.ny + q.y) * t.nx + q.x;
    if (!idx_ok(t.err, i, 6 * N)) continue;
    const float raw =
        f16 ? dec16(t.f, i, t.prec, t.shift_f[2 * (q.z / kSlabPlanes) + (q.comp >= 3)]) : t.f[i];
    if (q.record && st < q.nsteps) q.trace[st] = raw;
    if (st >= q.first_step && st < q.nsteps) {
      const double v = static_cast<double>(raw);
      for (int f = 0; f < q.nfreq; ++f) {
        q.sc[f] = __dadd_rn(q.sc[f], __dmul_rn(v, q.cos_tab[st * q.nfreq + f]));
        q.ss[f] = __dadd_rn(q.ss[f], __dmul_rn(v, q.sin_tab[st * q.nfreq + f]));
      }
      q.n[0] += 1ull;
    }
  }
  __syncthreads();
  if (f16) next_shifts(t, st + 1, s_src, true);
  if (threadIdx.x == 0) *t.step = st + 1;
}

__global__ void k_next_shifts(TailArgs t, long long next) {
  __shared__ float s_src[kMaxSlabs];
  next_shifts(t, next, s_src, false);
}

// 16-bit state from FP32 values, in three passes: slab maxima of the input,
// the shift they give each slab (from the larger of its E and H maxima),
// then the encoding (whose maxima remain).
__global__ void k_slab_max_f32(const float *in, long long N, int nxy, unsigned *slab_max) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * N) return;
  const int c = static_cast<int>(i / N);
  const int b = static_cast<int>((i % N) / nxy) / kSlabPlanes;
  const unsigned v = __float_as_uint(fabsf(in[i]));
  if (v) atomicMax(slab_max + 2 * b + (c >= 3), v);
}
__global__ void k_shift_from_max(unsigned *slab_max, int *shift, int nslab) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nslab) return;
  const int sh = store_shift_bits(max(slab_max[2 * b], slab_max[2 * b + 1]));
  shift[2 * b] = sh;
  shift[2 * b + 1] = sh;
  slab_max[2 * b] = slab_max[2 * b + 1] = 0u;
}
__global__ void k_encode(const float *in, void *out, int prec, long long N, int nxy,
                         const int *shift, unsigned *slab_max) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * N) return;
  const int c = static_cast<int>(i / N);
  const int k = 2 * (static_cast<int>((i % N) / nxy) / kSlabPlanes) + (c >= 3);
  const float d = enc16(out, i, prec, shift[k], in[i]);
  const unsigned v = __float_as_uint(fabsf(d));
  if (v) atomicMax(slab_max + k, v);
}
__global__ void k_state_max(const void *in, int prec, long long N, int nxy, const int *shift,
                            unsigned *slab_max) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * N) return;
  const int c = static_cast<int>(i / N);
  const int k = 2 * (static_cast<int>((i % N) / nxy) / kSlabPlanes) + (c >= 3);
  const unsigned v = __float_as_uint(fabsf(dec16(in, i, prec, shift[k])));
  if (v) atomicMax(slab_max + k, v);
}
__global__ void k_decode(const void *in, float *out, int prec, long long N, int nxy,
                         const int *shift) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= 6 * N) return;
  const int c = static_cast<int>(i / N);
  out[i] = dec16(in, i, prec, shift[2 * (static_cast<int>((i % N) / nxy) / kSlabPlanes) + (c >= 3)]);
}

// SoA (x fastest) <-> FieldBlock order (src/layout.rs:697-755)
__global__ void k_soa_to_blocks(const float *soa, float *blk, int nx, int ny, int nz) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int x, y, z;
  cell_xyz(i, nx, ny, x, y, z);
  const long long b = (static_cast<long long>(z / 8) * (ny / 8) + y / 8) * (nx / 8) + x / 8;
  const int l = ((z % 8) * 8 + (y % 8)) * 8 + (x % 8);
  for (int c = 0; c < 6; ++c) blk[b * 3072 + c * 512 + l] = soa[c * N + i];
}

__global__ void k_blocks_to_soa(const float *blk, float *soa, int nx, int ny, int nz) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int x, y, z;
  cell_xyz(i, nx, ny, x, y, z);
  const long long b = (static_cast<long long>(z / 8) * (ny / 8) + y / 8) * (nx / 8) + x / 8;
  const int l = ((z % 8) * 8 + (y % 8)) * 8 + (x % 8);
  for (int c = 0; c < 6; ++c) soa[c * N + i] = blk[b * 3072 + c * 512 + l];
}

}  // namespace

cudaError_t launch_split(const GridArgs &g, bool fma, cudaStream_t s) {
  const int threads = 256;
  const unsigned blocks = static_cast<unsigned>((g.N + threads - 1) / threads);
  if (fma) {
    k_split_h<true><<<blocks, threads, 0, s>>>(g);
    k_split_e<true><<<blocks, threads, 0, s>>>(g);
  } else {
    k_split_h<false><<<blocks, threads, 0, s>>>(g);
    k_split_e<false><<<blocks, threads, 0, s>>>(g);
  }
  return cudaGetLastError();
}

cudaError_t launch_tail(const TailArgs &t, cudaStream_t s) {
  if (t.prec != kPrecF32 && t.nslab > kMaxSlabs) return cudaErrorInvalidValue;
  k_tail<<<1, 256, 0, s>>>(t);
  return cudaGetLastError();
}

cudaError_t launch_tail_batch(const TailArgs *t, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_tail_batch<<<n, 256, 0, s>>>(t);
  return cudaGetLastError();
}

cudaError_t launch_next_shifts(const TailArgs &t, long long next, cudaStream_t s) {
  if (t.nslab > kMaxSlabs) return cudaErrorInvalidValue;
  k_next_shifts<<<1, 256, 0, s>>>(t, next);
  return cudaGetLastError();
}

cudaError_t launch_encode_state(const float *in, void *out, int prec, int nx, int ny, int nz,
                                int *shift, unsigned *slab_max, unsigned long long *ovf,
                                cudaStream_t s) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  const unsigned blocks = static_cast<unsigned>((6 * N + 255) / 256);
  const int nslab = nz / kSlabPlanes;
  cudaError_t e = cudaMemsetAsync(slab_max, 0, sizeof(unsigned) * 2 * nslab, s);
  if (e != cudaSuccess) return e;
  k_slab_max_f32<<<blocks, 256, 0, s>>>(in, N, nx * ny, slab_max);
  k_shift_from_max<<<(nslab + 255) / 256, 256, 0, s>>>(slab_max, shift, nslab);
  (void)ovf;  // encoding a given state saturates nothing it has to report
  k_encode<<<blocks, 256, 0, s>>>(in, out, prec, N, nx * ny, shift, slab_max);
  return cudaGetLastError();
}

cudaError_t launch_state_max(const void *in, int prec, int nx, int ny, int nz, const int *shift,
                             unsigned *slab_max, cudaStream_t s) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  cudaError_t e = cudaMemsetAsync(slab_max, 0, sizeof(unsigned) * 2 * (nz / kSlabPlanes), s);
  if (e != cudaSuccess) return e;
  k_state_max<<<static_cast<unsigned>((6 * N + 255) / 256), 256, 0, s>>>(in, prec, N, nx * ny,
                                                                         shift, slab_max);
  return cudaGetLastError();
}

cudaError_t launch_decode_state(const void *in, float *out, int prec, int nx, int ny, int nz,
                                const int *shift, cudaStream_t s) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  k_decode<<<static_cast<unsigned>((6 * N + 255) / 256), 256, 0, s>>>(in, out, prec, N, nx * ny,
                                                                       shift);
  return cudaGetLastError();
}

cudaError_t launch_soa_to_blocks(const float *soa, float *blk, int nx, int ny, int nz,
                                 cudaStream_t s) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  k_soa_to_blocks<<<static_cast<unsigned>((N + 255) / 256), 256, 0, s>>>(soa, blk, nx, ny, nz);
  return cudaGetLastError();
}

cudaError_t launch_blocks_to_soa(const float *blk, float *soa, int nx, int ny, int nz,
                                 cudaStream_t s) {
  const long long N = static_cast<long long>(nx) * ny * nz;
  k_blocks_to_soa<<<static_cast<unsigned>((N + 255) / 256), 256, 0, s>>>(blk, soa, nx, ny, nz);
  return cudaGetLastError();
}

}  // namespace wf
