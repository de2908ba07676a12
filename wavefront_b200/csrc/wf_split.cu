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
  const float ex = E[i], ey = E[N + i], ez = E[2 * N + i];
  const float ez_py = iyp >= 0 ? E[2 * N + iyp] : 0.0f, ex_py = iyp >= 0 ? E[iyp] : 0.0f;
  const float ey_pz = izp >= 0 ? E[N + izp] : 0.0f, ex_pz = izp >= 0 ? E[izp] : 0.0f;
  const float ez_px = ixp >= 0 ? E[2 * N + ixp] : 0.0f, ey_px = ixp >= 0 ? E[N + ixp] : 0.0f;
  float d_ez_dy = sub(ez_py, ez), d_ex_dy = sub(ex_py, ex);
  float d_ey_dz = sub(ey_pz, ey), d_ex_dz = sub(ex_pz, ex);
  float d_ez_dx = sub(ez_px, ez), d_ey_dx = sub(ey_px, ey);
  long long idx;
  float b, a, ik;
  if (pml_slot(g.pml[0], 0, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik)) {
    const PmlAxis &P = g.pml[0];
    float p0 = P.psi_cur[idx], p1 = P.psi_cur[P.cells + idx];
    d_ez_dx = pml_corr<FMA>(d_ez_dx, b, a, ik, p0);
    d_ey_dx = pml_corr<FMA>(d_ey_dx, b, a, ik, p1);
    P.psi_nxt[idx] = p0;
    P.psi_nxt[P.cells + idx] = p1;
  }
  if (pml_slot(g.pml[1], 1, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik)) {
    const PmlAxis &P = g.pml[1];
    float p0 = P.psi_cur[idx], p1 = P.psi_cur[P.cells + idx];
    d_ez_dy = pml_corr<FMA>(d_ez_dy, b, a, ik, p0);
    d_ex_dy = pml_corr<FMA>(d_ex_dy, b, a, ik, p1);
    P.psi_nxt[idx] = p0;
    P.psi_nxt[P.cells + idx] = p1;
  }
  if (pml_slot(g.pml[2], 2, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik)) {
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
  const float *H = g.cur + 3 * N;
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
  const float hx = H[i], hy = H[N + i], hz = H[2 * N + i];
  const float hz_my = iym >= 0 ? H[2 * N + iym] : 0.0f, hx_my = iym >= 0 ? H[iym] : 0.0f;
  const float hy_mz = izm >= 0 ? H[N + izm] : 0.0f, hx_mz = izm >= 0 ? H[izm] : 0.0f;
  const float hz_mx = ixm >= 0 ? H[2 * N + ixm] : 0.0f, hy_mx = ixm >= 0 ? H[N + ixm] : 0.0f;
  float d_hz_dy = sub(hz, hz_my), d_hx_dy = sub(hx, hx_my);
  float d_hy_dz = sub(hy, hy_mz), d_hx_dz = sub(hx, hx_mz);
  float d_hz_dx = sub(hz, hz_mx), d_hy_dx = sub(hy, hy_mx);
  long long idx;
  float b, a, ik;
  if (pml_slot(g.pml[0], 0, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik)) {
    const PmlAxis &P = g.pml[0];
    float p2 = P.psi_cur[2 * P.cells + idx], p3 = P.psi_cur[3 * P.cells + idx];
    d_hz_dx = pml_corr<FMA>(d_hz_dx, b, a, ik, p2);
    d_hy_dx = pml_corr<FMA>(d_hy_dx, b, a, ik, p3);
    P.psi_nxt[2 * P.cells + idx] = p2;
    P.psi_nxt[3 * P.cells + idx] = p3;
  }
  if (pml_slot(g.pml[1], 1, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik)) {
    const PmlAxis &P = g.pml[1];
    float p2 = P.psi_cur[2 * P.cells + idx], p3 = P.psi_cur[3 * P.cells + idx];
    d_hz_dy = pml_corr<FMA>(d_hz_dy, b, a, ik, p2);
    d_hx_dy = pml_corr<FMA>(d_hx_dy, b, a, ik, p3);
    P.psi_nxt[2 * P.cells + idx] = p2;
    P.psi_nxt[3 * P.cells + idx] = p3;
  }
  if (pml_slot(g.pml[2], 2, x, y, z, g.nx, g.ny, g.nz, idx, b, a, ik)) {
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

// Sources in list order (src/engine.rs:769-772, Source::inject
// src/source.rs:79-95), then probes (src/probe.rs:126-138).  One CTA; the
// step index lives in device memory so captured graphs stay replayable.
__global__ void k_tail(TailArgs t) {
  __shared__ long long s_step;
  if (threadIdx.x == 0) s_step = *t.step;
  __syncthreads();
  const long long st = s_step;
  const long long N = static_cast<long long>(t.nx) * t.ny * t.nz;
  for (int s = 0; s < t.nsrc; ++s) {
    const SrcDev q = t.src[s];
    const float v = st < q.nvals ? q.vals[st] : 0.0f;
    float *F = t.f + q.comp * N;
    if (q.mode == 0) {
      if (threadIdx.x == 0) {
        const long long i = (static_cast<long long>(q.z) * t.ny + q.y) * t.nx + q.x;
        F[i] = __fadd_rn(F[i], v);
      }
    } else {
      const long long m = static_cast<long long>(t.ny) * t.nz;
      for (long long c = threadIdx.x; c < m; c += blockDim.x) {
        const long long yy = c % t.ny, zz = c / t.ny;
        F[(zz * t.ny + yy) * t.nx + q.x] = v;
      }
    }
    __syncthreads();
  }
  for (int p = threadIdx.x; p < t.nprobe; p += blockDim.x) {
    const ProbeDev q = t.probe[p];
    const float raw = t.f[q.comp * N + (static_cast<long long>(q.z) * t.ny + q.y) * t.nx + q.x];
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
  if (threadIdx.x == 0) *t.step = st + 1;
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
  k_tail<<<1, 256, 0, s>>>(t);
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
