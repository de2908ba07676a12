// wf_engine.cu -- the C ABI of include/wavefront_gpu.h: device state, upload,
// step orchestration (fused or split step + tail kernel, replayed through
// captured CUDA graphs), and read-back in the reference's formats.
//
// Engine semantics follow src/engine.rs:747-782: each step is H everywhere,
// E everywhere, then every source in order, then every probe.
#include <cudaTypedefs.h>

#include <errno.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/wavefront_gpu.h"
#include "wf_closure.h"
#include "wf_launch.h"
#include "wf_pool.h"
#include "wf_scene.h"

using wf::FusedArgs;
using wf::FusedConfig;
using wf::GridArgs;
using wf::ProbeDev;
using wf::SrcDev;
using wf::TailArgs;

namespace {

thread_local std::string g_last_error;

struct SrcRec {
  SrcDev d;       // device view (vals points into device memory)
  float *vals;    // device
};

struct ProbeRec {
  ProbeDev d;
  double *cos_tab, *sin_tab, *sc, *ss, *base;
  unsigned long long *n;
  float *trace;
};

struct AxisState {
  int T = 0, W = 0, pitch = 0;
  float *prof = nullptr;       // [3][W]
  float *psi[2] = {nullptr, nullptr};
  long long cells = 0;
};

}  // namespace

struct wf_handle {
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int nx = 0, ny = 0, nz = 0;
  long long N = 0;
  int periodic[3] = {0, 0, 0};
  int arith = WF_ARITH_EXACT;
  int kernel_pref = WF_KERNEL_AUTO;
  int precision = WF_PREC_F32;
  float *fld[2] = {nullptr, nullptr};  // 16-bit elements unless precision is F32
  // 16-bit storage: per state buffer the [nslab][2] shifts it is stored with,
  // the slab maxima of the state being written, binary16 saturations, and
  // whether the next step's shifts must be derived from the current state
  int *shift[2] = {nullptr, nullptr};
  unsigned *slab_max = nullptr;
  unsigned long long *d_ovf = nullptr;
  int nslab = 0;
  bool shifts_dirty = true;
  float kh = 0.0f, ke = 0.0f;  // 8 * max |Db|, 8 * max |Cb|
  int cur = 0;
  uint8_t *mat = nullptr;
  int mat_pitch = 0;
  float4 *coef = nullptr;
  AxisState ax[3];
  std::vector<SrcRec> srcs;
  std::vector<ProbeRec> probes;
  SrcDev *d_src = nullptr;
  ProbeDev *d_probe = nullptr;
  bool tables_dirty = false;  // d_src / d_probe lag srcs / probes (flush_tables)
  long long *d_step = nullptr;
  int *d_err = nullptr;
  long long steps_done = 0;
  // learned boundary closure (applied after every step kernel when on)
  bool closure = false;
  void *cl_w[3] = {nullptr, nullptr, nullptr};  // bf16 weights, 6 faces per layer
  float *cl_buf = nullptr;                      // X, A1, A2, Y band tensors
  float cl_ge = 1.0f, cl_gh = 1.0f;
  bool cl_guard = false;  // wf_set_closure_guard
  int *cl_face = nullptr;                       // device {0, 1, ..., 5}
  // tensor-core closure with packed operands: three packed band tensors, the
  // FP32 output, RMS partials and scales; packed weights; TMA maps
  unsigned char *cl_fast = nullptr;
  void *cl_wp = nullptr;
  CUtensorMap cl_tm[3];
  bool cl_fast_ok = false;
  long long version = 0;               // bumped when device tables are reallocated
  long long kernel_launches = 0;       // step + tail kernels issued so far
  long long graph_kernels[2] = {0, 0};  // kernels in one replay of graph[parity]
  FusedConfig cfg{4, 12, 3};
  int test_extra_tx = 0;      // wf_set_test_stall
  bool cfg_user_set = false;  // otherwise chosen from the grid at first use
  wf::FusedMaps maps[2];      // per state buffer (the one read by the step)
  int *d_items = nullptr;     // work items grouped by kernel class
  int class_off[wf::kFusedClassCount] = {}, class_n[wf::kFusedClassCount] = {};
  // the class launches of one step run concurrently: forked from the main
  // stream onto these streams and joined back before the step tail
  cudaStream_t side[wf::kFusedClassCount - 1] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[wf::kFusedClassCount - 1] = {};
  // x-CPML column tiles (wf_set_column_tiles): whether they are in use, the
  // caller's preference, their maps, work lists and streams
  bool cols = false;
  bool col_pref = true;
  wf::FusedMaps col_maps[2];
  int col_off[wf::kColClassCount] = {}, col_n[wf::kColClassCount] = {};
  cudaStream_t side_col[wf::kColClassCount] = {};
  cudaEvent_t join_col[wf::kColClassCount] = {};
  bool maps_ok = false;
  // asynchronous FieldBlock download (wf_download_blocks_async): a staging
  // buffer the state is reordered into on the handle's stream, copied to the
  // host on a stream of its own while stepping goes on
  float *d_stage = nullptr;
  cudaStream_t copy = nullptr;
  cudaEvent_t staged = nullptr, copied = nullptr;
  bool copy_pending = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_steps = 0;
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;   // pairs: start, end per timed launch
  size_t ev_used = 0;
  std::string err;
};

namespace {

wf_status fail(wf_handle *h, wf_status s, const std::string &msg) {
  if (h) h->err = msg;
  g_last_error = msg;
  return s;
}

wf_status cuda_fail(wf_handle *h, cudaError_t e, const char *what) {
  const wf_status s = (e == cudaErrorMemoryAllocation) ? WF_ERR_OOM : WF_ERR_CUDA;
  return fail(h, s, std::string(what) + ": " + cudaGetErrorString(e));
}

// Host-to-device copies and device memsets of the set-up calls, ordered on
// the handle's stream and complete on return.  Plain cudaMemcpy from pageable
// memory may return before its DMA lands and cudaMemset is asynchronous, both
// on the legacy default stream, which kernels on the handles' non-blocking
// streams are not ordered after.
cudaError_t h2d_sync(void *dst, const void *src, size_t bytes, cudaStream_t s,
                     cudaMemcpyKind kind = cudaMemcpyHostToDevice) {
  if (bytes == 0) return cudaSuccess;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

cudaError_t memset_sync(void *dst, int value, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(dst, value, bytes, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

#define WF_CUDA(h, call)                                \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void drop_graphs(wf_handle *h) {
  for (auto &g : h->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

// The streams and events a fused step forks its class launches onto.  A
// handle takes a set before its first fused step (the grids of a batch, which
// step through the batch's own streams, never take one) and gives it back
// when it is destroyed: each device keeps up to kIdleStreamSets idle sets, so
// that the next handle skips 12 stream and 12 event creations (about 0.5 ms).
// Sets are returned idle (their streams synchronized), and every event of a
// set is recorded again before each wait on it.
struct StreamSet {
  cudaStream_t side[wf::kFusedClassCount - 1] = {};
  cudaEvent_t join_ev[wf::kFusedClassCount - 1] = {};
  cudaStream_t side_col[wf::kColClassCount] = {};
  cudaEvent_t join_col[wf::kColClassCount] = {};
  cudaEvent_t fork_ev = nullptr;
};
constexpr size_t kIdleStreamSets = 8;
std::mutex g_sets_mu;
std::map<int, std::vector<StreamSet>> g_idle_sets;  // per device (mutex held)

void destroy_set(StreamSet &ss) {
  for (auto s : ss.side)
    if (s) cudaStreamDestroy(s);
  for (auto s : ss.side_col)
    if (s) cudaStreamDestroy(s);
  for (auto ev : ss.join_ev)
    if (ev) cudaEventDestroy(ev);
  for (auto ev : ss.join_col)
    if (ev) cudaEventDestroy(ev);
  if (ss.fork_ev) cudaEventDestroy(ss.fork_ev);
  ss = StreamSet{};
}

// Gives h a stream set (an idle one of its device, else a new one); the
// device is current.  Outside any stream capture.
wf_status acquire_streams(wf_handle *h) {
  if (h->fork_ev) return WF_OK;
  StreamSet ss;
  bool cached = false;
  {
    std::lock_guard<std::mutex> lk(g_sets_mu);
    auto &v = g_idle_sets[h->dev];
    if (!v.empty()) {
      ss = v.back();
      v.pop_back();
      cached = true;
    }
  }
  if (!cached) {
    cudaError_t e = cudaEventCreateWithFlags(&ss.fork_ev, cudaEventDisableTiming);
    for (int k = 0; k < wf::kFusedClassCount - 1 && e == cudaSuccess; ++k) {
      e = cudaStreamCreateWithFlags(&ss.side[k], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.join_ev[k], cudaEventDisableTiming);
    }
    for (int k = 0; k < wf::kColClassCount && e == cudaSuccess; ++k) {
      e = cudaStreamCreateWithFlags(&ss.side_col[k], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.join_col[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
      destroy_set(ss);
      return cuda_fail(h, e, "side stream setup");
    }
  }
  std::copy(std::begin(ss.side), std::end(ss.side), h->side);
  std::copy(std::begin(ss.join_ev), std::end(ss.join_ev), h->join_ev);
  std::copy(std::begin(ss.side_col), std::end(ss.side_col), h->side_col);
  std::copy(std::begin(ss.join_col), std::end(ss.join_col), h->join_col);
  h->fork_ev = ss.fork_ev;
  return WF_OK;
}

// Returns h's stream set (if it took one) to its device's idle list, or
// destroys it when the list is full; the device is current.
void release_streams(wf_handle *h) {
  if (!h->fork_ev) return;
  StreamSet ss;
  std::copy(std::begin(h->side), std::end(h->side), ss.side);
  std::copy(std::begin(h->join_ev), std::end(h->join_ev), ss.join_ev);
  std::copy(std::begin(h->side_col), std::end(h->side_col), ss.side_col);
  std::copy(std::begin(h->join_col), std::end(h->join_col), ss.join_col);
  ss.fork_ev = h->fork_ev;
  h->fork_ev = nullptr;
  bool idle = true;
  for (auto st : ss.side) idle = idle && cudaStreamSynchronize(st) == cudaSuccess;
  for (auto st : ss.side_col) idle = idle && cudaStreamSynchronize(st) == cudaSuccess;
  if (idle) {
    std::lock_guard<std::mutex> lk(g_sets_mu);
    auto &v = g_idle_sets[h->dev];
    if (v.size() < kIdleStreamSets) {
      v.push_back(ss);
      return;
    }
  }
  destroy_set(ss);
}

}  // namespace

namespace wf {

void release_idle_stream_sets(int dev) {
  std::map<int, std::vector<StreamSet>> sets;
  {
    std::lock_guard<std::mutex> lk(g_sets_mu);
    for (auto &kv : g_idle_sets) {
      if (dev >= 0 && kv.first != dev) continue;
      sets[kv.first].swap(kv.second);
    }
  }
  for (auto &kv : sets) {
    DeviceGuard guard(kv.first);
    for (auto &ss : kv.second) destroy_set(ss);
  }
}

}  // namespace wf

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

bool fused_allowed(const wf_handle *h) {
  return !h->periodic[0] && !h->periodic[1] && !h->periodic[2];
}

bool store16(const wf_handle *h) { return h->precision != WF_PREC_F32; }
size_t elem_bytes(const wf_handle *h) { return store16(h) ? 2 : 4; }

bool use_fused(const wf_handle *h) {
  if (h->kernel_pref == WF_KERNEL_SPLIT) return false;
  // the fused kernel stages CPML profiles of up to 64 slab positions per axis
  // in shared memory; thicker layers take the split kernels
  for (const AxisState &A : h->ax)
    if (A.T > 0 && A.W > 64) return false;
  return fused_allowed(h) && encode_fn() != nullptr;
}

bool has_pml(const wf_handle *h) { return h->ax[0].T > 0 || h->ax[1].T > 0 || h->ax[2].T > 0; }
FusedArgs fused_args(const wf_handle *h);
FusedArgs col_args(const wf_handle *h);

// The x-CPML slabs run as 16-wide column tiles when each is at most 16
// cells deep and the grid leaves a wide region of at least 16 cells.
bool cols_apply(const wf_handle *h) {
  const int T = h->ax[0].T;
  return h->col_pref && T > 0 && T <= wf::kColWidth && h->nx >= 3 * wf::kColWidth;
}

// Column-class index (0..3) of CPML class 1, 3, 5, 7.
constexpr int col_slot(int ax) { return ax >> 1; }

// One tiled TMA descriptor (no swizzle, no interleave, zero out-of-bounds fill).
bool encode(CUtensorMap *m, CUtensorMapDataType t, int rank, void *base, const cuuint64_t *dims,
            const cuuint64_t *strides, const cuuint32_t *box) {
  static const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
  return encode_fn()(m, t, rank, base, dims, strides, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tiling used unless the caller set one: 4 rows, 3 stages, and the z chunk
// measured best on B200 (two_spheres 512^3, random spheres 1024^3).  A
// longer chunk recomputes the warm-up plane less often; the issue-bound
// 16-bit kernel gains most from that.
FusedConfig default_cfg(const wf_handle *h) {
  const bool big = h->nz >= 1024;
  if (store16(h)) return FusedConfig{4, big ? 48 : 32, 3};
  // FP32: 24-plane chunks (fewer warm-up planes) while they still give at
  // least four waves of work items at three CTAs per SM, else 12
  const long long tiles = static_cast<long long>((h->nx + wf::kTileX - 1) / wf::kTileX) *
                          ((h->ny + 3) / 4);
  const long long items24 = tiles * ((h->nz + 23) / 24);
  return FusedConfig{4, items24 >= 4LL * 148 * 3 ? 24 : 12, 3};
}

// TMA descriptors per state buffer: fields as a 4D tensor {nx, ny, nz, 6},
// ids as {nx, ny, nz} with a 16-byte-multiple row pitch, and each CPML
// axis's psi slab as a 4D tensor {.., .., .., 4 terms}.
wf_status build_maps(wf_handle *h, bool allow_cols = true) {
  h->maps_ok = false;
  if (!encode_fn()) return fail(h, WF_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  if (!h->cfg_user_set) h->cfg = default_cfg(h);
  h->cols = allow_cols && cols_apply(h);
  unsigned eb[4], hb[4], mb[3];
  wf::fused_boxes(h->cfg.ty, h->precision, eb, hb, mb);
  const cuuint64_t es = elem_bytes(h);
  const cuuint64_t fdim[4] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)h->nz, 6};
  const cuuint64_t fstr[3] = {(cuuint64_t)h->nx * es, (cuuint64_t)h->nx * h->ny * es,
                              (cuuint64_t)h->N * es};
  const CUtensorMapDataType ft = h->precision == WF_PREC_F16    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                 : h->precision == WF_PREC_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t mdim[3] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)h->nz};
  const cuuint64_t mstr[2] = {(cuuint64_t)h->mat_pitch, (cuuint64_t)h->mat_pitch * h->ny};
  const cuuint32_t ebox[4] = {eb[0], eb[1], eb[2], eb[3]};
  const cuuint32_t hbox[4] = {hb[0], hb[1], hb[2], hb[3]};
  const cuuint32_t mbox[3] = {mb[0], mb[1], mb[2]};
  for (int b = 0; b < 2; ++b) {
    wf::FusedMaps &m = h->maps[b];
    std::memset(&m, 0, sizeof(m));
    if (!encode(&m.e, ft, 4, h->fld[b], fdim, fstr, ebox) ||
        !encode(&m.h, ft, 4, h->fld[b], fdim, fstr, hbox) ||
        !encode(&m.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->mat, mdim, mstr, mbox))
      return fail(h, WF_ERR_CUDA, "cuTensorMapEncodeTiled(fields/ids) failed");
  }
  WF_CUDA(h, wf::fused_prepare(h->cfg, h->precision));
  if (h->cols) {
    wf::fused_col_boxes(h->precision, eb, hb, mb);
    const cuuint32_t cebox[4] = {eb[0], eb[1], eb[2], eb[3]};
    const cuuint32_t chbox[4] = {hb[0], hb[1], hb[2], hb[3]};
    const cuuint32_t cmbox[3] = {mb[0], mb[1], mb[2]};
    for (int b = 0; b < 2; ++b) {
      wf::FusedMaps &m = h->col_maps[b];
      std::memset(&m, 0, sizeof(m));
      if (!encode(&m.e, ft, 4, h->fld[b], fdim, fstr, cebox) ||
          !encode(&m.h, ft, 4, h->fld[b], fdim, fstr, chbox) ||
          !encode(&m.m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->mat, mdim, mstr, cmbox))
        return fail(h, WF_ERR_CUDA, "cuTensorMapEncodeTiled(column tiles) failed");
    }
    WF_CUDA(h, wf::fused_col_prepare(h->precision));
  }
  // Work lists, one per kernel class (interior first): each class runs the
  // kernel instantiation that carries only the CPML code it needs.
  const FusedArgs a = fused_args(h);
  const int n_items = a.tiles_x * a.tiles_y * ((h->nz + a.zchunk - 1) / a.zchunk);
  std::vector<int> lists[wf::kFusedClassCount];
  for (int i = 0; i < n_items; ++i) lists[wf::fused_item_class(a, h->cfg.ty, i)].push_back(i);
  std::vector<int> all;
  for (int k = 0; k < wf::kFusedClassCount; ++k) {
    h->class_off[k] = static_cast<int>(all.size());
    h->class_n[k] = static_cast<int>(lists[k].size());
    all.insert(all.end(), lists[k].begin(), lists[k].end());
  }
  // column items (low and high x edge, 32-row tiles), one list per class
  std::vector<int> clists[wf::kColClassCount];
  if (h->cols) {
    const FusedArgs c = col_args(h);
    const int nc = c.tiles_x * c.tiles_y * ((h->nz + c.zchunk - 1) / c.zchunk);
    for (int i = 0; i < nc; ++i) clists[col_slot(wf::fused_col_item_class(c, i))].push_back(i);
  }
  for (int k = 0; k < wf::kColClassCount; ++k) {
    h->col_off[k] = static_cast<int>(all.size());
    h->col_n[k] = static_cast<int>(clists[k].size());
    all.insert(all.end(), clists[k].begin(), clists[k].end());
  }
  wf::dev_free(h->d_items);
  h->d_items = nullptr;
  WF_CUDA(h, wf::dev_alloc(&h->d_items, sizeof(int) * std::max<size_t>(all.size(), 1)));
  WF_CUDA(h, h2d_sync(h->d_items, all.data(), sizeof(int) * all.size(), h->stream));
  h->maps_ok = true;
  return WF_OK;
}

GridArgs grid_args(const wf_handle *h) {
  GridArgs g{};
  g.nx = h->nx;
  g.ny = h->ny;
  g.nz = h->nz;
  g.N = h->N;
  for (int i = 0; i < 3; ++i) g.periodic[i] = h->periodic[i];
  g.cur = h->fld[h->cur];
  g.nxt = h->fld[h->cur ^ 1];
  g.mat = h->mat;
  g.mat_pitch = h->mat_pitch;
  g.coef = h->coef;
  for (int a = 0; a < 3; ++a) {
    const AxisState &A = h->ax[a];
    g.pml[a].T = A.T;
    g.pml[a].W = A.W;
    g.pml[a].pitch = A.pitch;
    g.pml[a].prof = A.prof;
    g.pml[a].psi_cur = A.psi[h->cur];
    g.pml[a].psi_nxt = A.psi[h->cur ^ 1];
    g.pml[a].cells = A.cells;
  }
  g.err = h->d_err;
  g.prec = h->precision;
  g.shift_rd = h->shift[h->cur];
  g.shift_wr = h->shift[h->cur ^ 1];
  g.slab_max = h->slab_max;
  g.ovf = h->d_ovf;
  g.nslab = h->nslab;
  return g;
}

// Raw view of state buffer b for the closure kernels.
wf::BandGrid band_grid(const wf_handle *h, int b) {
  wf::BandGrid g{};
  g.nx = h->nx;
  g.ny = h->ny;
  g.nz = h->nz;
  g.N = h->N;
  g.fields = h->fld[b];
  for (int a = 0; a < 3; ++a) {
    const AxisState &A = h->ax[a];
    g.psi[a] = wf::BandPsi{A.T, A.W, A.pitch, A.psi[b], A.cells};
  }
  return g;
}

constexpr int kClHidden = 16;  // closure hidden channels

// The closure on the state just written (buffer cur ^ 1): bands of the six
// faces (times the gains), each face divided by its band's E RMS -> conv
// 10->16 GELU -> conv 16->16 GELU -> conv 16->6 -> times that RMS -> fields
// += (over the gains).
// The same closure with the tensor-core kernels on packed operands
// (wf_closure_fast.cu): gather, RMS (fixed-order partial sums), pack divided
// by the RMS, three convolutions, each writing the next one's packed input,
// the last one FP32 times the RMS, scatter.
cudaError_t closure_enqueue_fast(wf_handle *h) {
  const int n = h->nx, D = wf::kBandDepth;
  const long long P = static_cast<long long>(D) * n * n;
  const size_t packed = 6 * 6 * static_cast<size_t>(P) * 16, wbytes = 6 * 27 * 512;
  unsigned char *pk[3] = {h->cl_fast, h->cl_fast + packed, h->cl_fast + 2 * packed};
  float *Y = reinterpret_cast<float *>(h->cl_fast + 3 * packed);
  float *scale = Y + 6 * 6 * P, *part = scale + 64;
  const unsigned char *wp = static_cast<const unsigned char *>(h->cl_wp);
  const wf::BandGrid g = band_grid(h, h->cur ^ 1);
  int e = wf::closure_fast_gather(g, pk[0], part, n, n, h->cl_ge, h->cl_gh, h->stream);
  if (!e) e = wf::closure_fast_rms(part, n, n, P, scale, h->stream);
  if (!e)
    e = wf::closure_fast_conv(h->cl_tm[0], wp, pk[1], nullptr, scale, scale, kClHidden, D, n, n, false,
                              h->stream);
  if (!e)
    e = wf::closure_fast_conv(h->cl_tm[1], wp + wbytes, pk[2], nullptr, scale, nullptr, kClHidden, D, n,
                              n, false, h->stream);
  if (!e)
    e = wf::closure_fast_conv(h->cl_tm[2], wp + 2 * wbytes, nullptr, Y, scale, nullptr, 6, D, n, n, true,
                              h->stream);
  if (!e) e = wf::band_scatter_add(g, Y, n, n, h->cl_ge, h->cl_gh, h->stream);
  return static_cast<cudaError_t>(e);
}

// Kernels closure_enqueue issues: the scatter takes one launch per axis whose
// two bands are disjoint (two otherwise); the packed path gathers, folds the
// RMS and runs the three layers; the FP32 path gathers, reduces the RMS,
// scales in and out around its three layers, and guards when asked.
int closure_launches(const wf_handle *h) {
  int scatter = 0;
  for (int n : {h->nx, h->ny, h->nz}) scatter += n >= 2 * wf::kBandDepth ? 1 : 2;
  if (h->cl_fast_ok && !h->cl_guard && wf::nn_tensor_cores()) return 3 + 1 + 3 + scatter;
  return 3 + 1 + 1 + 3 + 1 + (h->cl_guard ? 2 : 0) + scatter;
}

cudaError_t closure_enqueue(wf_handle *h) {
  if (h->cl_fast_ok && !h->cl_guard && wf::nn_tensor_cores()) return closure_enqueue_fast(h);
  const int n = h->nx, D = wf::kBandDepth;
  const long long P = static_cast<long long>(D) * n * n;
  float *X = h->cl_buf, *A1 = X + 6 * wf::kBandIn * P, *A2 = A1 + 6 * kClHidden * P,
        *Y = A2 + 6 * kClHidden * P;
  const wf::BandGrid g = band_grid(h, h->cur ^ 1);
  float *scale = Y + 6 * 6 * P, *lam = scale + 8;
  int e = wf::band_gather(g, X, n, n, h->cl_ge, h->cl_gh, h->stream);
  if (!e) e = wf::face_rms(X, wf::kBandIn, P, scale, h->stream);
  if (!e) e = wf::face_scale(X, wf::kBandIn, P, scale, 1, h->stream);
  // sample s of the band tensors is face s and uses face s's weights
  if (!e) e = wf::nn_conv_fwd(X, h->cl_w[0], h->cl_face, nullptr, A1, 6, wf::kBandIn, kClHidden, D, n, n, 1, h->stream);
  if (!e) e = wf::nn_conv_fwd(A1, h->cl_w[1], h->cl_face, nullptr, A2, 6, kClHidden, kClHidden, D, n, n, 1, h->stream);
  if (!e) e = wf::nn_conv_fwd(A2, h->cl_w[2], h->cl_face, nullptr, Y, 6, kClHidden, 6, D, n, n, 0, h->stream);
  if (!e) e = wf::face_scale(Y, 6, P, scale, 0, h->stream);
  if (!e && h->cl_guard) e = wf::face_guard(X, wf::kBandIn, Y, P, scale, lam, h->stream);
  if (!e && h->cl_guard) e = wf::face_scale(Y, 6, P, lam, 0, h->stream);
  if (!e) e = wf::band_scatter_add(g, Y, n, n, h->cl_ge, h->cl_gh, h->stream);
  return static_cast<cudaError_t>(e);
}

// Tail arguments of a step that reads buffer h->cur (16-bit fields included).
wf_status flush_tables(wf_handle *h);  // below, with the descriptor upload

TailArgs tail_args(const wf_handle *h) {
  TailArgs t{};
  t.f = h->fld[h->cur ^ 1];
  t.nx = h->nx;
  t.ny = h->ny;
  t.nz = h->nz;
  t.src = h->d_src;
  t.nsrc = static_cast<int>(h->srcs.size());
  t.probe = h->d_probe;
  t.nprobe = static_cast<int>(h->probes.size());
  t.step = h->d_step;
  t.prec = h->precision;
  t.shift_f = h->shift[h->cur ^ 1];
  t.slab_max = h->slab_max;
  t.shift_next = h->shift[h->cur];  // the next step reads cur ^ 1 and writes cur
  t.nslab = h->nslab;
  t.periodic_z = h->periodic[2];
  t.kh = h->kh;
  t.ke = h->ke;
  t.ovf = h->d_ovf;
  t.err = h->d_err;
  return t;
}

FusedArgs fused_args(const wf_handle *h) {
  FusedArgs a{};
  a.g = grid_args(h);
  a.x_lo = h->cols ? wf::kColWidth : 0;
  a.x_hi = h->cols ? h->nx - wf::kColWidth : h->nx;
  a.tiles_x = (a.x_hi - a.x_lo + wf::kTileX - 1) / wf::kTileX;
  a.tiles_y = (h->ny + h->cfg.ty - 1) / h->cfg.ty;
  a.zchunk = h->cfg.zchunk;
  a.has_pml = has_pml(h) ? 1 : 0;
  a.prof_in_smem = (h->ax[0].W <= 64 && h->ax[1].W <= 64 && h->ax[2].W <= 64) ? 1 : 0;
  a.test_extra_tx = h->test_extra_tx;
  return a;
}

// Arguments of a column-tile launch: two tiles across (the low and the high
// x edge), 32-row tiles, the wide tiles' z chunk.
FusedArgs col_args(const wf_handle *h) {
  FusedArgs a = fused_args(h);
  a.tiles_x = 2;
  a.tiles_y = (h->ny + wf::kColTileRows - 1) / wf::kColTileRows;
  return a;
}

// One full step on h->stream: step kernel(s) cur -> nxt, then the tail.
cudaEvent_t timing_event(wf_handle *h) {
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
    h->ev_pool.push_back(ev);
  }
  return h->ev_pool[h->ev_used++];
}

wf_status enqueue_one(wf_handle *h) {
  GridArgs g = grid_args(h);
  const bool fma = h->arith == WF_ARITH_FMA;
  cudaError_t e;
  if (h->timing) {
    cudaEvent_t ev = timing_event(h);
    if (!ev) return fail(h, WF_ERR_CUDA, "cudaEventCreate");
    WF_CUDA(h, cudaEventRecord(ev, h->stream));
  }
  if (use_fused(h)) {
    if (!h->maps_ok) {
      wf_status s = build_maps(h);
      if (s != WF_OK) return s;
    }
    if (!h->fork_ev) {
      wf_status s = acquire_streams(h);
      if (s != WF_OK) return s;
    }
    const FusedArgs a = fused_args(h);
    // class 0 (interior) on the main stream, the CPML classes on side
    // streams forked from it; they touch disjoint cells of the next state.
    // Launched costliest items first (three axes ... one axis, interior
    // last), so that the cheap interior items fill the end of the step.
    static constexpr int kOrder[wf::kFusedClassCount] = {7, 5, 3, 6, 1, 4, 2, 0};
    WF_CUDA(h, cudaEventRecord(h->fork_ev, h->stream));
    e = cudaSuccess;
    // the x-CPML column tiles first (every lane runs the psi recursion)
    const FusedArgs ca = col_args(h);
    for (int ax = 7; ax >= 1 && h->cols && e == cudaSuccess; ax -= 2) {
      const int k = col_slot(ax);
      if (h->col_n[k] == 0) continue;
      cudaStream_t s = h->side_col[k];
      WF_CUDA(h, cudaStreamWaitEvent(s, h->fork_ev, 0));
      e = wf::launch_fused_col(h->col_maps[h->cur], ca, h->d_items + h->col_off[k], h->col_n[k],
                               ax, fma, s);
      if (e == cudaSuccess) h->kernel_launches += 1;
      if (e == cudaSuccess) WF_CUDA(h, cudaEventRecord(h->join_col[k], s));
    }
    for (int i = 0; i < wf::kFusedClassCount && e == cudaSuccess; ++i) {
      const int k = kOrder[i];
      if (h->class_n[k] == 0) continue;
      cudaStream_t s = k == 0 ? h->stream : h->side[k - 1];
      if (k > 0) WF_CUDA(h, cudaStreamWaitEvent(s, h->fork_ev, 0));
      e = wf::launch_fused(h->cfg, h->maps[h->cur], a, h->d_items + h->class_off[k],
                           h->class_n[k], k, fma, s);
      if (e == cudaSuccess) h->kernel_launches += 1;
      if (e == cudaSuccess && k > 0) WF_CUDA(h, cudaEventRecord(h->join_ev[k - 1], s));
    }
    // the main stream waits for every side class only after all are launched
    for (int k = 1; k < wf::kFusedClassCount && e == cudaSuccess; ++k)
      if (h->class_n[k] > 0) WF_CUDA(h, cudaStreamWaitEvent(h->stream, h->join_ev[k - 1], 0));
    for (int k = 0; k < wf::kColClassCount && h->cols && e == cudaSuccess; ++k)
      if (h->col_n[k] > 0) WF_CUDA(h, cudaStreamWaitEvent(h->stream, h->join_col[k], 0));
  } else {
    e = wf::launch_split(g, fma, h->stream);
    if (e == cudaSuccess) h->kernel_launches += 2;  // H pass, E pass
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "step kernel launch");
  if (h->closure) {
    e = closure_enqueue(h);
    if (e != cudaSuccess) return cuda_fail(h, e, "closure launch");
    h->kernel_launches += closure_launches(h);
  }
  if (h->timing) {
    cudaEvent_t ev = timing_event(h);
    if (!ev) return fail(h, WF_ERR_CUDA, "cudaEventCreate");
    WF_CUDA(h, cudaEventRecord(ev, h->stream));
  }
  // 16-bit storage always runs the tail: it picks the next step's shifts
  if (!h->srcs.empty() || !h->probes.empty() || store16(h)) {
    if (h->tables_dirty) {
      wf_status s = flush_tables(h);
      if (s != WF_OK) return s;
    }
    e = wf::launch_tail(tail_args(h), h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "tail kernel launch");
    h->kernel_launches += 1;
  }
  h->cur ^= 1;
  return WF_OK;
}

// 16-bit storage: the slab maxima of the current state (from its data) and
// the shifts the next step writes with.
wf_status refresh_shifts(wf_handle *h) {
  if (h->tables_dirty) {  // the tail arguments below hold the descriptor arrays
    wf_status s = flush_tables(h);
    if (s != WF_OK) return s;
  }
  WF_CUDA(h, wf::launch_state_max(h->fld[h->cur], h->precision, h->nx, h->ny, h->nz,
                                  h->shift[h->cur], h->slab_max, h->stream));
  TailArgs t = tail_args(h);
  t.shift_next = h->shift[h->cur ^ 1];  // the next step reads cur, writes cur ^ 1
  WF_CUDA(h, wf::launch_next_shifts(t, h->steps_done, h->stream));
  h->shifts_dirty = false;
  return WF_OK;
}

wf_status upload_src_probe_tables(wf_handle *h) {
  drop_graphs(h);
  ++h->version;
  h->shifts_dirty = true;  // source amplitudes enter the 16-bit shifts
  h->tables_dirty = false;
  if (h->d_src) wf::dev_free(h->d_src);
  if (h->d_probe) wf::dev_free(h->d_probe);
  h->d_src = nullptr;
  h->d_probe = nullptr;
  if (!h->srcs.empty()) {
    std::vector<SrcDev> v;
    for (auto &s : h->srcs) v.push_back(s.d);
    WF_CUDA(h, wf::dev_alloc(&h->d_src, sizeof(SrcDev) * v.size()));
    WF_CUDA(h, h2d_sync(h->d_src, v.data(), sizeof(SrcDev) * v.size(), h->stream));
  }
  if (!h->probes.empty()) {
    std::vector<ProbeDev> v;
    for (auto &p : h->probes) v.push_back(p.d);
    WF_CUDA(h, wf::dev_alloc(&h->d_probe, sizeof(ProbeDev) * v.size()));
    WF_CUDA(h, h2d_sync(h->d_probe, v.data(), sizeof(ProbeDev) * v.size(), h->stream));
  }
  return WF_OK;
}

// A source or probe was added: its descriptor array is uploaded once, before
// the next step or batch build (flush_tables), rather than after every add;
// captured graphs and batch tables that hold the old arrays are dropped now.
void tables_changed(wf_handle *h) {
  drop_graphs(h);
  ++h->version;
  h->shifts_dirty = true;
  h->tables_dirty = true;
}

// Uploads the descriptor arrays if an add left them stale.  Outside any
// stream capture (it allocates and synchronizes).
// The 16-bit shift flag is left as it is: the add itself set it, and a
// checkpoint restore since then may have cleared it (the restored shifts are
// the ones the next step must use).
wf_status flush_tables(wf_handle *h) {
  if (!h->tables_dirty) return WF_OK;
  const bool shifts_dirty = h->shifts_dirty;
  const wf_status s = upload_src_probe_tables(h);
  h->shifts_dirty = shifts_dirty;
  return s;
}

bool tables_cover(const wf_handle *h, long long upto, std::string *why) {
  for (size_t i = 0; i < h->srcs.size(); ++i)
    if (h->srcs[i].d.nvals < upto) {
      *why = "source " + std::to_string(i) + " has values for " + std::to_string(h->srcs[i].d.nvals) +
             " steps, run needs " + std::to_string(upto);
      return false;
    }
  for (size_t i = 0; i < h->probes.size(); ++i)
    if (h->probes[i].d.nsteps < upto) {
      *why = "probe " + std::to_string(i) + " has tables for " + std::to_string(h->probes[i].d.nsteps) +
             " steps, run needs " + std::to_string(upto);
      return false;
    }
  return true;
}

wf_status device_error_status(wf_handle *h, int flag) {
  if (flag & wf::kErrTimeout)
    return fail(h, WF_ERR_TIMEOUT, "a device-side bounded wait timed out (TMA stage never arrived)");
  if (flag) return fail(h, WF_ERR_DEVICE_FLAG, "device error flag set: " + std::to_string(flag));
  return WF_OK;
}

wf_status check_device_error(wf_handle *h) {
  int flag = 0;
  WF_CUDA(h, cudaMemcpy(&flag, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  return device_error_status(h, flag);
}

}  // namespace

// A batch of independent grids stepped by one persistent kernel per step
// (config: many small scenes of uneven size).  Each grid is an ordinary
// handle on the batch's stream; the batch keeps device tables describing
// all of them for the batched step kernel and the batched tail.
struct wf_batch {
  int dev = 0;
  cudaStream_t stream = nullptr;
  std::vector<wf_handle *> h;
  FusedConfig cfg{4, 16, 3};
  wf::BatchScene *d_scenes = nullptr;
  int2 *d_items = nullptr;  // grouped by CPML class
  int n_items = 0;
  int class_off[wf::kFusedClassCount] = {}, class_n[wf::kFusedClassCount] = {};
  int class_ctas[wf::kFusedClassCount] = {};
  int step_kernels = 0;    // non-empty classes: step-kernel launches per step
  bool narrow = false;     // one launch over 16 x 32 tiles (tile_rows == kColTileRows)
  int narrow_ctas = 0;
  int *d_counter = nullptr;  // one work counter per class
  // the class launches of a step run concurrently: forked from `stream` onto
  // these and joined back before the tail
  cudaStream_t side[wf::kFusedClassCount - 1] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[wf::kFusedClassCount - 1] = {};
  TailArgs *d_tails[2] = {nullptr, nullptr};  // per parity of the state read
  bool have_tail = false;
  std::vector<long long> versions;  // handle versions the tables were built from
  bool built = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long launches = 0;
};

namespace {

void batch_drop(wf_batch *b) {
  for (auto &g : b->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  wf::dev_free(b->d_scenes);
  wf::dev_free(b->d_items);
  wf::dev_free(b->d_tails[0]);
  wf::dev_free(b->d_tails[1]);
  b->d_scenes = nullptr;
  b->d_items = nullptr;
  b->d_tails[0] = b->d_tails[1] = nullptr;
  b->built = false;
}

// A grid's TMA maps and fused arguments for the narrow batched step:
// 16-wide, 32-row tiles over the whole grid (the boxes of the column tiles).
wf_status narrow_batch_maps(wf_handle *h, int zchunk, wf::BatchScene *sc) {
  if (!encode_fn()) return fail(h, WF_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  unsigned eb[4], hb[4], mb[3];
  wf::fused_col_boxes(wf::kPrecF32, eb, hb, mb);
  const cuuint64_t es = sizeof(float);
  const cuuint64_t fdim[4] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)h->nz, 6};
  const cuuint64_t fstr[3] = {(cuuint64_t)h->nx * es, (cuuint64_t)h->nx * h->ny * es,
                              (cuuint64_t)h->N * es};
  const cuuint64_t mdim[3] = {(cuuint64_t)h->nx, (cuuint64_t)h->ny, (cuuint64_t)h->nz};
  const cuuint64_t mstr[2] = {(cuuint64_t)h->mat_pitch, (cuuint64_t)h->mat_pitch * h->ny};
  const cuuint32_t ebox[4] = {eb[0], eb[1], eb[2], eb[3]};
  const cuuint32_t hbox[4] = {hb[0], hb[1], hb[2], hb[3]};
  const cuuint32_t mbox[3] = {mb[0], mb[1], mb[2]};
  const int cur = h->cur;
  const FusedConfig saved = h->cfg;
  h->cfg = FusedConfig{wf::kColTileRows, zchunk, 3};
  h->cols = false;
  for (int p = 0; p < 2; ++p) {
    CUtensorMap *m = sc->maps[p];
    std::memset(m, 0, sizeof(CUtensorMap) * 3);
    if (!encode(&m[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->fld[p], fdim, fstr, ebox) ||
        !encode(&m[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->fld[p], fdim, fstr, hbox) ||
        !encode(&m[2], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->mat, mdim, mstr, mbox)) {
      h->cfg = saved;
      return fail(h, WF_ERR_CUDA, "cuTensorMapEncodeTiled(narrow batch) failed");
    }
    h->cur = p;
    FusedArgs a = fused_args(h);
    a.tiles_x = (h->nx + wf::kColWidth - 1) / wf::kColWidth;
    a.tiles_y = (h->ny + wf::kColTileRows - 1) / wf::kColTileRows;
    sc->args[p] = a;
  }
  h->cur = cur;
  h->cfg = saved;
  h->maps_ok = false;  // a single-grid step rebuilds its own maps and lists
  return WF_OK;
}

// CPML class of narrow batched item k (the axes whose slabs its cells, its
// -x/-y halo or its warm-up plane meet): orders the items, costliest first.
int narrow_item_class(const FusedArgs &a, int k) {
  const int txi = k % a.tiles_x, tyi = (k / a.tiles_x) % a.tiles_y, zc = k / (a.tiles_x * a.tiles_y);
  const int x0 = txi * wf::kColWidth, y0 = tyi * wf::kColTileRows;
  const int xh = std::min(x0 + wf::kColWidth, a.g.nx) - 1;
  const int yh = std::min(y0 + wf::kColTileRows, a.g.ny) - 1;
  const int k0 = zc * a.zchunk, k1 = std::min(k0 + a.zchunk, a.g.nz);
  const wf::PmlAxis &X = a.g.pml[0], &Y = a.g.pml[1], &Z = a.g.pml[2];
  int mask = 0;
  if (X.T > 0 && (x0 - 1 < X.T || xh >= a.g.nx - X.T)) mask |= 1;
  if (Y.T > 0 && (y0 - 1 < Y.T || yh >= a.g.ny - Y.T)) mask |= 2;
  if (Z.T > 0 && (k0 - 1 < Z.T || k1 - 1 >= a.g.nz - Z.T)) mask |= 4;
  return mask;
}

// (Re)builds the batch's device tables when any grid's tables changed.
wf_status batch_build(wf_batch *b) {
  bool fresh = b->built && b->versions.size() == b->h.size();
  for (size_t i = 0; fresh && i < b->h.size(); ++i) fresh = b->versions[i] == b->h[i]->version;
  if (fresh) return WF_OK;
  batch_drop(b);
  const size_t n = b->h.size();
  std::vector<wf::BatchScene> scenes(n);
  std::vector<int2> lists[wf::kFusedClassCount];
  std::vector<TailArgs> tails[2];
  b->have_tail = false;
  b->narrow = wf::fused_batch_narrow(b->cfg);
  for (size_t i = 0; i < n; ++i) {
    wf_handle *h = b->h[i];
    for (const AxisState &A : h->ax)
      if (A.T > 0 && A.W > 64)
        return fail(nullptr, WF_ERR_UNSUPPORTED, "batched grids need CPML slabs of at most 64 cells");
    wf_status st;
    if (b->narrow) {
      st = narrow_batch_maps(h, b->cfg.zchunk, &scenes[i]);
    } else {
      h->cfg = b->cfg;
      h->cfg_user_set = true;
      st = build_maps(h, false);  // the batched kernel tiles the whole x range
    }
    if (st == WF_OK) st = flush_tables(h);
    if (st != WF_OK) return st;
    const int cur = h->cur;
    for (int p = 0; p < 2; ++p) {
      h->cur = p;
      if (!b->narrow) {
        scenes[i].args[p] = fused_args(h);
        scenes[i].maps[p][0] = h->maps[p].e;
        scenes[i].maps[p][1] = h->maps[p].h;
        scenes[i].maps[p][2] = h->maps[p].m;
      }
      tails[p].push_back(tail_args(h));
    }
    h->cur = cur;
    if (!h->srcs.empty() || !h->probes.empty()) b->have_tail = true;
    const FusedArgs &a = scenes[i].args[0];
    const int nit = a.tiles_x * a.tiles_y * ((h->nz + a.zchunk - 1) / a.zchunk);
    for (int k = 0; k < nit; ++k)
      lists[b->narrow ? narrow_item_class(a, k) : wf::fused_item_class(a, b->cfg.ty, k)].push_back(
          make_int2(static_cast<int>(i), k));
  }
  std::vector<int2> items;
  b->step_kernels = 0;
  if (b->narrow) {
    // one list, grid by grid (largest grids first), and within a grid its
    // costliest items first (three CPML axes ... interior), each class in
    // tile order: the tiles of a grid run close together in time, so the
    // halo rows and columns they share are still in L2
    static constexpr int kOrder[wf::kFusedClassCount] = {7, 5, 3, 6, 1, 4, 2, 0};
    std::vector<std::vector<int2>> per_grid(n);
    for (int k : kOrder)
      for (const int2 &it : lists[k]) per_grid[it.x].push_back(it);
    std::vector<int> gorder(n);
    for (size_t i = 0; i < n; ++i) gorder[i] = static_cast<int>(i);
    std::stable_sort(gorder.begin(), gorder.end(),
                     [b](int p, int q) { return b->h[p]->N > b->h[q]->N; });
    for (int i : gorder) items.insert(items.end(), per_grid[i].begin(), per_grid[i].end());
    b->step_kernels = 1;
  }
  for (int k = 0; k < wf::kFusedClassCount && !b->narrow; ++k) {
    b->class_off[k] = static_cast<int>(items.size());
    b->class_n[k] = static_cast<int>(lists[k].size());
    if (b->class_n[k]) ++b->step_kernels;
    items.insert(items.end(), lists[k].begin(), lists[k].end());
  }
  WF_CUDA(nullptr, wf::dev_alloc(&b->d_scenes, sizeof(wf::BatchScene) * n));
  WF_CUDA(nullptr, h2d_sync(b->d_scenes, scenes.data(), sizeof(wf::BatchScene) * n, b->stream));
  WF_CUDA(nullptr, wf::dev_alloc(&b->d_items, sizeof(int2) * std::max<size_t>(items.size(), 1)));
  WF_CUDA(nullptr, h2d_sync(b->d_items, items.data(), sizeof(int2) * items.size(), b->stream));
  for (int p = 0; p < 2; ++p) {
    WF_CUDA(nullptr, wf::dev_alloc(&b->d_tails[p], sizeof(TailArgs) * n));
    WF_CUDA(nullptr, h2d_sync(b->d_tails[p], tails[p].data(), sizeof(TailArgs) * n, b->stream));
  }
  b->n_items = static_cast<int>(items.size());
  int sms = 0;
  WF_CUDA(nullptr, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev));
  if (b->narrow) {
    WF_CUDA(nullptr, wf::fused_batch_narrow_prepare());
    const int per_sm = std::max(1, wf::fused_batch_narrow_ctas_per_sm());
    b->narrow_ctas = std::max(1, std::min(sms * per_sm, b->n_items));
  } else {
    WF_CUDA(nullptr, wf::fused_batch_prepare(b->cfg));
  }
  for (int k = 0; k < wf::kFusedClassCount && !b->narrow; ++k) {
    const int per_sm = std::max(1, wf::fused_batch_ctas_per_sm(b->cfg, k));
    b->class_ctas[k] = std::max(1, std::min(sms * per_sm, b->class_n[k]));
  }
  b->versions.clear();
  for (wf_handle *h : b->h) b->versions.push_back(h->version);
  b->built = true;
  return WF_OK;
}

// The batched step kernels alone (read parity `cur`): one persistent launch
// per non-empty class, class 0 on the batch's stream and the others on side
// streams forked from it and joined back; the classes write disjoint cells.
wf_status batch_kernel(wf_batch *b, int cur) {
  WF_CUDA(nullptr, cudaMemsetAsync(b->d_counter, 0, sizeof(int) * wf::kFusedClassCount, b->stream));
  if (b->narrow) {
    WF_CUDA(nullptr, wf::launch_fused_batch_narrow(b->d_scenes, b->d_items, b->n_items, b->d_counter,
                                                   cur, b->narrow_ctas, b->stream));
    return WF_OK;
  }
  WF_CUDA(nullptr, cudaEventRecord(b->fork_ev, b->stream));
  // costliest items first, interior last (as in the single-grid step)
  static constexpr int kOrder[wf::kFusedClassCount] = {7, 5, 3, 6, 1, 4, 2, 0};
  for (int i = 0; i < wf::kFusedClassCount; ++i) {
    const int k = kOrder[i];
    if (!b->class_n[k]) continue;
    cudaStream_t s = k == 0 ? b->stream : b->side[k - 1];
    if (k > 0) WF_CUDA(nullptr, cudaStreamWaitEvent(s, b->fork_ev, 0));
    WF_CUDA(nullptr, wf::launch_fused_batch(b->cfg, b->d_scenes, b->d_items + b->class_off[k],
                                            b->class_n[k], b->d_counter + k, cur,
                                            b->class_ctas[k], k, s));
    if (k > 0) WF_CUDA(nullptr, cudaEventRecord(b->join_ev[k - 1], s));
  }
  for (int k = 1; k < wf::kFusedClassCount; ++k)
    if (b->class_n[k]) WF_CUDA(nullptr, cudaStreamWaitEvent(b->stream, b->join_ev[k - 1], 0));
  return WF_OK;
}

// One batched step: the step kernel, then the tail of every grid.
wf_status batch_enqueue(wf_batch *b, int cur) {
  wf_status st = batch_kernel(b, cur);
  if (st != WF_OK) return st;
  if (b->have_tail)
    WF_CUDA(nullptr, wf::launch_tail_batch(b->d_tails[cur], static_cast<int>(b->h.size()), b->stream));
  return WF_OK;
}

}  // namespace

extern "C" {

const char *wf_status_string(wf_status s) {
  switch (s) {
    case WF_OK: return "ok";
    case WF_ERR_ARG: return "invalid argument";
    case WF_ERR_CUDA: return "CUDA error";
    case WF_ERR_OOM: return "out of device memory";
    case WF_ERR_TIMEOUT: return "device wait timed out";
    case WF_ERR_DEVICE_FLAG: return "device error flag";
    case WF_ERR_STATE: return "invalid state";
    case WF_ERR_UNSUPPORTED: return "unsupported";
    case WF_ERR_IO: return "file I/O error";
  }
  return "unknown";
}

const char *wf_last_error(const wf_handle *h) {
  return h ? h->err.c_str() : g_last_error.c_str();
}

wf_status wf_create(const wf_grid_desc *d, wf_handle **out) {
  if (!d || !out) return fail(nullptr, WF_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || d->nx % 8 || d->ny % 8 || d->nz % 8)
    return fail(nullptr, WF_ERR_ARG,
                "grid dimensions must be positive multiples of BLOCK_DIM (8)");
  if (d->arith != WF_ARITH_EXACT && d->arith != WF_ARITH_FMA)
    return fail(nullptr, WF_ERR_ARG, "unknown arith mode");
  if (d->precision != WF_PREC_F32 && d->precision != WF_PREC_F16 && d->precision != WF_PREC_BF16)
    return fail(nullptr, WF_ERR_ARG, "unknown precision");
  if (d->precision != WF_PREC_F32) {
    // 16-bit storage: the fused kernel with the exact arithmetic, zero-field
    // boundaries, and at most 1024 scale slabs along z
    if (d->arith != WF_ARITH_EXACT)
      return fail(nullptr, WF_ERR_UNSUPPORTED, "16-bit storage uses the exact arithmetic");
    if (d->kernel == WF_KERNEL_SPLIT || d->boundary[0] || d->boundary[1] || d->boundary[2])
      return fail(nullptr, WF_ERR_UNSUPPORTED,
                  "16-bit storage runs the fused kernel (zero-field boundaries)");
    if (d->nz / 8 > 1024) return fail(nullptr, WF_ERR_UNSUPPORTED, "16-bit storage: nz <= 8192");
  }
  for (int i = 0; i < 3; ++i)
    if (d->boundary[i] != WF_BOUNDARY_ZERO && d->boundary[i] != WF_BOUNDARY_PERIODIC)
      return fail(nullptr, WF_ERR_ARG, "unknown boundary kind");
  if (d->kernel == WF_KERNEL_FUSED &&
      (d->boundary[0] || d->boundary[1] || d->boundary[2]))
    return fail(nullptr, WF_ERR_UNSUPPORTED, "the fused kernel supports zero-field boundaries only");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, WF_ERR_CUDA, "no CUDA device");
  if (d->device < 0 || d->device >= ndev) return fail(nullptr, WF_ERR_ARG, "bad device ordinal");
  DeviceGuard guard(d->device);
  // one attribute, not cudaGetDeviceProperties: that fills the whole property
  // struct, which takes milliseconds, inside every handle's creation
  int cc_major = 0;
  if (cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, d->device) != cudaSuccess ||
      cc_major < 10)
    return fail(nullptr, WF_ERR_UNSUPPORTED, "this library is built for sm_100a (B200)");

  wf_handle *h = new wf_handle();
  h->dev = d->device;
  h->nx = d->nx;
  h->ny = d->ny;
  h->nz = d->nz;
  h->N = static_cast<long long>(d->nx) * d->ny * d->nz;
  for (int i = 0; i < 3; ++i) h->periodic[i] = d->boundary[i] == WF_BOUNDARY_PERIODIC;
  h->arith = d->arith;
  h->kernel_pref = d->kernel;
  h->precision = d->precision;
  h->mat_pitch = (d->nx + 15) / 16 * 16;
  auto cleanup_fail = [&](wf_status s) {
    wf_destroy(h);
    return s;
  };
  cudaError_t e;
  if (d->stream) {
    h->stream = static_cast<cudaStream_t>(d->stream);
  } else {
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cleanup_fail(cuda_fail(nullptr, e, "cudaStreamCreate"));
    h->own_stream = true;
  }
  // (the side streams of the fused step are taken at its first use, acquire_streams)
  // Only the state the first step reads starts at zero: every step writes
  // every cell of the other buffer before anything reads it (the work classes
  // of the fused step, or the split H and E passes, cover the whole grid).
  for (int b = 0; b < 2; ++b) {
    e = wf::dev_alloc(&h->fld[b], elem_bytes(h) * 6 * h->N);
    if (e != cudaSuccess) return cleanup_fail(cuda_fail(nullptr, e, "cudaMalloc(fields)"));
    if (b != h->cur) continue;
    e = cudaMemsetAsync(h->fld[b], 0, elem_bytes(h) * 6 * h->N, h->stream);
    if (e != cudaSuccess) return cleanup_fail(cuda_fail(nullptr, e, "cudaMemset(fields)"));
  }
  if (store16(h)) {
    h->nslab = h->nz / 8;
    const size_t sb = sizeof(int) * 2 * h->nslab;
    if ((e = wf::dev_alloc(&h->shift[0], sb)) != cudaSuccess ||
        (e = wf::dev_alloc(&h->shift[1], sb)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->shift[0], 0, sb, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->shift[1], 0, sb, h->stream)) != cudaSuccess ||
        (e = wf::dev_alloc(&h->slab_max, sb)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->slab_max, 0, sb, h->stream)) != cudaSuccess ||
        (e = wf::dev_alloc(&h->d_ovf, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_ovf, 0, sizeof(unsigned long long), h->stream)) != cudaSuccess)
      return cleanup_fail(cuda_fail(nullptr, e, "cudaMalloc(storage scales)"));
  }
  const size_t mbytes = static_cast<size_t>(h->mat_pitch) * d->ny * d->nz;
  if ((e = wf::dev_alloc(&h->mat, mbytes)) != cudaSuccess ||
      (e = cudaMemsetAsync(h->mat, 0, mbytes, h->stream)) != cudaSuccess ||
      (e = wf::dev_alloc(&h->coef, sizeof(float4) * 256)) != cudaSuccess ||
      (e = cudaMemsetAsync(h->coef, 0, sizeof(float4) * 256, h->stream)) != cudaSuccess ||
      (e = wf::dev_alloc(&h->d_step, sizeof(long long))) != cudaSuccess ||
      (e = cudaMemsetAsync(h->d_step, 0, sizeof(long long), h->stream)) != cudaSuccess ||
      (e = wf::dev_alloc(&h->d_err, sizeof(int))) != cudaSuccess ||
      (e = cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream)) != cudaSuccess)
    return cleanup_fail(cuda_fail(nullptr, e, "cudaMalloc(state)"));
  if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
    return cleanup_fail(cuda_fail(nullptr, e, "cudaStreamSynchronize"));
  *out = h;
  return WF_OK;
}

wf_status wf_destroy(wf_handle *h) {
  if (!h) return WF_OK;
  DeviceGuard guard(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  for (auto ev : h->ev_pool) cudaEventDestroy(ev);
  release_streams(h);
  if (h->copy) {
    cudaStreamSynchronize(h->copy);
    cudaStreamDestroy(h->copy);
  }
  if (h->staged) cudaEventDestroy(h->staged);
  if (h->copied) cudaEventDestroy(h->copied);
  wf::dev_free(h->d_stage);
  for (auto &f : h->fld) wf::dev_free(f);
  for (auto &s : h->shift) wf::dev_free(s);
  for (auto &w : h->cl_w) wf::dev_free(w);
  wf::dev_free(h->cl_buf);
  wf::dev_free(h->cl_fast);
  wf::dev_free(h->cl_wp);
  wf::dev_free(h->cl_face);
  wf::dev_free(h->slab_max);
  wf::dev_free(h->d_ovf);
  wf::dev_free(h->mat);
  wf::dev_free(h->coef);
  wf::dev_free(h->d_step);
  wf::dev_free(h->d_err);
  wf::dev_free(h->d_src);
  wf::dev_free(h->d_probe);
  wf::dev_free(h->d_items);
  for (auto &a : h->ax) {
    wf::dev_free(a.prof);
    wf::dev_free(a.psi[0]);
    wf::dev_free(a.psi[1]);
  }
  for (auto &s : h->srcs) wf::dev_free(s.vals);
  for (auto &p : h->probes) {
    wf::dev_free(p.base);
    wf::dev_free(p.n);
    wf::dev_free(p.trace);
  }
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return WF_OK;
}

namespace {

// The coefficient table as the kernels read it (stream-ordered upload).
wf_status upload_coef(wf_handle *h, const int32_t (*table)[4]) {
  // FixedQ16_16::to_f32 (src/layout.rs:123-125): q as f32 * (1/65536)
  float4 coef[256];
  float cbmax = 0.0f, dbmax = 0.0f;
  for (int m = 0; m < 256; ++m) {
    coef[m] = make_float4(wf_q16_to_f32(table[m][0]), wf_q16_to_f32(table[m][1]),
                          wf_q16_to_f32(table[m][2]), wf_q16_to_f32(table[m][3]));
    cbmax = std::max(cbmax, std::fabs(coef[m].y));
    dbmax = std::max(dbmax, std::fabs(coef[m].w));
  }
  h->kh = 8.0f * dbmax;  // 16-bit storage: E/H coupling of the shift bounds
  h->ke = 8.0f * cbmax;
  h->shifts_dirty = true;
  WF_CUDA(h, cudaMemcpyAsync(h->coef, coef, sizeof(coef), cudaMemcpyHostToDevice, h->stream));
  return WF_OK;
}

}  // namespace

wf_status wf_set_materials(wf_handle *h, const uint8_t *ids, const int32_t (*table)[4]) {
  if (!h || !ids || !table) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  wf_status st = upload_coef(h, table);
  if (st != WF_OK) return st;
  WF_CUDA(h, cudaMemcpy2DAsync(h->mat, h->mat_pitch, ids, h->nx, h->nx,
                               static_cast<size_t>(h->ny) * h->nz, cudaMemcpyHostToDevice,
                               h->stream));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  return WF_OK;
}

wf_status wf_set_scene(wf_handle *h, const char *text, float dt, float dx,
                       int32_t (*table)[4], int *n_materials) {
  if (!h) return fail(h, WF_ERR_ARG, "null argument");
  return wf_set_scene_window(h, text, dt, dx, h->nz, 0, table, n_materials);
}

wf_status wf_set_scene_window(wf_handle *h, const char *text, float dt, float dx, int nz_global,
                              int z_offset, int32_t (*table)[4], int *n_materials) {
  if (!h || !text || !table) return fail(h, WF_ERR_ARG, "null argument");
  if (nz_global < h->nz || z_offset < 0 || z_offset > nz_global - h->nz)
    return fail(h, WF_ERR_ARG, "the window [z_offset, z_offset + nz) must lie in [0, nz_global)");
  std::vector<wf::RasterOp> ops;
  std::string msg;
  if (!wf::scene_parse(text, h->nx, h->ny, nz_global, dt, dx, &ops, table, n_materials, &msg))
    return fail(h, WF_ERR_ARG, msg);
  DeviceGuard guard(h->dev);
  wf_status st = upload_coef(h, table);
  if (st != WF_OK) return st;
  WF_CUDA(h, static_cast<cudaError_t>(wf::launch_voxelize(ops, h->mat, h->nx, h->ny, h->nz,
                                                          h->mat_pitch, 0, h->stream, z_offset)));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  return WF_OK;
}

namespace {

// The state of planes [z0, z0 + np) as segments of the packed slab layout:
// Ex Ey Ez Hx Hy Hz [np][ny][nx], then the x psi slots [4][np][ny][pitch],
// then the y psi slots [4][np][W][nx] (each present when that axis has CPML).
wf::SlabSegments slab_segments(const wf_handle *h, int z0, int np) {
  wf::SlabSegments sg{};
  long long off = 0;
  auto add = [&](float *dev, long long n) {
    sg.seg[sg.n++] = wf::SlabSegment{dev, off, n};
    off += n;
  };
  const long long plane = static_cast<long long>(h->nx) * h->ny;
  for (int c = 0; c < 6; ++c) add(h->fld[h->cur] + c * h->N + z0 * plane, np * plane);
  const AxisState &X = h->ax[0], &Y = h->ax[1];
  if (X.T > 0) {
    const long long row = static_cast<long long>(h->ny) * X.pitch;
    for (int k = 0; k < 4; ++k) add(X.psi[h->cur] + k * X.cells + z0 * row, np * row);
  }
  if (Y.T > 0) {
    const long long row = static_cast<long long>(Y.W) * h->nx;
    for (int k = 0; k < 4; ++k) add(Y.psi[h->cur] + k * Y.cells + z0 * row, np * row);
  }
  return sg;
}

wf_status slab_copy(wf_handle *h, int z0, int np, float *buf, int64_t capacity, bool unpack) {
  if (!h || !buf) return fail(h, WF_ERR_ARG, "null argument");
  if (store16(h)) return fail(h, WF_ERR_UNSUPPORTED, "slab copies need FP32 storage");
  if (np < 1 || z0 < 0 || z0 > h->nz - np) return fail(h, WF_ERR_ARG, "planes outside the grid");
  if (reinterpret_cast<uintptr_t>(buf) & 15) return fail(h, WF_ERR_ARG, "buffer not 16-byte aligned");
  const wf::SlabSegments sg = slab_segments(h, z0, np);
  const long long need = sg.seg[sg.n - 1].off + sg.seg[sg.n - 1].n;
  if (capacity < need)
    return fail(h, WF_ERR_ARG, "buffer holds " + std::to_string(capacity) + " floats, the planes need " +
                                   std::to_string(need));
  DeviceGuard guard(h->dev);
  WF_CUDA(h, wf::launch_slab_copy(sg, buf, unpack, h->stream));
  return WF_OK;
}

}  // namespace

int64_t wf_slab_floats(const wf_handle *h, int nplanes) {
  if (!h || nplanes < 1 || nplanes > h->nz) return -1;
  const wf::SlabSegments sg = slab_segments(h, 0, nplanes);
  return sg.seg[sg.n - 1].off + sg.seg[sg.n - 1].n;
}

wf_status wf_slab_pack(wf_handle *h, int z0, int nplanes, float *dst, int64_t capacity) {
  return slab_copy(h, z0, nplanes, dst, capacity, false);
}

wf_status wf_slab_unpack(wf_handle *h, int z0, int nplanes, const float *src, int64_t capacity) {
  return slab_copy(h, z0, nplanes, const_cast<float *>(src), capacity, true);
}

wf_status wf_get_materials(wf_handle *h, uint8_t *ids) {
  if (!h || !ids) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaMemcpy2DAsync(ids, h->nx, h->mat, h->mat_pitch, h->nx,
                               static_cast<size_t>(h->ny) * h->nz, cudaMemcpyDeviceToHost,
                               h->stream));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  return WF_OK;
}

wf_status wf_set_pml(wf_handle *h, int axis, int T, const float *b, const float *a,
                     const float *ik) {
  if (!h || axis < 0 || axis > 2) return fail(h, WF_ERR_ARG, "bad axis");
  const int n = axis == 0 ? h->nx : (axis == 1 ? h->ny : h->nz);
  if (T < 0 || T > n) return fail(h, WF_ERR_ARG, "CPML thickness out of range");
  if (T > 0 && (!b || !a || !ik)) return fail(h, WF_ERR_ARG, "null profile");
  ++h->version;  // psi and profile arrays are reallocated
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->maps_ok = false;  // the work lists depend on the CPML slabs
  AxisState &A = h->ax[axis];
  wf::dev_free(A.prof);
  wf::dev_free(A.psi[0]);
  wf::dev_free(A.psi[1]);
  A = AxisState();
  if (T == 0) return WF_OK;
  A.T = T;
  A.W = std::min(2 * T, n);
  // x rows are padded to a multiple of 4 positions (16 bytes) for TMA
  A.pitch = axis == 0 ? (A.W + 3) / 4 * 4 : A.W;
  const long long cross = axis == 0 ? static_cast<long long>(h->ny) * h->nz
                        : axis == 1 ? static_cast<long long>(h->nx) * h->nz
                                    : static_cast<long long>(h->nx) * h->ny;
  A.cells = cross * A.pitch;
  std::vector<float> prof(3 * A.W);
  for (int s = 0; s < A.W; ++s) {
    const int c = s < T ? s : s + (n - A.W);  // slab position -> axis coordinate
    prof[s] = b[c];
    prof[A.W + s] = a[c];
    prof[2 * A.W + s] = ik[c];
  }
  WF_CUDA(h, wf::dev_alloc(&A.prof, sizeof(float) * prof.size()));
  WF_CUDA(h, h2d_sync(A.prof, prof.data(), sizeof(float) * prof.size(), h->stream));
  for (int k = 0; k < 2; ++k) {
    WF_CUDA(h, wf::dev_alloc(&A.psi[k], sizeof(float) * 4 * A.cells));
    WF_CUDA(h, memset_sync(A.psi[k], 0, sizeof(float) * 4 * A.cells, h->stream));  // PmlAux::ZERO
  }
  return WF_OK;
}

wf_status wf_add_source(wf_handle *h, int x, int y, int z, int comp, int mode,
                        const float *values, int nvalues, int *out_index) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (x < 0 || x >= h->nx || y < 0 || y >= h->ny || z < 0 || z >= h->nz)
    return fail(h, WF_ERR_ARG, "source position outside the domain");
  if (comp < 0 || comp > 2) return fail(h, WF_ERR_ARG, "source component must be Ex, Ey or Ez");
  if (mode != WF_SRC_SOFT && mode != WF_SRC_HARD_SHEET_X) return fail(h, WF_ERR_ARG, "bad source mode");
  if (nvalues < 0 || (nvalues > 0 && !values)) return fail(h, WF_ERR_ARG, "bad source values");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  SrcRec r{};
  WF_CUDA(h, wf::dev_alloc(&r.vals, sizeof(float) * std::max(nvalues, 1)));
  if (nvalues > 0)
    WF_CUDA(h, h2d_sync(r.vals, values, sizeof(float) * nvalues, h->stream));
  r.d.comp = comp;
  r.d.mode = mode;
  r.d.x = x;
  r.d.y = y;
  r.d.z = z;
  r.d.nvals = nvalues;
  r.d.vals = r.vals;
  h->srcs.push_back(r);
  if (out_index) *out_index = static_cast<int>(h->srcs.size()) - 1;
  tables_changed(h);
  return WF_OK;
}

wf_status wf_add_probe(wf_handle *h, int x, int y, int z, int comp, int nfreq,
                       const double *cos_tab, const double *sin_tab, int nsteps, int first_step,
                       int record_trace, int *out_index) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (x < 0 || x >= h->nx || y < 0 || y >= h->ny || z < 0 || z >= h->nz)
    return fail(h, WF_ERR_ARG, "probe position outside the domain");
  if (comp < 0 || comp > 5) return fail(h, WF_ERR_ARG, "probe component must be 0..5");
  if (nfreq < 0 || nsteps < 0 || first_step < 0) return fail(h, WF_ERR_ARG, "bad probe sizes");
  if (nfreq > 0 && nsteps > 0 && (!cos_tab || !sin_tab)) return fail(h, WF_ERR_ARG, "null probe tables");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  ProbeRec r{};
  const size_t tab = static_cast<size_t>(nsteps) * nfreq;
  const size_t total = 2 * tab + 2 * static_cast<size_t>(nfreq) + 1;
  WF_CUDA(h, wf::dev_alloc(&r.base, sizeof(double) * total));
  r.cos_tab = r.base;
  r.sin_tab = r.base + tab;
  r.sc = r.base + 2 * tab;
  r.ss = r.sc + nfreq;
  // one copy lays out the whole block (cos and sin tables, then zeroed DFT
  // sums); the count and the trace are cleared on the stream, and the copy
  // at the end of the call waits for all three
  {
    std::vector<double> blk(total, 0.0);
    if (tab) {
      std::memcpy(blk.data(), cos_tab, sizeof(double) * tab);
      std::memcpy(blk.data() + tab, sin_tab, sizeof(double) * tab);
    }
    WF_CUDA(h, cudaMemcpyAsync(r.base, blk.data(), sizeof(double) * total, cudaMemcpyHostToDevice,
                               h->stream));
  }
  WF_CUDA(h, wf::dev_alloc(&r.n, sizeof(unsigned long long)));
  WF_CUDA(h, cudaMemsetAsync(r.n, 0, sizeof(unsigned long long), h->stream));
  WF_CUDA(h, wf::dev_alloc(&r.trace, sizeof(float) * std::max(nsteps, 1)));
  WF_CUDA(h, cudaMemsetAsync(r.trace, 0, sizeof(float) * std::max(nsteps, 1), h->stream));
  r.d.comp = comp;
  r.d.x = x;
  r.d.y = y;
  r.d.z = z;
  r.d.nfreq = nfreq;
  r.d.nsteps = nsteps;
  r.d.first_step = first_step;
  r.d.record = record_trace ? 1 : 0;
  r.d.cos_tab = r.cos_tab;
  r.d.sin_tab = r.sin_tab;
  r.d.sc = r.sc;
  r.d.ss = r.ss;
  r.d.n = r.n;
  r.d.trace = r.trace;
  h->probes.push_back(r);
  if (out_index) *out_index = static_cast<int>(h->probes.size()) - 1;
  tables_changed(h);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));  // complete on return, as every set-up call
  return WF_OK;
}

wf_status wf_step(wf_handle *h, int nsteps) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (nsteps < 0) return fail(h, WF_ERR_ARG, "negative step count");
  if (nsteps == 0) return WF_OK;
  std::string why;
  if (!tables_cover(h, h->steps_done + nsteps, &why)) return fail(h, WF_ERR_ARG, why);
  DeviceGuard guard(h->dev);
  if (store16(h) && !use_fused(h))
    return fail(h, WF_ERR_UNSUPPORTED,
                "16-bit storage runs the fused kernel only: CPML slabs of at most 64 cells");
  if (use_fused(h) && !h->maps_ok) {  // descriptors + smem limit, outside any capture
    wf_status s = build_maps(h);
    if (s != WF_OK) return s;
  }
  if (use_fused(h) && !h->fork_ev) {  // the side streams, outside any capture too
    wf_status s = acquire_streams(h);
    if (s != WF_OK) return s;
  }
  if (h->tables_dirty) {  // sources/probes added since the last step
    wf_status s = flush_tables(h);
    if (s != WF_OK) return s;
  }
  if (store16(h) && h->shifts_dirty) {
    wf_status s = refresh_shifts(h);
    if (s != WF_OK) return s;
  }
  // Long runs replay a captured graph of an even number of steps (the
  // state buffers ping-pong, so an even count returns to the same parity).
  const int G = h->graph_steps > 0 ? h->graph_steps : 32;
  int left = nsteps;
  while (left >= G && !h->timing) {
    cudaGraphExec_t &ge = h->graph[h->cur];
    if (!ge) {
      const int cur0 = h->cur;
      const long long k0 = h->kernel_launches;
      cudaGraph_t graph;
      WF_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      wf_status st = WF_OK;
      for (int i = 0; i < G && st == WF_OK; ++i) st = enqueue_one(h);
      cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
      h->cur = cur0;
      // captured launches run at each replay, not now
      h->graph_kernels[cur0] = h->kernel_launches - k0;
      h->kernel_launches = k0;
      if (st != WF_OK) return st;
      if (ec != cudaSuccess) return cuda_fail(h, ec, "cudaStreamEndCapture");
      ec = cudaGraphInstantiate(&ge, graph, 0);
      cudaGraphDestroy(graph);
      if (ec != cudaSuccess) return cuda_fail(h, ec, "cudaGraphInstantiate");
    }
    WF_CUDA(h, cudaGraphLaunch(ge, h->stream));
    h->kernel_launches += h->graph_kernels[h->cur];
    left -= G;
    h->steps_done += G;
    if (G % 2) h->cur ^= 1;
  }
  for (; left > 0; --left) {
    wf_status st = enqueue_one(h);
    if (st != WF_OK) return st;
    h->steps_done += 1;
  }
  return WF_OK;
}

wf_status wf_sync(wf_handle *h) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->copy_pending) {
    WF_CUDA(h, cudaEventSynchronize(h->copied));
    h->copy_pending = false;
  }
  return check_device_error(h);
}

wf_status wf_reserve_download(wf_handle *h) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (store16(h))
    return fail(h, WF_ERR_UNSUPPORTED, "asynchronous downloads need FP32 storage (use wf_download_blocks)");
  DeviceGuard guard(h->dev);
  if (!h->d_stage) {
    WF_CUDA(h, wf::dev_alloc(&h->d_stage, sizeof(float) * 6 * h->N));
    WF_CUDA(h, cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking));
    WF_CUDA(h, cudaEventCreateWithFlags(&h->staged, cudaEventDisableTiming));
    WF_CUDA(h, cudaEventCreateWithFlags(&h->copied, cudaEventDisableTiming));
  }
  return WF_OK;
}

wf_status wf_download_blocks_async(wf_handle *h, void *out) {
  if (!h || !out) return fail(h, WF_ERR_ARG, "null argument");
  wf_status st = wf_reserve_download(h);
  if (st != WF_OK) return st;
  DeviceGuard guard(h->dev);
  // the staging buffer may still feed the previous download
  if (h->copy_pending) WF_CUDA(h, cudaStreamWaitEvent(h->stream, h->copied, 0));
  WF_CUDA(h, wf::launch_soa_to_blocks(h->fld[h->cur], h->d_stage, h->nx, h->ny, h->nz, h->stream));
  WF_CUDA(h, cudaEventRecord(h->staged, h->stream));
  WF_CUDA(h, cudaStreamWaitEvent(h->copy, h->staged, 0));
  WF_CUDA(h, cudaMemcpyAsync(out, h->d_stage, sizeof(float) * 6 * h->N, cudaMemcpyDeviceToHost,
                             h->copy));
  WF_CUDA(h, cudaEventRecord(h->copied, h->copy));
  h->copy_pending = true;
  h->kernel_launches += 1;  // the reorder
  return WF_OK;
}

int64_t wf_steps_done(const wf_handle *h) { return h ? h->steps_done : -1; }

int64_t wf_kernel_launches(const wf_handle *h) { return h ? h->kernel_launches : -1; }

wf_status wf_probe_sums(wf_handle *h, int p, double *c, double *s, uint64_t *n) {
  if (!h || p < 0 || p >= static_cast<int>(h->probes.size())) return fail(h, WF_ERR_ARG, "bad probe index");
  DeviceGuard guard(h->dev);
  const ProbeRec &r = h->probes[p];
  // the cos and sin sums are adjacent: one copy of both, plus the count and
  // the error flag, read on the handle's stream after the steps, one wait
  std::vector<double> cs(2 * static_cast<size_t>(r.d.nfreq));
  unsigned long long v = 0;
  int flag = 0;
  if (!cs.empty())
    WF_CUDA(h, cudaMemcpyAsync(cs.data(), r.sc, sizeof(double) * cs.size(), cudaMemcpyDeviceToHost,
                               h->stream));
  if (n) WF_CUDA(h, cudaMemcpyAsync(&v, r.n, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  WF_CUDA(h, cudaMemcpyAsync(&flag, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  if (c) std::copy(cs.begin(), cs.begin() + r.d.nfreq, c);
  if (s) std::copy(cs.begin() + r.d.nfreq, cs.end(), s);
  if (n) *n = v;
  return device_error_status(h, flag);
}

wf_status wf_probe_trace(wf_handle *h, int p, float *out, int n) {
  if (!h || p < 0 || p >= static_cast<int>(h->probes.size()) || !out) return fail(h, WF_ERR_ARG, "bad probe index");
  const ProbeRec &r = h->probes[p];
  if (n < 0 || n > r.d.nsteps) return fail(h, WF_ERR_ARG, "trace length exceeds the probe's steps");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  if (n) WF_CUDA(h, cudaMemcpy(out, r.trace, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return WF_OK;
}

// Device scratch of 6*N floats for 16-bit conversions (freed on scope exit).
struct Scratch {
  float *p = nullptr;
  ~Scratch() { wf::dev_free(p); }
};

// FP32 SoA copy of the current 16-bit state into `tmp`.
wf_status decode_current(wf_handle *h, Scratch &tmp) {
  WF_CUDA(h, wf::dev_alloc(&tmp.p, sizeof(float) * 6 * h->N));
  WF_CUDA(h, wf::launch_decode_state(h->fld[h->cur], tmp.p, h->precision, h->nx, h->ny, h->nz,
                                     h->shift[h->cur], h->stream));
  return WF_OK;
}

// Encodes the FP32 SoA state at device pointer `src` as the current state.
wf_status encode_current(wf_handle *h, const float *src) {
  WF_CUDA(h, wf::launch_encode_state(src, h->fld[h->cur], h->precision, h->nx, h->ny, h->nz,
                                     h->shift[h->cur], h->slab_max, h->d_ovf, h->stream));
  h->shifts_dirty = true;
  return WF_OK;
}

wf_status wf_get_fields(wf_handle *h, float *out6) {
  if (!h || !out6) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  if (store16(h)) {
    Scratch tmp;
    wf_status s = decode_current(h, tmp);
    if (s != WF_OK) return s;
    WF_CUDA(h, cudaMemcpyAsync(out6, tmp.p, sizeof(float) * 6 * h->N, cudaMemcpyDeviceToHost,
                               h->stream));
    WF_CUDA(h, cudaStreamSynchronize(h->stream));
    return WF_OK;
  }
  WF_CUDA(h, cudaMemcpy(out6, h->fld[h->cur], sizeof(float) * 6 * h->N, cudaMemcpyDeviceToHost));
  return WF_OK;
}

wf_status wf_set_fields(wf_handle *h, const float *in6) {
  if (!h || !in6) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  if (store16(h)) {
    Scratch tmp;
    WF_CUDA(h, wf::dev_alloc(&tmp.p, sizeof(float) * 6 * h->N));
    WF_CUDA(h, cudaMemcpyAsync(tmp.p, in6, sizeof(float) * 6 * h->N, cudaMemcpyHostToDevice,
                               h->stream));
    wf_status s = encode_current(h, tmp.p);
    if (s != WF_OK) return s;
    WF_CUDA(h, cudaStreamSynchronize(h->stream));
    return WF_OK;
  }
  WF_CUDA(h, h2d_sync(h->fld[h->cur], in6, sizeof(float) * 6 * h->N, h->stream));
  return WF_OK;
}

wf_status wf_download_blocks(wf_handle *h, void *out) {
  if (!h || !out) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  if (store16(h)) {  // decode, then reorder into a second scratch buffer
    Scratch soa, blk;
    wf_status s = decode_current(h, soa);
    if (s != WF_OK) return s;
    WF_CUDA(h, wf::dev_alloc(&blk.p, sizeof(float) * 6 * h->N));
    WF_CUDA(h, wf::launch_soa_to_blocks(soa.p, blk.p, h->nx, h->ny, h->nz, h->stream));
    WF_CUDA(h, cudaMemcpyAsync(out, blk.p, sizeof(float) * 6 * h->N, cudaMemcpyDeviceToHost,
                               h->stream));
    WF_CUDA(h, cudaStreamSynchronize(h->stream));
    return WF_OK;
  }
  // the next-state buffer is dead between steps: use it to reorder
  float *tmp = h->fld[h->cur ^ 1];
  WF_CUDA(h, wf::launch_soa_to_blocks(h->fld[h->cur], tmp, h->nx, h->ny, h->nz, h->stream));
  WF_CUDA(h, cudaMemcpyAsync(out, tmp, sizeof(float) * 6 * h->N, cudaMemcpyDeviceToHost, h->stream));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  return WF_OK;
}

wf_status wf_upload_blocks(wf_handle *h, const void *in) {
  if (!h || !in) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  if (store16(h)) {
    Scratch blk, soa;
    WF_CUDA(h, wf::dev_alloc(&blk.p, sizeof(float) * 6 * h->N));
    WF_CUDA(h, wf::dev_alloc(&soa.p, sizeof(float) * 6 * h->N));
    WF_CUDA(h, cudaMemcpyAsync(blk.p, in, sizeof(float) * 6 * h->N, cudaMemcpyHostToDevice,
                               h->stream));
    WF_CUDA(h, wf::launch_blocks_to_soa(blk.p, soa.p, h->nx, h->ny, h->nz, h->stream));
    wf_status s = encode_current(h, soa.p);
    if (s != WF_OK) return s;
    WF_CUDA(h, cudaStreamSynchronize(h->stream));
    return WF_OK;
  }
  float *tmp = h->fld[h->cur ^ 1];
  WF_CUDA(h, cudaMemcpyAsync(tmp, in, sizeof(float) * 6 * h->N, cudaMemcpyHostToDevice, h->stream));
  WF_CUDA(h, wf::launch_blocks_to_soa(tmp, h->fld[h->cur], h->nx, h->ny, h->nz, h->stream));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  return WF_OK;
}

wf_status wf_get_psi(wf_handle *h, int which, float *out) {
  if (!h || !out || which < 0 || which > 11) return fail(h, WF_ERR_ARG, "bad psi index");
  // PmlAux order (src/layout.rs:545-558) -> (axis, slot)
  static const int kAxis[12] = {0, 0, 1, 1, 2, 2, 0, 0, 1, 1, 2, 2};
  static const int kSlot[12] = {0, 1, 0, 1, 0, 1, 2, 3, 3, 2, 2, 3};
  const int axis = kAxis[which], slot = kSlot[which];
  std::fill(out, out + h->N, 0.0f);
  const AxisState &A = h->ax[axis];
  if (A.T == 0) return WF_OK;
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  std::vector<float> buf(A.cells);
  WF_CUDA(h, cudaMemcpy(buf.data(), A.psi[h->cur] + slot * A.cells, sizeof(float) * A.cells,
                        cudaMemcpyDeviceToHost));
  const int n = axis == 0 ? h->nx : (axis == 1 ? h->ny : h->nz);
  for (int z = 0; z < h->nz; ++z)
    for (int y = 0; y < h->ny; ++y)
      for (int x = 0; x < h->nx; ++x) {
        const int c = axis == 0 ? x : (axis == 1 ? y : z);
        int s = -1;
        if (c < A.T) s = c;
        else if (c >= n - A.T) s = c - (n - A.W);
        if (s < 0) continue;
        long long idx;
        if (axis == 0) idx = (static_cast<long long>(z) * h->ny + y) * A.pitch + s;
        else if (axis == 1) idx = (static_cast<long long>(z) * A.W + s) * h->nx + x;
        else idx = (static_cast<long long>(s) * h->ny + y) * h->nx + x;
        out[(static_cast<long long>(z) * h->ny + y) * h->nx + x] = buf[idx];
      }
  return WF_OK;
}

wf_status wf_storage_info(wf_handle *h, int *shift_e, int *shift_h, uint64_t *overflows) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (!store16(h)) {
    if (overflows) *overflows = 0;
    return WF_OK;
  }
  DeviceGuard guard(h->dev);
  if (h->shifts_dirty) {
    wf_status s = refresh_shifts(h);
    if (s != WF_OK) return s;
  }
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  std::vector<int> sh(2 * h->nslab);
  WF_CUDA(h, cudaMemcpy(sh.data(), h->shift[h->cur ^ 1], sizeof(int) * sh.size(),
                        cudaMemcpyDeviceToHost));
  for (int b = 0; b < h->nslab; ++b) {
    if (shift_e) shift_e[b] = sh[2 * b];
    if (shift_h) shift_h[b] = sh[2 * b + 1];
  }
  if (overflows) {
    unsigned long long v = 0;
    WF_CUDA(h, cudaMemcpy(&v, h->d_ovf, sizeof(v), cudaMemcpyDeviceToHost));
    *overflows = v;
  }
  return WF_OK;
}

wf_status wf_device_fields(wf_handle *h, float **out6) {
  if (!h || !out6) return fail(h, WF_ERR_ARG, "null argument");
  if (store16(h)) return fail(h, WF_ERR_UNSUPPORTED, "device FP32 fields need FP32 storage");
  for (int c = 0; c < 6; ++c) out6[c] = h->fld[h->cur] + c * h->N;
  return WF_OK;
}

wf_status wf_get_stream(wf_handle *h, void **out) {
  if (!h || !out) return fail(h, WF_ERR_ARG, "null argument");
  *out = h->stream;
  return WF_OK;
}

wf_status wf_set_timing(wf_handle *h, int enable) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  h->timing = enable != 0;
  h->ev_used = 0;
  return WF_OK;
}

wf_status wf_get_timing(wf_handle *h, double *total_ms, int64_t *launches) {
  if (!h || !total_ms || !launches) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  double tot = 0.0;
  for (size_t i = 0; i + 1 < h->ev_used; i += 2) {
    float ms = 0.0f;
    WF_CUDA(h, cudaEventElapsedTime(&ms, h->ev_pool[i], h->ev_pool[i + 1]));
    tot += ms;
  }
  *total_ms = tot;
  *launches = static_cast<int64_t>(h->ev_used / 2);
  return WF_OK;
}

wf_status wf_set_graph_steps(wf_handle *h, int steps) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (steps < 2 || steps > 1024 || steps % 2)
    return fail(h, WF_ERR_ARG, "graph steps must be even, in [2, 1024]");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->graph_steps = steps;
  return WF_OK;
}

wf_status wf_set_test_stall(wf_handle *h, int extra_bytes) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  if (extra_bytes < 0 || extra_bytes > 65536) return fail(h, WF_ERR_ARG, "extra_bytes outside [0, 65536]");
  drop_graphs(h);  // captured launches hold the old arguments
  h->test_extra_tx = extra_bytes;
  return WF_OK;
}

wf_status wf_get_tiling(const wf_handle *h, wf_tiling *out) {
  if (!h || !out) return WF_ERR_ARG;
  const FusedConfig c = h->cfg_user_set ? h->cfg : default_cfg(h);
  out->tile_rows = c.ty;
  out->z_chunk = c.zchunk;
  out->stages = c.stages;
  return WF_OK;
}

wf_status wf_set_tiling(wf_handle *h, const wf_tiling *t) {
  if (!h || !t) return fail(h, WF_ERR_ARG, "null argument");
  FusedConfig c{t->tile_rows, t->z_chunk, t->stages};
  if (!wf::fused_supported(c, h->precision)) return fail(h, WF_ERR_ARG, "tiling not instantiated");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->cfg = c;
  h->cfg_user_set = true;
  ++h->version;
  h->maps_ok = false;
  return WF_OK;
}

wf_status wf_set_column_tiles(wf_handle *h, int enable) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->col_pref = enable != 0;
  ++h->version;
  h->maps_ok = false;
  return WF_OK;
}

int wf_column_tiles_active(const wf_handle *h) {
  if (!h) return -1;
  if (!use_fused(h)) return 0;
  return (h->maps_ok ? h->cols : cols_apply(h)) ? 1 : 0;
}

wf_status wf_autotune(wf_handle *h, int steps, wf_tiling *best, float *best_ms) {
  if (!h || steps <= 0) return fail(h, WF_ERR_ARG, "bad autotune arguments");
  if (!use_fused(h)) return fail(h, WF_ERR_UNSUPPORTED, "autotuning applies to the fused kernel");
  if (h->steps_done != 0)
    return fail(h, WF_ERR_STATE, "autotune before the first step (it runs trial steps)");
  DeviceGuard guard(h->dev);
  // Tuning must not disturb the run: snapshot the state and restore it.
  std::vector<float> saved(6 * h->N);
  wf_status st = wf_get_fields(h, saved.data());
  if (st != WF_OK) return st;
  const FusedConfig orig = h->cfg;
  const int orig_cur = h->cur;
  h->cfg_user_set = true;  // trials and the result are explicit tilings
  std::vector<FusedConfig> cands;
  const int tys[] = {4, 8, 16};
  const int stg[] = {3, 4};
  const int zcs[] = {16, 32, 64, 128, 1 << 20};
  for (int ty : tys)
    for (int s : stg)
      for (int zc : zcs) {
        FusedConfig c{ty, std::min(zc, h->nz), s};
        if (wf::fused_supported(c, h->precision)) cands.push_back(c);
      }
  cudaEvent_t e0, e1;
  WF_CUDA(h, cudaEventCreate(&e0));
  WF_CUDA(h, cudaEventCreate(&e1));
  float bms = 1e30f;
  FusedConfig bc = orig;
  // Source/probe tails are excluded: tuning times the stencil alone.
  std::vector<SrcRec> srcs;
  std::vector<ProbeRec> probes;
  srcs.swap(h->srcs);
  probes.swap(h->probes);
  for (const FusedConfig &c : cands) {
    h->cfg = c;
    h->maps_ok = false;
    if (enqueue_one(h) != WF_OK) continue;  // warm-up and attribute set
    cudaEventRecord(e0, h->stream);
    bool okc = true;
    for (int i = 0; i < steps && okc; ++i) okc = enqueue_one(h) == WF_OK;
    cudaEventRecord(e1, h->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess || !okc) continue;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= steps;
    if (ms < bms) {
      bms = ms;
      bc = c;
    }
  }
  srcs.swap(h->srcs);
  probes.swap(h->probes);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->cfg = bc;
  h->maps_ok = false;
  drop_graphs(h);
  h->cur = orig_cur;
  // the trial steps advanced fields and psi: put the initial state back
  st = wf_set_fields(h, saved.data());
  if (st != WF_OK) return st;
  for (auto &A : h->ax)
    for (int k = 0; k < 2; ++k)
      if (A.psi[k]) WF_CUDA(h, memset_sync(A.psi[k], 0, sizeof(float) * 4 * A.cells, h->stream));
  WF_CUDA(h, memset_sync(h->d_err, 0, sizeof(int), h->stream));
  if (store16(h)) {  // the trial steps ran the 16-bit tail: rewind its counters
    WF_CUDA(h, memset_sync(h->d_step, 0, sizeof(long long), h->stream));
    WF_CUDA(h, memset_sync(h->d_ovf, 0, sizeof(unsigned long long), h->stream));
  }
  if (best) {
    best->tile_rows = bc.ty;
    best->z_chunk = bc.zchunk;
    best->stages = bc.stages;
  }
  if (best_ms) *best_ms = bms;
  return WF_OK;
}


/* ---- learned boundary closure -------------------------------------------- */

wf_status wf_set_closure(wf_handle *h, const void *w1, const void *w2, const void *w3,
                         float gain_e, float gain_h) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  if (!w1) {
    h->closure = false;
    return WF_OK;
  }
  if (!w2 || !w3) return fail(h, WF_ERR_ARG, "closure needs three weight arrays");
  if (store16(h)) return fail(h, WF_ERR_UNSUPPORTED, "the closure works on FP32 fields");
  if (h->nx != h->ny || h->ny != h->nz || h->nx < wf::kBandDepth)
    return fail(h, WF_ERR_UNSUPPORTED, "the closure needs a cubic grid");
  const size_t nw[3] = {6u * kClHidden * wf::kBandIn * 27, 6u * kClHidden * kClHidden * 27,
                        6u * 6 * kClHidden * 27};
  const void *src[3] = {w1, w2, w3};
  for (int l = 0; l < 3; ++l) {
    if (!h->cl_w[l]) WF_CUDA(h, wf::dev_alloc(&h->cl_w[l], 2 * nw[l]));
    WF_CUDA(h, h2d_sync(h->cl_w[l], src[l], 2 * nw[l], h->stream, cudaMemcpyDefault));
  }
  if (!h->cl_buf) {
    const long long P = static_cast<long long>(wf::kBandDepth) * h->nx * h->nx;
    WF_CUDA(h, wf::dev_alloc(&h->cl_buf, sizeof(float) * (6 * P * (wf::kBandIn + 2 * kClHidden + 6) + 16)));
    const int faces[6] = {0, 1, 2, 3, 4, 5};
    WF_CUDA(h, wf::dev_alloc(&h->cl_face, sizeof(faces)));
    WF_CUDA(h, h2d_sync(h->cl_face, faces, sizeof(faces), h->stream));
  }
  h->cl_ge = gain_e;
  h->cl_gh = gain_h;
  h->closure = true;
  // the tensor-core path's operands: packed weights and band buffers, and a
  // TMA map over each packed band tensor (the buffers never move).  Grids
  // narrower than one 32-voxel box row, or a map the driver refuses, keep
  // the FP32-in path.
  h->cl_fast_ok = false;
  if (encode_fn() && h->nx >= 32) {
    const int n = h->nx, D = wf::kBandDepth;
    const size_t P = static_cast<size_t>(D) * n * n;
    const size_t packed = 6 * 6 * P * 16, wbytes = 6 * 27 * 512;
    if (!h->cl_wp) WF_CUDA(h, wf::dev_alloc(&h->cl_wp, 3 * wbytes));
    if (!h->cl_fast)
      WF_CUDA(h, wf::dev_alloc(&h->cl_fast, 3 * packed + sizeof(float) * (6 * 6 * P + 64 +
                                                                          6 * wf::closure_fast_parts(n, n))));
    const int co[3] = {kClHidden, kClHidden, 6}, ci[3] = {wf::kBandIn, kClHidden, kClHidden};
    for (int l = 0; l < 3; ++l)
      WF_CUDA(h, static_cast<cudaError_t>(wf::closure_fast_pack_weights(
                     h->cl_w[l], co[l], ci[l], static_cast<unsigned char *>(h->cl_wp) + l * wbytes,
                     h->stream)));
    WF_CUDA(h, cudaStreamSynchronize(h->stream));
    // one box = one plane of a tile's input: 6 rows of 32 voxels of the six
    // arrays; x and the 8 channels of a word form one 512-byte box row
    const cuuint64_t dims[4] = {8ull * n, (cuuint64_t)n, (cuuint64_t)D, 36};
    const cuuint64_t strides[3] = {16ull * n, 16ull * n * n, 16ull * n * n * D};
    const cuuint32_t box[4] = {8 * 32, 6, 1, 6};
    bool mapped = true;
    for (int l = 0; l < 3; ++l)
      mapped = mapped && encode(&h->cl_tm[l], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, h->cl_fast + l * packed,
                                dims, strides, box);
    h->cl_fast_ok = mapped;
  }
  return WF_OK;
}

wf_status wf_set_closure_guard(wf_handle *h, int on) {
  if (!h) return fail(h, WF_ERR_ARG, "null handle");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->cl_guard = on != 0;
  return WF_OK;
}

wf_status wf_band_gather(wf_handle *h, float *X, float gain_e, float gain_h) {
  if (!h || !X) return fail(h, WF_ERR_ARG, "null argument");
  if (store16(h) || h->nx != h->ny || h->ny != h->nz)
    return fail(h, WF_ERR_UNSUPPORTED, "band moves need a cubic FP32 grid");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, static_cast<cudaError_t>(
                 wf::band_gather(band_grid(h, h->cur), X, h->nx, h->nx, gain_e, gain_h, h->stream)));
  return WF_OK;
}

wf_status wf_band_scatter_add(wf_handle *h, const float *Y, float gain_e, float gain_h) {
  if (!h || !Y) return fail(h, WF_ERR_ARG, "null argument");
  if (store16(h) || h->nx != h->ny || h->ny != h->nz)
    return fail(h, WF_ERR_UNSUPPORTED, "band moves need a cubic FP32 grid");
  DeviceGuard guard(h->dev);
  WF_CUDA(h, static_cast<cudaError_t>(wf::band_scatter_add(band_grid(h, h->cur), Y, h->nx, h->nx,
                                                           gain_e, gain_h, h->stream)));
  return WF_OK;
}

wf_status wf_restrict_state(wf_handle *teacher, wf_handle *student, int offset) {
  if (!teacher || !student) return fail(student, WF_ERR_ARG, "null handle");
  if (store16(teacher) || store16(student) || offset < 0 || student->nx + offset > teacher->nx ||
      student->ny + offset > teacher->ny || student->nz + offset > teacher->nz)
    return fail(student, WF_ERR_ARG, "the student must fit inside the teacher (FP32 grids)");
  DeviceGuard guard(student->dev);
  WF_CUDA(student, cudaStreamSynchronize(teacher->stream));
  WF_CUDA(student, static_cast<cudaError_t>(wf::band_restrict(
                       band_grid(teacher, teacher->cur), band_grid(student, student->cur), offset,
                       student->stream)));
  WF_CUDA(student, cudaStreamSynchronize(student->stream));
  return WF_OK;
}

wf_status wf_nn_conv3d_forward(const float *in, const void *w_bf16, const int32_t *face,
                               float *pre, float *out, int n, int cin, int cout, int d, int hh,
                               int ww, int gelu, void *stream) {
  WF_CUDA(nullptr, static_cast<cudaError_t>(
                       wf::nn_conv_fwd(in, w_bf16, face, pre, out, n, cin, cout, d, hh, ww, gelu, stream)));
  return WF_OK;
}

wf_status wf_nn_conv3d_backward_data(const float *dpre, const void *w_bf16, const int32_t *face,
                                     float *din, int n, int cin, int cout, int d, int hh, int ww,
                                     void *stream) {
  WF_CUDA(nullptr, static_cast<cudaError_t>(
                       wf::nn_conv_bwd_data(dpre, w_bf16, face, din, n, cin, cout, d, hh, ww, stream)));
  return WF_OK;
}

wf_status wf_nn_conv3d_backward_weight(const float *in, const float *dpre, const int32_t *face,
                                       float *dw, int n, int cin, int cout, int d, int hh, int ww,
                                       int nface, void *stream) {
  WF_CUDA(nullptr, static_cast<cudaError_t>(wf::nn_conv_bwd_weight(in, dpre, face, dw, n, cin, cout,
                                                                   d, hh, ww, nface, stream)));
  return WF_OK;
}

wf_status wf_nn_set_tensor_cores(int enable) {
  wf::nn_set_tensor_cores(enable);
  return WF_OK;
}

int64_t wf_nn_tensor_core_timeouts(void) {
  return static_cast<int64_t>(wf::nn_tc_timeouts() + wf::closure_fast_timeouts());
}

wf_status wf_nn_gelu_backward(const float *dout, const float *pre, float *dpre, int64_t m,
                              void *stream) {
  WF_CUDA(nullptr, static_cast<cudaError_t>(wf::nn_gelu_bwd(dout, pre, dpre, m, stream)));
  return WF_OK;
}

wf_status wf_nn_mse(const float *y, const float *t, float *dy, float *loss, int64_t m, void *stream) {
  WF_CUDA(nullptr, static_cast<cudaError_t>(wf::nn_mse(y, t, dy, loss, m, stream)));
  return WF_OK;
}

wf_status wf_nn_adam(float *w, void *w_bf16, const float *g, float *m1, float *m2, int64_t n,
                     float lr, float b1, float b2, float eps, int t, void *stream) {
  WF_CUDA(nullptr, static_cast<cudaError_t>(wf::nn_adam(w, w_bf16, g, m1, m2, n, lr, b1, b2, eps, t, stream)));
  return WF_OK;
}

/* ---- trajectory snapshots ---------------------------------------------- */

struct wf_snapshot_writer {
  wf_handle *h = nullptr;
  int fd = -1;
  bool direct = false;
  size_t bytes = 0;          // one snapshot
  float *d_stage = nullptr;  // the state in FieldBlock order (FP32)
  float *d_soa = nullptr;    // 16-bit storage: the decoded state
  void *host[2] = {nullptr, nullptr};  // pinned
  cudaStream_t copy = nullptr;
  cudaEvent_t staged = nullptr, copied[2] = {nullptr, nullptr};
  int last_slot = -1;  // slot of the latest copy out of d_stage
  int next_slot = 0;
  uint64_t offset = 0;   // file offset of the next capture
  uint64_t written = 0;  // bytes the writer thread has written
  std::thread thr;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<int, uint64_t>> jobs;  // (slot, file offset)
  bool busy[2] = {false, false};               // slot queued or being written
  bool stop = false;
  std::string err;  // first error of the writer thread
};

namespace {

// pwrite of n bytes at off in chunks of at most 1 GiB (src/engine.rs:602 caps
// a single O_DIRECT write the same way).  A file system that refuses
// O_DIRECT at write time gets buffered writes from then on.
std::string write_all(wf_snapshot_writer *w, const unsigned char *p, size_t n, uint64_t off) {
  while (n > 0) {
    const size_t len = std::min<size_t>(n, size_t(1) << 30);
    const ssize_t r = pwrite(w->fd, p, len, static_cast<off_t>(off));
    if (r < 0 && errno == EINTR) continue;
    if (r < 0 && errno == EINVAL && w->direct) {
      const int fl = fcntl(w->fd, F_GETFL);
      if (fl >= 0 && fcntl(w->fd, F_SETFL, fl & ~O_DIRECT) == 0) {
        w->direct = false;
        continue;
      }
    }
    if (r <= 0) return std::string("snapshot write failed: ") + std::strerror(r < 0 ? errno : EIO);
    p += r;
    n -= static_cast<size_t>(r);
    off += static_cast<uint64_t>(r);
  }
  return std::string();
}

void snapshot_thread(wf_snapshot_writer *w) {
  cudaSetDevice(w->h->dev);
  for (;;) {
    std::pair<int, uint64_t> job;
    {
      std::unique_lock<std::mutex> lk(w->mu);
      w->cv.wait(lk, [w] { return w->stop || !w->jobs.empty(); });
      if (w->jobs.empty()) return;
      job = w->jobs.front();
      w->jobs.pop_front();
    }
    const int s = job.first;
    std::string why;
    const cudaError_t e = cudaEventSynchronize(w->copied[s]);
    if (e != cudaSuccess)
      why = std::string("snapshot copy failed: ") + cudaGetErrorString(e);
    else
      why = write_all(w, static_cast<const unsigned char *>(w->host[s]), w->bytes, job.second);
    {
      std::lock_guard<std::mutex> lk(w->mu);
      if (why.empty()) w->written += w->bytes;
      if (!why.empty() && w->err.empty()) w->err = why;
      w->busy[s] = false;
    }
    w->cv.notify_all();
  }
}

// Frees everything a writer holds (the thread must have been joined).
void snapshot_free(wf_snapshot_writer *w) {
  for (void *p : w->host)
    if (p) cudaFreeHost(p);
  wf::dev_free(w->d_stage);
  wf::dev_free(w->d_soa);
  if (w->staged) cudaEventDestroy(w->staged);
  for (cudaEvent_t e : w->copied)
    if (e) cudaEventDestroy(e);
  if (w->copy) cudaStreamDestroy(w->copy);
  if (w->fd >= 0) close(w->fd);
  delete w;
}

}  // namespace

wf_status wf_snapshot_open(wf_handle *h, const char *path, wf_snapshot_writer **out) {
  if (!h || !path || !out) return fail(h, WF_ERR_ARG, "null argument");
  *out = nullptr;
  DeviceGuard guard(h->dev);
  wf_snapshot_writer *w = new wf_snapshot_writer;
  w->h = h;
  w->bytes = sizeof(float) * 6 * static_cast<size_t>(h->N);
  w->fd = open(path, O_WRONLY | O_CREAT | O_TRUNC | O_DIRECT, 0644);
  w->direct = w->fd >= 0;
  if (w->fd < 0 && errno == EINVAL) w->fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (w->fd < 0) {
    const std::string why = std::string("cannot open ") + path + ": " + std::strerror(errno);
    snapshot_free(w);
    return fail(h, WF_ERR_IO, why);
  }
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaHostAlloc(&w->host[i], w->bytes, cudaHostAllocDefault);
  if (e == cudaSuccess) e = wf::dev_alloc(&w->d_stage, w->bytes);
  if (e == cudaSuccess && store16(h)) e = wf::dev_alloc(&w->d_soa, w->bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->staged, cudaEventDisableTiming);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&w->copied[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    snapshot_free(w);
    return cuda_fail(h, e, "snapshot writer setup");
  }
  w->thr = std::thread(snapshot_thread, w);
  *out = w;
  return WF_OK;
}

wf_status wf_snapshot_capture(wf_snapshot_writer *w) {
  if (!w) return fail(nullptr, WF_ERR_ARG, "null writer");
  wf_handle *h = w->h;
  DeviceGuard guard(h->dev);
  const int s = w->next_slot;
  {
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [w, s] { return !w->busy[s]; });  // the one stall point
    if (!w->err.empty()) return fail(h, WF_ERR_IO, w->err);
  }
  // the staging buffer may still feed the previous copy
  if (w->last_slot >= 0) WF_CUDA(h, cudaStreamWaitEvent(h->stream, w->copied[w->last_slot], 0));
  const float *src = h->fld[h->cur];
  if (store16(h)) {
    WF_CUDA(h, wf::launch_decode_state(h->fld[h->cur], w->d_soa, h->precision, h->nx, h->ny, h->nz,
                                       h->shift[h->cur], h->stream));
    src = w->d_soa;
  }
  WF_CUDA(h, wf::launch_soa_to_blocks(src, w->d_stage, h->nx, h->ny, h->nz, h->stream));
  WF_CUDA(h, cudaEventRecord(w->staged, h->stream));
  WF_CUDA(h, cudaStreamWaitEvent(w->copy, w->staged, 0));
  WF_CUDA(h, cudaMemcpyAsync(w->host[s], w->d_stage, w->bytes, cudaMemcpyDeviceToHost, w->copy));
  WF_CUDA(h, cudaEventRecord(w->copied[s], w->copy));
  w->last_slot = s;
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->busy[s] = true;
    w->jobs.emplace_back(s, w->offset);
  }
  w->cv.notify_all();
  w->offset += w->bytes;
  w->next_slot ^= 1;
  return WF_OK;
}

wf_status wf_snapshot_close(wf_snapshot_writer *w, uint64_t *bytes_written) {
  if (!w) return fail(nullptr, WF_ERR_ARG, "null writer");
  wf_handle *h = w->h;
  DeviceGuard guard(h->dev);
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->stop = true;
  }
  w->cv.notify_all();
  w->thr.join();  // the thread drains the queue before it returns
  const std::string err = w->err;
  if (bytes_written) *bytes_written = w->written;
  snapshot_free(w);
  return err.empty() ? WF_OK : fail(h, WF_ERR_IO, err);
}

/* ---- checkpoint / resume ------------------------------------------------ */

namespace {

constexpr char kCkptMagic[8] = {'W', 'F', 'C', 'K', 'P', 'T', '\0', '\1'};
constexpr uint32_t kCkptVersion = 1;

// Fixed 256-byte header: the configuration the state belongs to.
struct CkptHeader {
  char magic[8];
  uint32_t version, header_bytes;
  int32_t nx, ny, nz, precision, arith, periodic[3], T[3], nsrc, nprobe, nslab;
  int64_t steps_done;
  uint64_t ovf, payload_bytes, checksum;
  unsigned char pad[256 - 8 - 8 - 4 * 14 - 8 * 4];
};
static_assert(sizeof(CkptHeader) == 256, "checkpoint header is 256 bytes");

// 64-bit FNV-1a over 8-byte little-endian words (tail bytes one by one).
struct Fnv64 {
  uint64_t v = 1469598103934665603ull;
  void add(const unsigned char *p, size_t n) {
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
      uint64_t w;
      std::memcpy(&w, p + i, 8);
      v = (v ^ w) * 1099511628211ull;
    }
    for (; i < n; ++i) v = (v ^ p[i]) * 1099511628211ull;
  }
};

// One device region of the payload.
struct CkptPiece {
  void *dev;
  size_t bytes;
};

// The shape records (sources, then probes) and the device regions of the
// payload, in file order.
void ckpt_layout(const wf_handle *h, std::vector<int32_t> *shape, std::vector<CkptPiece> *pieces) {
  for (const SrcRec &s : h->srcs)
    shape->insert(shape->end(), {s.d.x, s.d.y, s.d.z, s.d.comp, s.d.mode, s.d.nvals, 0, 0});
  for (const ProbeRec &p : h->probes)
    shape->insert(shape->end(), {p.d.x, p.d.y, p.d.z, p.d.comp, p.d.nfreq, p.d.nsteps,
                                 p.d.first_step, p.d.record});
  pieces->push_back({h->fld[h->cur], elem_bytes(h) * 6 * static_cast<size_t>(h->N)});
  if (store16(h)) {
    pieces->push_back({h->shift[h->cur], sizeof(int) * 2 * h->nslab});
    pieces->push_back({h->shift[h->cur ^ 1], sizeof(int) * 2 * h->nslab});
  }
  for (const AxisState &A : h->ax)
    if (A.T > 0) pieces->push_back({A.psi[h->cur], sizeof(float) * 4 * static_cast<size_t>(A.cells)});
  for (const ProbeRec &p : h->probes) {
    pieces->push_back({p.sc, sizeof(double) * 2 * p.d.nfreq});  // sc, then ss
    pieces->push_back({p.n, sizeof(unsigned long long)});
    if (p.d.record) pieces->push_back({p.trace, sizeof(float) * p.d.nsteps});
  }
}

CkptHeader ckpt_header(const wf_handle *h, size_t shape_bytes, const std::vector<CkptPiece> &pieces) {
  CkptHeader c;
  std::memset(&c, 0, sizeof(c));
  std::memcpy(c.magic, kCkptMagic, 8);
  c.version = kCkptVersion;
  c.header_bytes = sizeof(CkptHeader);
  c.nx = h->nx;
  c.ny = h->ny;
  c.nz = h->nz;
  c.precision = h->precision;
  c.arith = h->arith;
  for (int i = 0; i < 3; ++i) {
    c.periodic[i] = h->periodic[i];
    c.T[i] = h->ax[i].T;
  }
  c.nsrc = static_cast<int32_t>(h->srcs.size());
  c.nprobe = static_cast<int32_t>(h->probes.size());
  c.nslab = h->nslab;
  c.steps_done = h->steps_done;
  c.payload_bytes = shape_bytes;
  for (const CkptPiece &p : pieces) c.payload_bytes += p.bytes;
  return c;
}

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

struct PinnedBuf {
  unsigned char *p = nullptr;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

constexpr size_t kCkptChunk = size_t(64) << 20;

}  // namespace

wf_status wf_checkpoint_save(wf_handle *h, const char *path) {
  if (!h || !path) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  wf_status st = wf_sync(h);
  if (st != WF_OK) return st;
  if (store16(h) && h->shifts_dirty) {  // the next step's shifts are part of the state
    st = refresh_shifts(h);
    if (st != WF_OK) return st;
  }
  unsigned long long ovf = 0;
  if (store16(h)) WF_CUDA(h, cudaMemcpyAsync(&ovf, h->d_ovf, sizeof(ovf), cudaMemcpyDeviceToHost, h->stream));
  WF_CUDA(h, cudaStreamSynchronize(h->stream));
  std::vector<int32_t> shape;
  std::vector<CkptPiece> pieces;
  ckpt_layout(h, &shape, &pieces);
  CkptHeader c = ckpt_header(h, sizeof(int32_t) * shape.size(), pieces);
  c.ovf = ovf;
  File f;
  f.f = fopen(path, "wb");
  if (!f.f) return fail(h, WF_ERR_IO, std::string("cannot open ") + path + ": " + std::strerror(errno));
  PinnedBuf buf;
  WF_CUDA(h, cudaHostAlloc(reinterpret_cast<void **>(&buf.p), kCkptChunk, cudaHostAllocDefault));
  // header first (checksum filled in at the end), then the payload
  Fnv64 sum;
  bool ok = fwrite(&c, sizeof(c), 1, f.f) == 1;
  const unsigned char *sp = reinterpret_cast<const unsigned char *>(shape.data());
  sum.add(sp, sizeof(int32_t) * shape.size());
  ok = ok && (shape.empty() || fwrite(sp, sizeof(int32_t), shape.size(), f.f) == shape.size());
  for (const CkptPiece &p : pieces) {
    for (size_t off = 0; ok && off < p.bytes; off += kCkptChunk) {
      const size_t n = std::min(kCkptChunk, p.bytes - off);
      WF_CUDA(h, cudaMemcpy(buf.p, static_cast<unsigned char *>(p.dev) + off, n, cudaMemcpyDeviceToHost));
      sum.add(buf.p, n);
      ok = fwrite(buf.p, 1, n, f.f) == n;
    }
  }
  c.checksum = sum.v;
  ok = ok && fseek(f.f, 0, SEEK_SET) == 0 && fwrite(&c, sizeof(c), 1, f.f) == 1;
  ok = ok && fflush(f.f) == 0;
  if (!ok) return fail(h, WF_ERR_IO, std::string("checkpoint write failed: ") + path);
  return WF_OK;
}

wf_status wf_checkpoint_load(wf_handle *h, const char *path) {
  if (!h || !path) return fail(h, WF_ERR_ARG, "null argument");
  DeviceGuard guard(h->dev);
  wf_status st = wf_sync(h);
  if (st != WF_OK) return st;
  File f;
  f.f = fopen(path, "rb");
  if (!f.f) return fail(h, WF_ERR_IO, std::string("cannot open ") + path + ": " + std::strerror(errno));
  CkptHeader c;
  if (fread(&c, sizeof(c), 1, f.f) != 1 || std::memcmp(c.magic, kCkptMagic, 8) != 0 ||
      c.version != kCkptVersion || c.header_bytes != sizeof(CkptHeader))
    return fail(h, WF_ERR_IO, "not a checkpoint of this library version");
  std::vector<int32_t> shape;
  std::vector<CkptPiece> pieces;
  ckpt_layout(h, &shape, &pieces);
  const CkptHeader mine = ckpt_header(h, sizeof(int32_t) * shape.size(), pieces);
  const bool same = c.nx == mine.nx && c.ny == mine.ny && c.nz == mine.nz &&
                    c.precision == mine.precision && c.arith == mine.arith &&
                    std::equal(c.periodic, c.periodic + 3, mine.periodic) &&
                    std::equal(c.T, c.T + 3, mine.T) && c.nsrc == mine.nsrc &&
                    c.nprobe == mine.nprobe && c.nslab == mine.nslab &&
                    c.payload_bytes == mine.payload_bytes;
  if (!same) return fail(h, WF_ERR_ARG, "checkpoint of a differently configured grid");
  std::vector<int32_t> file_shape(shape.size());
  if (!shape.empty() && fread(file_shape.data(), sizeof(int32_t), shape.size(), f.f) != shape.size())
    return fail(h, WF_ERR_IO, "checkpoint truncated");
  if (file_shape != shape) return fail(h, WF_ERR_ARG, "checkpoint sources or probes differ");
  Fnv64 sum;
  sum.add(reinterpret_cast<const unsigned char *>(file_shape.data()), sizeof(int32_t) * shape.size());
  PinnedBuf buf;
  WF_CUDA(h, cudaHostAlloc(reinterpret_cast<void **>(&buf.p), kCkptChunk, cudaHostAllocDefault));
  for (const CkptPiece &p : pieces) {
    for (size_t off = 0; off < p.bytes; off += kCkptChunk) {
      const size_t n = std::min(kCkptChunk, p.bytes - off);
      if (fread(buf.p, 1, n, f.f) != n) return fail(h, WF_ERR_IO, "checkpoint truncated");
      sum.add(buf.p, n);
      WF_CUDA(h, h2d_sync(static_cast<unsigned char *>(p.dev) + off, buf.p, n, h->stream));
    }
  }
  if (sum.v != c.checksum) return fail(h, WF_ERR_IO, "checkpoint checksum mismatch");
  h->steps_done = c.steps_done;
  const long long step = c.steps_done;
  WF_CUDA(h, h2d_sync(h->d_step, &step, sizeof(step), h->stream));
  if (store16(h)) {
    const unsigned long long ovf = c.ovf;
    WF_CUDA(h, h2d_sync(h->d_ovf, &ovf, sizeof(ovf), h->stream));
    WF_CUDA(h, memset_sync(h->slab_max, 0, sizeof(unsigned) * 2 * h->nslab, h->stream));
    h->shifts_dirty = false;
  }
  return WF_OK;
}

/* ---- batched stepping -------------------------------------------------- */

wf_status wf_batch_create(int n, const wf_grid_desc *descs, wf_batch **out) {
  if (!out || !descs || n <= 0) return fail(nullptr, WF_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    const wf_grid_desc &d = descs[i];
    if (d.precision != WF_PREC_F32 || d.arith != WF_ARITH_EXACT || d.kernel == WF_KERNEL_SPLIT ||
        d.boundary[0] || d.boundary[1] || d.boundary[2])
      return fail(nullptr, WF_ERR_UNSUPPORTED,
                  "batched grids use FP32 storage, the exact arithmetic and zero-field boundaries");
    if (d.device != descs[0].device) return fail(nullptr, WF_ERR_ARG, "batched grids share one device");
  }
  DeviceGuard guard(descs[0].device);
  wf_batch *b = new wf_batch();
  b->dev = descs[0].device;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(nullptr, e, "cudaStreamCreate");
  }
  if ((e = wf::dev_alloc(&b->d_counter, sizeof(int) * wf::kFusedClassCount)) != cudaSuccess) {
    wf_batch_destroy(b);
    return cuda_fail(nullptr, e, "cudaMalloc(counter)");
  }
  e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
  for (int k = 0; k < wf::kFusedClassCount - 1 && e == cudaSuccess; ++k) {
    e = cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join_ev[k], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    wf_batch_destroy(b);
    return cuda_fail(nullptr, e, "side stream setup");
  }
  for (int i = 0; i < n; ++i) {
    wf_grid_desc d = descs[i];
    d.stream = b->stream;  // one stream orders every grid's calls and the batch steps
    wf_handle *h = nullptr;
    wf_status st = wf_create(&d, &h);
    if (st != WF_OK) {
      wf_batch_destroy(b);
      return st;
    }
    b->h.push_back(h);
  }
  *out = b;
  return WF_OK;
}

wf_status wf_batch_destroy(wf_batch *b) {
  if (!b) return WF_OK;
  DeviceGuard guard(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop(b);
  for (wf_handle *h : b->h) wf_destroy(h);
  wf::dev_free(b->d_counter);
  for (int k = 0; k < wf::kFusedClassCount - 1; ++k) {
    if (b->side[k]) {
      cudaStreamSynchronize(b->side[k]);
      cudaStreamDestroy(b->side[k]);
    }
    if (b->join_ev[k]) cudaEventDestroy(b->join_ev[k]);
  }
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return WF_OK;
}

int wf_batch_size(const wf_batch *b) { return b ? static_cast<int>(b->h.size()) : 0; }

wf_handle *wf_batch_handle(wf_batch *b, int i) {
  if (!b || i < 0 || i >= static_cast<int>(b->h.size())) return nullptr;
  return b->h[i];
}

wf_status wf_batch_set_tiling(wf_batch *b, const wf_tiling *t) {
  if (!b || !t) return fail(nullptr, WF_ERR_ARG, "null argument");
  FusedConfig c{t->tile_rows, t->z_chunk, t->stages};
  if (!wf::fused_supported(c, wf::kPrecF32) && !wf::fused_batch_narrow(c))
    return fail(nullptr, WF_ERR_ARG, "tiling not instantiated");
  DeviceGuard guard(b->dev);
  WF_CUDA(nullptr, cudaStreamSynchronize(b->stream));
  batch_drop(b);
  b->cfg = c;
  return WF_OK;
}

wf_status wf_batch_get_tiling(const wf_batch *b, wf_tiling *out) {
  if (!b || !out) return fail(nullptr, WF_ERR_ARG, "null argument");
  out->tile_rows = b->cfg.ty;
  out->z_chunk = b->cfg.zchunk;
  out->stages = b->cfg.stages;
  return WF_OK;
}

wf_status wf_batch_step(wf_batch *b, int nsteps) {
  if (!b) return fail(nullptr, WF_ERR_ARG, "null batch");
  if (nsteps < 0) return fail(nullptr, WF_ERR_ARG, "negative step count");
  if (nsteps == 0) return WF_OK;
  const wf_handle *h0 = b->h[0];
  std::string why;
  for (wf_handle *h : b->h) {
    if (h->steps_done != h0->steps_done || h->cur != h0->cur)
      return fail(nullptr, WF_ERR_STATE, "batched grids must have taken the same steps");
    if (!tables_cover(h, h->steps_done + nsteps, &why)) return fail(nullptr, WF_ERR_ARG, why);
  }
  DeviceGuard guard(b->dev);
  wf_status st = batch_build(b);
  if (st != WF_OK) return st;
  const int G = 32;  // even: the state buffers return to the same parity
  int left = nsteps;
  int cur = h0->cur;
  while (left >= G) {
    cudaGraphExec_t &ge = b->graph[cur];
    if (!ge) {
      cudaGraph_t graph;
      WF_CUDA(nullptr, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      wf_status s2 = WF_OK;
      for (int i = 0; i < G && s2 == WF_OK; ++i) s2 = batch_enqueue(b, (cur + i) & 1);
      cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
      if (s2 != WF_OK) return s2;
      if (ec != cudaSuccess) return cuda_fail(nullptr, ec, "cudaStreamEndCapture");
      ec = cudaGraphInstantiate(&ge, graph, 0);
      cudaGraphDestroy(graph);
      if (ec != cudaSuccess) return cuda_fail(nullptr, ec, "cudaGraphInstantiate");
    }
    WF_CUDA(nullptr, cudaGraphLaunch(ge, b->stream));
    b->launches += static_cast<long long>(G) * (b->step_kernels + (b->have_tail ? 1 : 0));
    left -= G;
  }
  for (int i = 0; i < left; ++i) {
    st = batch_enqueue(b, cur);
    if (st != WF_OK) return st;
    b->launches += b->step_kernels + (b->have_tail ? 1 : 0);
    cur ^= 1;
  }
  for (wf_handle *h : b->h) {
    h->cur = cur;
    h->steps_done += nsteps;
  }
  return WF_OK;
}

wf_status wf_batch_sync(wf_batch *b) {
  if (!b) return fail(nullptr, WF_ERR_ARG, "null batch");
  DeviceGuard guard(b->dev);
  WF_CUDA(nullptr, cudaStreamSynchronize(b->stream));
  for (wf_handle *h : b->h) {
    wf_status st = check_device_error(h);
    if (st != WF_OK) return st;
  }
  return WF_OK;
}

int64_t wf_batch_kernel_launches(const wf_batch *b) { return b ? b->launches : -1; }

wf_status wf_batch_get_stream(wf_batch *b, void **out) {
  if (!b || !out) return fail(nullptr, WF_ERR_ARG, "null argument");
  *out = b->stream;
  return WF_OK;
}

wf_status wf_batch_autotune(wf_batch *b, int steps, wf_tiling *best, float *best_ms) {
  if (!b || steps <= 0) return fail(nullptr, WF_ERR_ARG, "bad autotune arguments");
  DeviceGuard guard(b->dev);
  WF_CUDA(nullptr, cudaStreamSynchronize(b->stream));
  // Trials advance fields and psi: keep device copies of both and put them back.
  std::vector<void *> saved;
  auto free_saved = [&]() {
    for (void *p : saved) wf::dev_free(p);
  };
  for (wf_handle *h : b->h) {
    void *p = nullptr;
    if (wf::dev_alloc(&p, sizeof(float) * 6 * h->N) != cudaSuccess) {
      free_saved();
      return fail(nullptr, WF_ERR_OOM, "autotune: no room to save the state");
    }
    saved.push_back(p);
    cudaMemcpyAsync(p, h->fld[h->cur], sizeof(float) * 6 * h->N, cudaMemcpyDeviceToDevice, b->stream);
    for (auto &A : h->ax) {
      void *q = nullptr;
      if (A.T > 0) {
        if (wf::dev_alloc(&q, sizeof(float) * 4 * A.cells) != cudaSuccess) {
          free_saved();
          return fail(nullptr, WF_ERR_OOM, "autotune: no room to save the state");
        }
        cudaMemcpyAsync(q, A.psi[h->cur], sizeof(float) * 4 * A.cells, cudaMemcpyDeviceToDevice,
                        b->stream);
      }
      saved.push_back(q);
    }
  }
  const FusedConfig orig = b->cfg;
  const int cur0 = b->h[0]->cur;
  float bms = 1e30f;
  FusedConfig bc = orig;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int tys[] = {4, 8, 16, wf::kColTileRows}, stg[] = {3, 4}, zcs[] = {8, 12, 16, 24, 32, 64, 128};
  for (int ty : tys)
    for (int sg : stg)
      for (int zc : zcs) {
        FusedConfig c{ty, zc, sg};
        if (!wf::fused_supported(c, wf::kPrecF32) && !wf::fused_batch_narrow(c)) continue;
        batch_drop(b);
        b->cfg = c;
        if (batch_build(b) != WF_OK) continue;
        int parity = cur0;
        bool okc = batch_kernel(b, parity) == WF_OK;  // warm-up
        parity ^= 1;
        cudaEventRecord(e0, b->stream);
        for (int i = 0; i < steps && okc; ++i, parity ^= 1) okc = batch_kernel(b, parity) == WF_OK;
        cudaEventRecord(e1, b->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess || !okc) continue;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= steps;
        if (ms < bms) {
          bms = ms;
          bc = c;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  batch_drop(b);
  b->cfg = bc;
  size_t k = 0;
  for (wf_handle *h : b->h) {
    cudaMemcpyAsync(h->fld[h->cur], saved[k++], sizeof(float) * 6 * h->N, cudaMemcpyDeviceToDevice,
                    b->stream);
    for (auto &A : h->ax) {
      void *q = saved[k++];
      if (q)
        cudaMemcpyAsync(A.psi[h->cur], q, sizeof(float) * 4 * A.cells, cudaMemcpyDeviceToDevice,
                        b->stream);
    }
    cudaMemsetAsync(h->d_err, 0, sizeof(int), b->stream);
  }
  cudaError_t e = cudaStreamSynchronize(b->stream);
  free_saved();
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "autotune restore");
  if (best) {
    best->tile_rows = bc.ty;
    best->z_chunk = bc.zchunk;
    best->stages = bc.stages;
  }
  if (best_ms) *best_ms = bms;
  return WF_OK;
}

}  // extern "C"
