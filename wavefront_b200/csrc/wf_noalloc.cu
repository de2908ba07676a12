// wf_noalloc.cu -- an allocation-free way to advance caller-owned fields.
//
// Some callers cannot call cudaMalloc: an application whose device memory
// is owned entirely by its own pool allocator (no outside allocations
// allowed), or a latency-critical loop where an allocation, which may
// synchronise the whole device, is not acceptable.  They already hold their
// field state in device memory; wf_step_fields_noalloc advances it in place
// without allocating anything.
//
// It runs the split H and E kernels (wf_split.cu) with the caller's fields
// as one state buffer and a file-scope static device array as the other
// (the next-state buffer the kernels write).  The array has a fixed maximum
// size; every GPU that loads this library holds it until the process exits.
#include <mutex>
#include <string>

#include "../../include/wavefront_gpu.h"
#include "wf_launch.h"

namespace {

// Largest grid the static scratch can hold: 262144 cells (64^3 or any other
// shape of at most that many cells).  Six f32 components: 6 MiB per device.
constexpr long long kMaxCells = 1LL << 18;

__device__ __align__(256) float g_next_state[6 * kMaxCells];
__device__ __align__(256) float4 g_coef[256];

// Host-side stand-ins above are not device addresses; their device
// addresses are looked up with the device current, once per device and
// context: a context created anew on the device (after cudaDeviceReset, or
// another context made current) loads the module again at other addresses,
// so the lookup is repeated whenever the current context changes.
struct DeviceScratch {
  void *ctx = nullptr;  // the CUcontext the addresses belong to
  float *next_state = nullptr;
  float4 *coef = nullptr;
};
constexpr int kMaxDevices = 64;
DeviceScratch g_scratch[kMaxDevices];
std::mutex g_setup_mutex;
thread_local std::string g_err;

wf_status fail(wf_status s, const std::string &msg) {
  g_err = msg;
  return s;
}

// cuCtxGetCurrent through the runtime's driver entry point (the library
// links no libcuda).
using CtxGetCurrentFn = int (*)(void **);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<CtxGetCurrentFn>(p);
    return static_cast<CtxGetCurrentFn>(nullptr);
  }();
  return fn;
}

wf_status scratch_for_current_device(int *dev_out, DeviceScratch **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(WF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(WF_ERR_UNSUPPORTED, "device ordinal above 63");
  // the context the kernels will run in: the current one, or, when none is
  // current yet, the device's primary context (cudaSetDevice initialises
  // and binds it; it allocates nothing)
  CtxGetCurrentFn get = ctx_get_current();
  void *ctx = nullptr;
  if (!get || get(&ctx) != 0) return fail(WF_ERR_CUDA, "cuCtxGetCurrent failed");
  if (!ctx) {
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return fail(WF_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    if (get(&ctx) != 0 || !ctx) return fail(WF_ERR_CUDA, "no CUDA context on the current device");
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceScratch &s = g_scratch[dev];
  if (s.ctx != ctx) {
    s.ctx = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.next_state), g_next_state);
    if (e != cudaSuccess)
      return fail(WF_ERR_CUDA, std::string("cudaGetSymbolAddress(next state): ") + cudaGetErrorString(e));
    e = cudaGetSymbolAddress(reinterpret_cast<void **>(&s.coef), g_coef);
    if (e != cudaSuccess)
      return fail(WF_ERR_CUDA, std::string("cudaGetSymbolAddress(coefficients): ") + cudaGetErrorString(e));
    s.ctx = ctx;
  }
  *dev_out = dev;
  *out = &s;
  return WF_OK;
}

// The caller's buffers must be device (or managed) memory that the current
// device can address: a host pointer handed to the kernels would fault the
// GPU (or, where the GPU can reach host memory, silently use it).
wf_status check_device_buffer(const void *p, int dev, const char *what) {
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the (non-sticky) error the query recorded
    return fail(WF_ERR_ARG, std::string(what) + ": not a CUDA allocation (" + cudaGetErrorString(e) + ")");
  }
  if (a.type == cudaMemoryTypeManaged) return WF_OK;
  if (a.type != cudaMemoryTypeDevice)
    return fail(WF_ERR_ARG, std::string(what) + ": host memory; a device pointer is required");
  if (a.device != dev)
    return fail(WF_ERR_ARG, std::string(what) + ": memory of device " + std::to_string(a.device) +
                                ", but device " + std::to_string(dev) + " is current");
  return WF_OK;
}

}  // namespace

extern "C" {

const char *wf_noalloc_last_error(void) { return g_err.c_str(); }

wf_status wf_step_fields_noalloc(float *fields6, const uint8_t *ids,
                                 const int32_t (*table_q16)[4], int nx, int ny, int nz,
                                 const int32_t boundary[3], int arith, int nsteps,
                                 void *stream) {
  if (!fields6 || !ids || !table_q16 || !boundary) return fail(WF_ERR_ARG, "null argument");
  if (nx <= 0 || ny <= 0 || nz <= 0 || nx % 8 || ny % 8 || nz % 8)
    return fail(WF_ERR_ARG, "grid dimensions must be positive multiples of BLOCK_DIM (8)");
  const long long n = static_cast<long long>(nx) * ny * nz;
  if (n > kMaxCells)
    return fail(WF_ERR_ARG, "grid of " + std::to_string(n) +
                                " cells exceeds the allocation-free limit of " +
                                std::to_string(kMaxCells) + " cells");
  if (arith != WF_ARITH_EXACT && arith != WF_ARITH_FMA) return fail(WF_ERR_ARG, "unknown arith mode");
  if (nsteps < 0) return fail(WF_ERR_ARG, "negative step count");
  for (int i = 0; i < 3; ++i)
    if (boundary[i] != WF_BOUNDARY_ZERO && boundary[i] != WF_BOUNDARY_PERIODIC)
      return fail(WF_ERR_ARG, "unknown boundary kind");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The coefficient upload below reads a host array that lives only for
  // this call; a captured graph would replay it from a dead stack frame.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return fail(WF_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(WF_ERR_UNSUPPORTED, "the stream is capturing a graph; call outside stream capture");
  int dev = -1;
  DeviceScratch *sc = nullptr;
  wf_status st = scratch_for_current_device(&dev, &sc);
  if (st != WF_OK) return st;
  if ((st = check_device_buffer(fields6, dev, "fields6")) != WF_OK) return st;
  if ((st = check_device_buffer(ids, dev, "ids")) != WF_OK) return st;

  float4 coef[256];
  for (int m = 0; m < 256; ++m)
    coef[m] = make_float4(wf_q16_to_f32(table_q16[m][0]), wf_q16_to_f32(table_q16[m][1]),
                          wf_q16_to_f32(table_q16[m][2]), wf_q16_to_f32(table_q16[m][3]));
  // The table is rewritten on every call (the array keeps the previous
  // call's contents otherwise).  The next-state array needs no clearing:
  // each step writes every cell of it before anything reads it.
  e = cudaMemcpyAsync(sc->coef, coef, sizeof(coef), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail(WF_ERR_CUDA, std::string("coefficient upload: ") + cudaGetErrorString(e));

  wf::GridArgs g{};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.N = n;
  for (int i = 0; i < 3; ++i) g.periodic[i] = boundary[i] == WF_BOUNDARY_PERIODIC;
  g.mat = ids;
  g.mat_pitch = nx;
  g.coef = sc->coef;
  g.err = nullptr;  // the split kernels have no waits and set no flags
  float *bufs[2] = {fields6, sc->next_state};
  for (int k = 0; k < nsteps; ++k) {
    g.cur = bufs[k & 1];
    g.nxt = bufs[(k & 1) ^ 1];
    e = wf::launch_split(g, arith == WF_ARITH_FMA, s);
    if (e != cudaSuccess) return fail(WF_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
  }
  if (nsteps & 1) {  // the result is in the scratch array: copy it home
    e = cudaMemcpyAsync(fields6, sc->next_state, sizeof(float) * 6 * n, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return fail(WF_ERR_CUDA, std::string("state copy: ") + cudaGetErrorString(e));
  }
  return WF_OK;
}

}  // extern "C"
