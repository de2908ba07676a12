/*
 * wavefront_gpu.h -- C ABI of the B200 (sm_100a) FDTD timestep library.
 *
 * The library replaces the per-step hot path of the reference engine
 * (AndrejRumenovski/wavefront):
 *
 *   src/engine.rs:291-422  step_all_slabs   (H phase, barrier, E phase over
 *                                            rayon Z-slabs, calling the four
 *                                            src/fdtd.rs kernels per block)
 *   src/source.rs:79-95    Source::inject   (soft E source, after E)
 *   src/probe.rs:126-138   Probe::accumulate (f64 running DFT, after inject)
 *
 * with device code, while the setup math (src/layout.rs material table, CPML
 * profiles, src/scene.rs voxelizer, waveform evaluation) stays on the host.
 * The host helpers at the end of this header restate that setup math in the
 * library so a caller without the Rust crate gets identical tables.
 *
 * Conventions (no exceptions or aborts cross this ABI):
 *   - every call returns wf_status; wf_last_error() gives a message;
 *   - the handle owns all device memory; the caller owns host buffers, which
 *     are copied during the call;
 *   - a handle is not thread-safe; separate handles on separate streams are;
 *   - device-side error flags (bounded-wait timeouts) are latched and
 *     reported by the next wf_sync().
 *
 * Device layout (not visible through the ABI): six SoA field arrays, x
 * fastest ((z*ny+y)*nx+x), double-buffered so one fused kernel can read a
 * step's inputs and write its outputs with no cross-block hazard; a 1-byte
 * material id per voxel plus a 256-entry coefficient table; CPML psi stored
 * per axis only inside that axis's graded slab.
 */
#ifndef WAVEFRONT_GPU_H
#define WAVEFRONT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  WF_OK = 0,
  WF_ERR_ARG = 1,         /* bad argument (dims, index, table length)        */
  WF_ERR_CUDA = 2,        /* a CUDA runtime/driver call failed               */
  WF_ERR_OOM = 3,         /* device allocation failed                        */
  WF_ERR_TIMEOUT = 4,     /* a bounded device wait gave up (flag latched)    */
  WF_ERR_DEVICE_FLAG = 5, /* another device-side error flag was set          */
  WF_ERR_STATE = 6,       /* call not valid in the handle's current state    */
  WF_ERR_UNSUPPORTED = 7, /* option not supported on this device/build       */
  WF_ERR_IO = 8           /* a file could not be opened, read or written     */
} wf_status;

typedef enum { WF_BOUNDARY_ZERO = 0, WF_BOUNDARY_PERIODIC = 1 } wf_boundary;

typedef enum {
  WF_ARITH_EXACT = 0, /* separate IEEE mul/add: bit-exact with the reference */
  WF_ARITH_FMA = 1    /* fused multiply-add (<= 1e-6 relative L2)           */
} wf_arith;

typedef enum {
  WF_KERNEL_AUTO = 0,  /* fused when the grid allows it, else split          */
  WF_KERNEL_FUSED = 1, /* one TMA z-march kernel per step (zero boundaries)  */
  WF_KERNEL_SPLIT = 2  /* an H kernel then an E kernel (any boundaries)      */
} wf_kernel;

/* Field storage.  The 16-bit forms (no reference counterpart) store each
 * field value v as a 16-bit number of v * 2^-shift, round to nearest even,
 * with one power-of-two shift per z slab of 8 planes and per kind (E, H);
 * arithmetic is FP32 in the reference's order, probe sums FP64, CPML psi
 * FP32.  They need the exact arithmetic, the fused kernel (zero-field
 * boundaries, CPML slabs of at most 64 cells) and nz <= 8192; the FP32 view
 * (get/set fields, snapshots) converts at the boundary. */
typedef enum {
  WF_PREC_F32 = 0,  /* FP32 field storage (reference parity)               */
  WF_PREC_BF16 = 1, /* BF16 storage, per-slab power-of-two scale, FP32 math */
  WF_PREC_F16 = 2   /* FP16 storage, per-slab power-of-two scale, FP32 math */
} wf_precision;

/* Field component order of FieldBlock, src/layout.rs:699-706. */
enum { WF_EX = 0, WF_EY = 1, WF_EZ = 2, WF_HX = 3, WF_HY = 4, WF_HZ = 5 };

/* Source modes. */
enum {
  WF_SRC_SOFT = 0,        /* E_c[x,y,z] += v[step]; Source::inject          */
  WF_SRC_HARD_SHEET_X = 1 /* E_c[x, every y, every z] = v[step]: the hard
                             sheet source of examples/convergence_study.rs:
                             165-173 and examples/pml_reflection_study.rs   */
};

typedef struct {
  int32_t nx, ny, nz;  /* voxels; multiples of 8 (GridDims::new, src/layout.rs:60-67) */
  int32_t boundary[3]; /* wf_boundary per axis x, y, z                       */
  int32_t arith;       /* wf_arith                                           */
  int32_t kernel;      /* wf_kernel                                          */
  int32_t precision;   /* wf_precision                                       */
  int32_t device;      /* CUDA device ordinal                                */
  void *stream;        /* cudaStream_t to run on, or NULL for a private one  */
} wf_grid_desc;

typedef struct wf_handle wf_handle;

/* ---- lifetime -------------------------------------------------------- */

/* Allocates a zero-filled field grid (FieldGrid::zeroed, src/layout.rs:740)
 * with every voxel vacuum-id 0 and no CPML. */
wf_status wf_create(const wf_grid_desc *desc, wf_handle **out);
wf_status wf_destroy(wf_handle *h);
/* Message for the last failing call on h (or on this thread when h is NULL). */
const char *wf_last_error(const wf_handle *h);
const char *wf_status_string(wf_status s);

/* ---- scene upload ------------------------------------------------------ */

/* Material ids, nz*ny*nx bytes in MaterialGrid order (z,y,x; x fastest,
 * src/layout.rs:327-329), and the 256-entry Q16.16 coefficient table
 * {ca, cb, da, db} (MaterialTable, src/layout.rs:167-216).  Together they
 * replace CoeffGrid::build (src/layout.rs:230-260): the kernels dequantize
 * with FixedQ16_16::to_f32, so the FP32 multipliers are identical. */
wf_status wf_set_materials(wf_handle *h, const uint8_t *ids,
                           const int32_t (*table_q16)[4]);

/* Scene::parse + Scene::voxelize (src/scene.rs:81-230) with the ids
 * rasterized on the device: every cell starts as material 0 (vacuum), then
 * each primitive in file order overwrites the cells it covers (sphere:
 * cell-centre test in f32, box: floor/ceil clamped ranges), the ids equal
 * wf_scene_voxelize's.  table is in/out as for wf_scene_voxelize (entry 0 is
 * the caller's vacuum; registered materials are written) and is uploaded as
 * the coefficient table.  Parse errors return WF_ERR_ARG with the
 * reference's message. */
wf_status wf_set_scene(wf_handle *h, const char *text, float dt, float dx,
                       int32_t (*table_q16)[4], int *n_materials);
/* wf_set_scene for the z window [z_offset, z_offset + nz) of a scene on an
 * nx x ny x nz_global grid: the primitives are placed and clamped in the
 * global grid and the handle receives that window's planes, the ids the
 * global grid holds there (one z slab of a decomposed grid). */
wf_status wf_set_scene_window(wf_handle *h, const char *text, float dt, float dx,
                              int nz_global, int z_offset, int32_t (*table_q16)[4],
                              int *n_materials);
/* The material ids on the device, nz*ny*nx bytes (MaterialGrid order). */
wf_status wf_get_materials(wf_handle *h, uint8_t *ids);

/* CPML on one axis (0=x, 1=y, 2=z): the graded profile of that axis (n
 * entries each of b, a, 1/kappa: PmlProfile1D::build, src/layout.rs:471-513)
 * and the graded thickness T in voxels.  psi memory is kept for the cells
 * with that axis coordinate in [0,T) or [n-T,n).  Passing the same T on all
 * three axes with T a multiple of 8 reproduces PmlContext::build and the
 * PmlAuxGrid shell (src/layout.rs:594-656) bit for bit; other T values give
 * the exact per-cell layer.  T=0 removes the axis's CPML. */
wf_status wf_set_pml(wf_handle *h, int axis, int thickness_voxels,
                     const float *b, const float *a, const float *inv_kappa);

/* ---- sources and probes ------------------------------------------------ */

/* Adds a source driving E component comp (0..2) with per-step values
 * values[s] = amplitude * waveform(t_s), t_s = (s+1)*dt in f32, s counting
 * from the handle's first step (src/engine.rs:769).  Sources apply in the
 * order added, after the E update of each step. */
wf_status wf_add_source(wf_handle *h, int x, int y, int z, int comp, int mode,
                        const float *values, int nvalues, int *out_index);

/* Adds a DFT probe on component comp (0..5).  cos_tab/sin_tab hold
 * nsteps*nfreq doubles, [s*nfreq + f] = cos/sin(omega_f * (double)t_s), with
 * omega_f = 2*pi*(double)freq_f (src/probe.rs:126-138).  Steps s >=
 * first_step are accumulated (the t >= start_recording_at_s test of
 * src/probe.rs:127).  record_trace keeps the raw f32 sample of every step. */
wf_status wf_add_probe(wf_handle *h, int x, int y, int z, int comp, int nfreq,
                       const double *cos_tab, const double *sin_tab,
                       int nsteps, int first_step, int record_trace,
                       int *out_index);

/* ---- stepping ------------------------------------------------------------ */

/* Enqueues nsteps full timesteps: H everywhere, E everywhere, sources in
 * order, probes (src/engine.rs:747-782).  Asynchronous on the handle's
 * stream; long runs replay captured CUDA graphs.  The fused step forks its
 * work classes onto side streams forked from and joined back to the handle's
 * stream; the handle takes them at its first fused step, from a per-device
 * cache of idle sets that wf_destroy refills. */
wf_status wf_step(wf_handle *h, int nsteps);
/* Waits for the stream and reports any latched device error. */
wf_status wf_sync(wf_handle *h);
int64_t wf_steps_done(const wf_handle *h);

/* ---- read-back ----------------------------------------------------------- */

wf_status wf_probe_sums(wf_handle *h, int probe, double *cos_out,
                        double *sin_out, uint64_t *n_out);
wf_status wf_probe_trace(wf_handle *h, int probe, float *out, int n);
/* Six SoA host arrays (6*nz*ny*nx floats, component-major, x fastest). */
wf_status wf_get_fields(wf_handle *h, float *out6);
wf_status wf_set_fields(wf_handle *h, const float *in6);
/* Snapshot bytes in the reference's FieldBlock order (serialize_snapshot,
 * src/engine.rs:622-640): blocks (bz*nby+by)*nbx+bx, each ex..hz x 512. */
wf_status wf_download_blocks(wf_handle *h, void *out);
wf_status wf_upload_blocks(wf_handle *h, const void *in);
/* The same FieldBlock bytes, downloaded while stepping goes on (FP32
 * storage): the state is reordered on the handle's stream into a staging
 * buffer of the handle's, and copied to `out` on a copy stream of its own;
 * the call returns at once.  `out` must stay valid, and should be pinned
 * host memory for the copy to overlap, until wf_sync returns (wf_sync waits
 * for the copy).  The reference's writer overlaps its snapshot writes with
 * stepping the same way (src/engine.rs:617-640, 784-802).  The staging
 * buffer (24 bytes a voxel) is allocated at the first call, or beforehand by
 * wf_reserve_download; WF_ERR_UNSUPPORTED for 16-bit storage. */
wf_status wf_download_blocks_async(wf_handle *h, void *out);
wf_status wf_reserve_download(wf_handle *h);

/* ---- trajectory snapshots (src/engine.rs:617-640, 688-802) --------------- */

/* A writer of the reference's wave_trajectory.bin: each capture appends the
 * current state's FieldBlock bytes (wf_download_blocks' layout, nblocks *
 * 12288 bytes, no header) at offset k * that size, the stream
 * src/bin/wavefront-view.rs:280-305 reads.  The device reorders the state
 * into a staging buffer, a copy stream moves it into one of two pinned host
 * buffers, and a host thread writes that buffer to the file (O_DIRECT where
 * the file system allows it) while the handle keeps stepping.  A capture
 * waits only when both host buffers are still being written, the point at
 * which src/engine.rs:784-802 stalls too; the next capture's reorder waits
 * on the device for the previous copy out of the staging buffer.  Close the
 * writer before destroying its handle. */
typedef struct wf_snapshot_writer wf_snapshot_writer;
wf_status wf_snapshot_open(wf_handle *h, const char *path, wf_snapshot_writer **out);
wf_status wf_snapshot_capture(wf_snapshot_writer *w);
/* Waits until every capture is in the file, closes it and frees the writer
 * (also after an error); bytes_written (may be NULL) receives the bytes
 * written.  Returns the first error of any capture's write. */
wf_status wf_snapshot_close(wf_snapshot_writer *w, uint64_t *bytes_written);

/* ---- checkpoint / resume (no reference counterpart) --------------------- */

/* The complete stepping state in one file: the fields as stored (16-bit words
 * and their shifts included), every CPML psi array, probe sums and traces,
 * the step count and the binary16 saturation count, with the handle's
 * configuration (dimensions, storage, arithmetic, boundaries, CPML
 * thicknesses, source count, probe shapes) and a checksum.  Loading it into
 * a handle configured the same way (materials, CPML, sources, probes)
 * resumes the run bit for bit.  A configuration mismatch returns WF_ERR_ARG
 * before anything is changed; a damaged payload returns WF_ERR_IO and leaves
 * the handle's state undefined. */
wf_status wf_checkpoint_save(wf_handle *h, const char *path);
wf_status wf_checkpoint_load(wf_handle *h, const char *path);
/* psi of the reference PmlAux array `which` (0..11 in the declaration order
 * of src/layout.rs:545-558), as an nz*ny*nx grid, zero where none is kept. */
wf_status wf_get_psi(wf_handle *h, int which, float *out);
/* Device pointers of the current six field arrays (FP32 precision only). */
wf_status wf_device_fields(wf_handle *h, float **out6);
/* 16-bit storage: the shifts the next step stores E and H with, per z slab
 * (nz/8 entries each; either may be NULL; a slab's E and H share one shift,
 * so both arrays receive it), and a saturation count: one per step, slab and
 * kind whose largest stored binary16 magnitude was 65504 (where larger
 * values saturate).  FP32 and bfloat16 storage report 0. */
wf_status wf_storage_info(wf_handle *h, int *shift_e, int *shift_h, uint64_t *overflows);

/* ---- z-slab decomposition ------------------------------------------------ */

/* The reference splits its grid into z slabs of whole blocks for threads
 * that share one address space and read their neighbours' planes in place
 * (src/engine.rs:8-13, 291-422).  Here a grid split along z runs one handle
 * per slab: the slab's own planes plus a ghost block of neighbouring planes
 * on each inner side, refreshed by copies.  These copy the
 * complete stepping state of the planes [z0, z0 + nplanes) (six field
 * components and the x and y CPML psi of those planes) between the current
 * state and a packed device buffer of wf_slab_floats(h, nplanes) floats
 * (16-byte aligned), enqueued on the handle's stream without waiting.
 * capacity_floats is the buffer's size: a buffer smaller than the planes
 * need returns WF_ERR_ARG before anything is launched.
 * z CPML psi is not part of a slab: a decomposition keeps the z-CPML planes
 * out of every ghost block.  FP32 storage only (WF_ERR_UNSUPPORTED
 * otherwise).  wf_slab_floats returns -1 for bad arguments. */
int64_t wf_slab_floats(const wf_handle *h, int nplanes);
wf_status wf_slab_pack(wf_handle *h, int z0, int nplanes, float *dst_device,
                       int64_t capacity_floats);
wf_status wf_slab_unpack(wf_handle *h, int z0, int nplanes, const float *src_device,
                         int64_t capacity_floats);

/* The handle's CUDA stream (cudaStream_t) for event timing and interop. */
wf_status wf_get_stream(wf_handle *h, void **out_stream);
/* Kernel timing: while enabled, every step kernel launch (fused, or the
 * split H+E pair) is bracketed by CUDA events on the handle's stream and
 * steps are launched directly instead of through graphs.  wf_get_timing
 * waits for the stream and returns the summed kernel time and launch count
 * since timing was enabled. */
wf_status wf_set_timing(wf_handle *h, int enable);
wf_status wf_get_timing(wf_handle *h, double *total_ms, int64_t *launches);
/* Steps per captured CUDA graph (even, 2..1024; default 32): wf_step replays
 * graphs for whole multiples of it and launches the remainder directly, so a
 * caller that steps in chunks of k (a z slab exchanging ghost blocks every k
 * steps) sets k.  Drops the graphs captured so far. */
wf_status wf_set_graph_steps(wf_handle *h, int steps);
/* Testing aid for the device timeout path (no reference counterpart): while
 * extra_bytes > 0, every fused step kernel's CTAs expect extra_bytes more on
 * their first TMA stage than its copies deliver.  The copies land, the
 * stage's phase never completes, its bounded wait gives up after about a
 * second, and the CTA latches the timeout flag, drains its other copies and
 * exits; the next wf_sync returns WF_ERR_TIMEOUT.  No fault and no hang: the
 * GPU context stays usable for other handles.  0 (the default) turns it off;
 * the split kernels have no TMA stages and ignore it. */
wf_status wf_set_test_stall(wf_handle *h, int extra_bytes);
/* Device kernels this handle has launched for steps so far (step kernels of
 * every work class plus the source/probe tail), graph replays included. */
int64_t wf_kernel_launches(const wf_handle *h);

/* ---- fused-kernel tiling (autotuner surface) --------------------------- */

typedef struct {
  int32_t tile_rows;  /* y rows per CTA tile (x width is fixed at 128)      */
  int32_t z_chunk;    /* planes per CTA z-march                            */
  int32_t stages;     /* TMA pipeline depth                                */
} wf_tiling;

wf_status wf_get_tiling(const wf_handle *h, wf_tiling *out);
wf_status wf_set_tiling(wf_handle *h, const wf_tiling *t);
/* Times each candidate tiling for `steps` steps and keeps the fastest. */
wf_status wf_autotune(wf_handle *h, int steps, wf_tiling *best, float *best_ms);
/* Fused-kernel work layout of the x-CPML slabs (no counterpart in the
 * reference, whose rayon slabs split along z only, src/engine.rs:291-422).
 * With column tiles on (the default), the two x slabs run as tiles 16 cells
 * wide and 32 rows tall in which every lane holds graded cells, and the wide
 * 128-cell tiles cover x in [16, nx-16) with no x-psi work; this applies when
 * the x CPML is at most 16 cells deep and nx >= 48.  Off: the wide tiles
 * cover the whole x range and their edge lanes run the x-psi recursion.
 * Results are bit-identical either way. */
wf_status wf_set_column_tiles(wf_handle *h, int enable);
/* 1 when the handle's fused step uses column tiles, 0 otherwise, -1 on a
 * null handle. */
int wf_column_tiles_active(const wf_handle *h);

/* ---- learned boundary closure (no reference counterpart) ---------------- */

/* A per-face 3-layer 3D conv network (3x3x3 kernels, channels 10 -> 16 -> 16
 * -> 6, GELU after the first two layers, no bias, bfloat16 weights, FP32
 * accumulation) that corrects the fields in the 8-cell band next to each
 * face of a grid with a thin CPML.  Its input is the band's six fields and
 * the four psi terms of the face's normal axis, E-side values times gain_e
 * and H-side values times gain_h, each face's band then divided by the RMS
 * of its E channels; its output, times that RMS and divided by the gains,
 * is added to the band's fields after every step kernel (before sources and
 * probes).  Band tensors are [6 faces][channels][8][n][n] (cubic grids:
 * face f has normal axis f/2, at the low side for even f; distance 0 is the
 * outermost cell; the two tangential axes follow in increasing order).
 * Weights are device or host arrays of bfloat16 [6][cout][cin][27]. */
wf_status wf_set_closure(wf_handle *h, const void *w1_bf16, const void *w2_bf16,
                         const void *w3_bf16, float gain_e, float gain_h);  /* w1 NULL: off */
/* Energy guard of the closure (off by default): per face, the correction is
 * scaled by the largest factor in [0, 1] that keeps it from raising the sum
 * of squares of the band's six fields in the gained units (with gain_h = 377
 * gain_e, the field energy density up to a constant).  It is not a stability
 * guarantee: the Yee scheme's conserved energy pairs E and H at staggered
 * times, and the CPML's psi is not covered. */
wf_status wf_set_closure_guard(wf_handle *h, int on);
/* The current state's bands into device X[6][10][8][n][n] (scaled as above).
 * Both band moves are enqueued on the handle's own (non-blocking) stream: a
 * caller that produces Y or consumes X on another stream orders the two
 * itself (wf_sync, or an event). */
wf_status wf_band_gather(wf_handle *h, float *X, float gain_e, float gain_h);
/* fields += Y[6][6][8][n][n] / gain over the current state's bands. */
wf_status wf_band_scatter_add(wf_handle *h, const float *Y, float gain_e, float gain_h);
/* Student state = teacher state restricted to the student's extent at
 * `offset` cells on every axis: fields, and the student's psi from the
 * teacher's psi at the same cells (zero where the teacher keeps none). */
wf_status wf_restrict_state(wf_handle *teacher, wf_handle *student, int offset);

/* The closure network's training kernels on device arrays (stream: a
 * cudaStream_t or NULL).  Tensors are [n][c][d][h][w]; sample i uses the
 * weights of face[i] (face NULL: all use face 0); weights bfloat16
 * [faces][cout][cin][27]; accumulation FP32.  forward: pre (may be NULL) =
 * conv(in), out = GELU(pre) if gelu else pre.  backward_data: din =
 * conv^T(dpre).  backward_weight: dw[face] += sum over the face's samples.
 * mse: loss += mean((y-t)^2), dy = 2(y-t)/m.  adam: one Adam step on FP32
 * master weights w (t counts from 1), refreshing the bfloat16 copy. */
wf_status wf_nn_conv3d_forward(const float *in, const void *w_bf16, const int32_t *face,
                               float *pre, float *out, int n, int cin, int cout, int d, int h,
                               int w, int gelu, void *stream);
wf_status wf_nn_conv3d_backward_data(const float *dpre, const void *w_bf16, const int32_t *face,
                                     float *din, int n, int cin, int cout, int d, int h, int w,
                                     void *stream);
wf_status wf_nn_conv3d_backward_weight(const float *in, const float *dpre, const int32_t *face,
                                       float *dw, int n, int cin, int cout, int d, int h, int w,
                                       int nface, void *stream);
wf_status wf_nn_gelu_backward(const float *dout, const float *pre, float *dpre, int64_t m,
                              void *stream);
wf_status wf_nn_mse(const float *y, const float *t, float *dy, float *loss, int64_t m, void *stream);
wf_status wf_nn_adam(float *w, void *w_bf16, const float *g, float *m1, float *m2, int64_t n,
                     float lr, float b1, float b2, float eps, int t, void *stream);
/* Which kernels run conv3d_forward and conv3d_backward_data (process-wide):
 * 1 (default) the tensor cores -- tcgen05 implicit GEMMs, 128 voxels x 16
 * channels per tile, FP32 activations split into two bfloat16 parts so the
 * operands keep 16 significant bits, FP32 accumulation in tensor memory --
 * or 0 the FP32 CUDA-core kernels.  The two agree to about 1e-6 relative. */
wf_status wf_nn_set_tensor_cores(int enable);
/* Tensor-core convolution tiles whose bounded completion wait ran out
 * (their outputs were not written); 0 in a healthy run. */
int64_t wf_nn_tensor_core_timeouts(void);

/* ---- batched stepping (no reference counterpart) ------------------------ */

/* Many independent grids of uneven size stepped together: each step is one
 * persistent kernel launch over the work items (tile x z chunk) of every
 * grid, then one tail launch for every grid's sources and probes; runs of
 * 32 steps replay a captured CUDA graph.  The grids are ordinary handles,
 * created on the batch's stream: set them up and read them back with the
 * per-grid calls through wf_batch_handle (wf_step on one of them is allowed
 * but breaks the lockstep that wf_batch_step requires).  Every grid needs
 * FP32 storage, the exact arithmetic, zero-field boundaries and CPML slabs
 * of at most 64 cells; results equal wf_step's bit for bit. */
typedef struct wf_batch wf_batch;
wf_status wf_batch_create(int n, const wf_grid_desc *descs, wf_batch **out);
wf_status wf_batch_destroy(wf_batch *b);
int wf_batch_size(const wf_batch *b);
wf_handle *wf_batch_handle(wf_batch *b, int i);
/* Steps every grid nsteps times (all must have taken the same steps). */
wf_status wf_batch_step(wf_batch *b, int nsteps);
/* Waits for the batch's stream; reports any grid's latched device error. */
wf_status wf_batch_sync(wf_batch *b);
wf_status wf_batch_get_stream(wf_batch *b, void **out_stream);
/* Kernel launches issued for batched steps so far (graph replays included). */
int64_t wf_batch_kernel_launches(const wf_batch *b);
wf_status wf_batch_get_tiling(const wf_batch *b, wf_tiling *out);
wf_status wf_batch_set_tiling(wf_batch *b, const wf_tiling *t);
/* Times the batched step kernel for `steps` steps under each instantiated
 * tiling and z chunk, keeps the fastest, and restores every grid's fields
 * and psi (sources and probes do not run during the trials). */
wf_status wf_batch_autotune(wf_batch *b, int steps, wf_tiling *best, float *best_ms);

/* ---- device memory cache (no reference counterpart) ---------------------- */

/* Device blocks the library frees (a destroyed handle's state buffers,
 * material ids, psi arrays and tables) are kept in a per-device cache, at
 * most 16 GiB per device, and handed to the next allocation of the same
 * rounded size, so a handle created after another of the same shape skips
 * CUDA's page mapping.  Freeing waits for the device first, as cudaFree
 * does.  An allocation that runs out of memory returns the device's cache
 * to CUDA and tries again.  wf_release_cached_memory returns the cache of
 * `device` (-1: every device) to CUDA now, and destroys the idle side-stream
 * sets kept for the fused step (call it before resetting a device that the
 * library has used); wf_cached_bytes reports the cached bytes. */
wf_status wf_release_cached_memory(int device);
int64_t wf_cached_bytes(int device);

/* ---- allocation-free stepping of caller-owned fields --------------------- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * -- an application whose device memory belongs entirely to its own pool
 * allocator, or a latency-critical loop in which an allocation (which can
 * synchronise the device) is not allowed.  Advances the caller's device
 * fields in place by nsteps Yee steps with no CPML, sources or probes:
 *   fields6   device pointer, 6*nx*ny*nz floats, component-major ex..hz,
 *             x fastest (the layout wf_device_fields reports);
 *   ids       device pointer, nz*ny*nx material ids (MaterialGrid order);
 *   table_q16 host pointer, the 256-entry Q16.16 table {ca, cb, da, db};
 *   boundary  wf_boundary per axis; arith wf_arith; stream cudaStream_t.
 * Allocates nothing: the next-state buffer is a static device array of at
 * most 262144 cells (6 MiB, held by every GPU that loads the library until
 * the process exits); larger grids are rejected with WF_ERR_ARG.  The first
 * call on a device (and the first after a new context is made current on it)
 * looks up that array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture.  fields6 and ids must be device or managed
 * memory of the current device: a host pointer or another device's memory is
 * refused with WF_ERR_ARG before anything is launched.  Each call uploads the
 * coefficient table from a host array that lives only for the call, so a call
 * on a stream that is capturing a graph is refused with WF_ERR_UNSUPPORTED.
 * Every call shares the array, so calls that overlap on the GPU (other
 * streams, other threads) race.  Results are bit-identical to wf_step on a
 * handle with the same inputs.  Errors are described by
 * wf_noalloc_last_error(). */
wf_status wf_step_fields_noalloc(float *fields6, const uint8_t *ids,
                                 const int32_t (*table_q16)[4], int nx, int ny,
                                 int nz, const int32_t boundary[3], int arith,
                                 int nsteps, void *stream);
const char *wf_noalloc_last_error(void);

/* ---- host helpers: the reference's setup math ---------------------------- */

int32_t wf_q16_from_f32(float v);   /* FixedQ16_16::from_f32, src/layout.rs:114-116 */
float wf_q16_to_f32(int32_t q);     /* FixedQ16_16::to_f32,   src/layout.rs:123-125 */
/* MaterialTable::coeffs_from_physical, src/layout.rs:194-208 */
void wf_material_coeffs(float eps_r, float mu_r, float sigma, float dt, float d,
                        int32_t out_q16[4]);
/* effective_pml_thickness_blocks, src/layout.rs:525-533 */
int wf_effective_pml_thickness_blocks(int nx, int ny, int nz, int requested_voxels);
/* PmlProfile1D::build, src/layout.rs:471-513 (PmlConfig fields spelled out) */
void wf_pml_profile(int n, float grading_order, float kappa_max,
                    float alpha_max, float target_reflection, float dt,
                    float dx, int thickness_voxels, float *b, float *a,
                    float *inv_kappa);
/* Waveform::evaluate, src/source.rs:46-59.  kind 0 GaussianPulse(p0=t0,
 * p1=spread), 1 Sinusoid(p0=freq), 2 RickerWavelet(p0=peak_freq, p1=t0). */
float wf_waveform_eval(int kind, float p0, float p1, float t);
/* values[i] = amplitude * evaluate(((first_step+i) as f32 + 1) * dt). */
void wf_source_values(int kind, float p0, float p1, float amplitude, float dt,
                      int first_step, int nsteps, float *values);
/* First step index whose t=(s+1)*dt is not below start (src/probe.rs:127). */
int wf_probe_first_step(float start_recording_at_s, float dt);
/* cos/sin tables for wf_add_probe, steps [first_step, first_step+nsteps). */
void wf_probe_tables(const float *freqs, int nfreq, float dt, int first_step,
                     int nsteps, double *cos_tab, double *sin_tab);
/* Probe::spectrum, src/probe.rs:143-167. */
void wf_spectrum(const double *sum_cos, const double *sum_sin, uint64_t n,
                 int nfreq, double *amplitude, double *phase_rad);
/* Scene::parse + Scene::voxelize, src/scene.rs:81-230.  grid must hold
 * nx*ny*nz bytes (left as given outside primitives); table[id] receives the
 * Q16.16 coefficients of each registered material.  Returns WF_ERR_ARG with
 * the reference's message in err on a parse error. */
wf_status wf_scene_voxelize(const char *text, int nx, int ny, int nz, float dt,
                            float dx, uint8_t *grid, int32_t (*table)[4],
                            int *n_materials, char *err, int errlen);
/* voxelize_demo_sphere, src/main.rs:403-425 (material id 1). */
void wf_demo_sphere(int nx, int ny, int nz, uint8_t *grid);

#ifdef __cplusplus
}
#endif
#endif /* WAVEFRONT_GPU_H */
