//! Raw bindings of `include/wavefront_gpu.h`, the C ABI of the B200 FDTD
//! timestep library, plus a small safe [`Handle`] (module `safe`).
//!
//! The library replaces the reference engine's per-step work --
//! `step_all_slabs` (src/engine.rs:291-422), `Source::inject`
//! (src/source.rs:79-95) and `Probe::accumulate` (src/probe.rs:126-138) -- so
//! that `engine::run` (src/engine.rs:653-661) can drive a device grid.  Every
//! declaration below mirrors one of the header's, in the header's order; the
//! header's comments are the reference for each call's contract.
//!
//! This crate is source only in the tree that builds the library: that
//! build environment has no Rust toolchain, so it has not been compiled
//! there.  The same ABI is exercised from Python (ctypes) by every test.
#![allow(non_camel_case_types, non_snake_case, clippy::missing_safety_doc)]

use std::os::raw::{c_char, c_int, c_void};

pub mod safe;
pub use safe::{Error, Handle};

/// Status of every call (0 = OK).
pub type wf_status = c_int;
pub const WF_OK: wf_status = 0;
pub const WF_ERR_ARG: wf_status = 1;
pub const WF_ERR_CUDA: wf_status = 2;
pub const WF_ERR_OOM: wf_status = 3;
pub const WF_ERR_TIMEOUT: wf_status = 4;
pub const WF_ERR_DEVICE_FLAG: wf_status = 5;
pub const WF_ERR_STATE: wf_status = 6;
pub const WF_ERR_UNSUPPORTED: wf_status = 7;
pub const WF_ERR_IO: wf_status = 8;

pub const WF_BOUNDARY_ZERO: i32 = 0;
pub const WF_BOUNDARY_PERIODIC: i32 = 1;
pub const WF_ARITH_EXACT: i32 = 0;
pub const WF_ARITH_FMA: i32 = 1;
pub const WF_KERNEL_AUTO: i32 = 0;
pub const WF_KERNEL_FUSED: i32 = 1;
pub const WF_KERNEL_SPLIT: i32 = 2;
pub const WF_PREC_F32: i32 = 0;
pub const WF_PREC_BF16: i32 = 1;
pub const WF_PREC_F16: i32 = 2;

/// Grid description handed to `wf_create`.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct wf_grid_desc {
    pub nx: i32,
    pub ny: i32,
    pub nz: i32,
    pub boundary: [i32; 3],
    pub arith: i32,
    pub kernel: i32,
    pub precision: i32,
    pub device: i32,
    pub stream: *mut c_void,
}

/// Fused-kernel tiling (tile rows, z chunk, pipeline stages).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wf_tiling {
    pub tile_rows: i32,
    pub z_chunk: i32,
    pub stages: i32,
}

#[repr(C)]
pub struct wf_handle {
    _private: [u8; 0],
}
#[repr(C)]
pub struct wf_batch {
    _private: [u8; 0],
}
#[repr(C)]
pub struct wf_snapshot_writer {
    _private: [u8; 0],
}

#[link(name = "wavefront_gpu")]
extern "C" {
    pub fn wf_create(desc: *const wf_grid_desc, out: *mut *mut wf_handle) -> wf_status;
    pub fn wf_destroy(h: *mut wf_handle) -> wf_status;
    pub fn wf_last_error(h: *const wf_handle) -> *const c_char;
    pub fn wf_status_string(s: wf_status) -> *const c_char;
    pub fn wf_set_materials(h: *mut wf_handle, ids: *const u8, table_q16: *const [i32; 4]) -> wf_status;
    pub fn wf_set_scene(h: *mut wf_handle, text: *const c_char, dt: f32, dx: f32, table_q16: *mut [i32; 4], n_materials: *mut c_int) -> wf_status;
    pub fn wf_set_scene_window(h: *mut wf_handle, text: *const c_char, dt: f32, dx: f32, nz_global: c_int, z_offset: c_int, table_q16: *mut [i32; 4], n_materials: *mut c_int) -> wf_status;
    pub fn wf_get_materials(h: *mut wf_handle, ids: *mut u8) -> wf_status;
    pub fn wf_set_pml(h: *mut wf_handle, axis: c_int, thickness_voxels: c_int, b: *const f32, a: *const f32, inv_kappa: *const f32) -> wf_status;
    pub fn wf_add_source(h: *mut wf_handle, x: c_int, y: c_int, z: c_int, comp: c_int, mode: c_int, values: *const f32, nvalues: c_int, out_index: *mut c_int) -> wf_status;
    pub fn wf_add_probe(h: *mut wf_handle, x: c_int, y: c_int, z: c_int, comp: c_int, nfreq: c_int, cos_tab: *const f64, sin_tab: *const f64, nsteps: c_int, first_step: c_int, record_trace: c_int, out_index: *mut c_int) -> wf_status;
    pub fn wf_step(h: *mut wf_handle, nsteps: c_int) -> wf_status;
    pub fn wf_sync(h: *mut wf_handle) -> wf_status;
    pub fn wf_steps_done(h: *const wf_handle) -> i64;
    pub fn wf_probe_sums(h: *mut wf_handle, probe: c_int, cos_out: *mut f64, sin_out: *mut f64, n_out: *mut u64) -> wf_status;
    pub fn wf_probe_trace(h: *mut wf_handle, probe: c_int, out: *mut f32, n: c_int) -> wf_status;
    pub fn wf_get_fields(h: *mut wf_handle, out6: *mut f32) -> wf_status;
    pub fn wf_set_fields(h: *mut wf_handle, in6: *const f32) -> wf_status;
    pub fn wf_download_blocks(h: *mut wf_handle, out: *mut c_void) -> wf_status;
    pub fn wf_upload_blocks(h: *mut wf_handle, in_: *const c_void) -> wf_status;
    pub fn wf_download_blocks_async(h: *mut wf_handle, out: *mut c_void) -> wf_status;
    pub fn wf_reserve_download(h: *mut wf_handle) -> wf_status;
    pub fn wf_snapshot_open(h: *mut wf_handle, path: *const c_char, out: *mut *mut wf_snapshot_writer) -> wf_status;
    pub fn wf_snapshot_capture(w: *mut wf_snapshot_writer) -> wf_status;
    pub fn wf_snapshot_close(w: *mut wf_snapshot_writer, bytes_written: *mut u64) -> wf_status;
    pub fn wf_checkpoint_save(h: *mut wf_handle, path: *const c_char) -> wf_status;
    pub fn wf_checkpoint_load(h: *mut wf_handle, path: *const c_char) -> wf_status;
    pub fn wf_get_psi(h: *mut wf_handle, which: c_int, out: *mut f32) -> wf_status;
    pub fn wf_device_fields(h: *mut wf_handle, out6: *mut *mut f32) -> wf_status;
    pub fn wf_storage_info(h: *mut wf_handle, shift_e: *mut c_int, shift_h: *mut c_int, overflows: *mut u64) -> wf_status;
    pub fn wf_slab_floats(h: *const wf_handle, nplanes: c_int) -> i64;
    pub fn wf_slab_pack(h: *mut wf_handle, z0: c_int, nplanes: c_int, dst_device: *mut f32, capacity_floats: i64) -> wf_status;
    pub fn wf_slab_unpack(h: *mut wf_handle, z0: c_int, nplanes: c_int, src_device: *const f32, capacity_floats: i64) -> wf_status;
    pub fn wf_get_stream(h: *mut wf_handle, out_stream: *mut *mut c_void) -> wf_status;
    pub fn wf_set_timing(h: *mut wf_handle, enable: c_int) -> wf_status;
    pub fn wf_get_timing(h: *mut wf_handle, total_ms: *mut f64, launches: *mut i64) -> wf_status;
    pub fn wf_set_graph_steps(h: *mut wf_handle, steps: c_int) -> wf_status;
    pub fn wf_set_test_stall(h: *mut wf_handle, extra_bytes: c_int) -> wf_status;
    pub fn wf_kernel_launches(h: *const wf_handle) -> i64;
    pub fn wf_get_tiling(h: *const wf_handle, out: *mut wf_tiling) -> wf_status;
    pub fn wf_set_tiling(h: *mut wf_handle, t: *const wf_tiling) -> wf_status;
    pub fn wf_autotune(h: *mut wf_handle, steps: c_int, best: *mut wf_tiling, best_ms: *mut f32) -> wf_status;
    pub fn wf_set_column_tiles(h: *mut wf_handle, enable: c_int) -> wf_status;
    pub fn wf_column_tiles_active(h: *const wf_handle) -> c_int;
    pub fn wf_set_closure(h: *mut wf_handle, w1_bf16: *const c_void, w2_bf16: *const c_void, w3_bf16: *const c_void, gain_e: f32, gain_h: f32) -> wf_status;
    pub fn wf_set_closure_guard(h: *mut wf_handle, on: c_int) -> wf_status;
    pub fn wf_band_gather(h: *mut wf_handle, X: *mut f32, gain_e: f32, gain_h: f32) -> wf_status;
    pub fn wf_band_scatter_add(h: *mut wf_handle, Y: *const f32, gain_e: f32, gain_h: f32) -> wf_status;
    pub fn wf_restrict_state(teacher: *mut wf_handle, student: *mut wf_handle, offset: c_int) -> wf_status;
    pub fn wf_nn_conv3d_forward(in_: *const f32, w_bf16: *const c_void, face: *const i32, pre: *mut f32, out: *mut f32, n: c_int, cin: c_int, cout: c_int, d: c_int, h: c_int, w: c_int, gelu: c_int, stream: *mut c_void) -> wf_status;
    pub fn wf_nn_conv3d_backward_data(dpre: *const f32, w_bf16: *const c_void, face: *const i32, din: *mut f32, n: c_int, cin: c_int, cout: c_int, d: c_int, h: c_int, w: c_int, stream: *mut c_void) -> wf_status;
    pub fn wf_nn_conv3d_backward_weight(in_: *const f32, dpre: *const f32, face: *const i32, dw: *mut f32, n: c_int, cin: c_int, cout: c_int, d: c_int, h: c_int, w: c_int, nface: c_int, stream: *mut c_void) -> wf_status;
    pub fn wf_nn_gelu_backward(dout: *const f32, pre: *const f32, dpre: *mut f32, m: i64, stream: *mut c_void) -> wf_status;
    pub fn wf_nn_mse(y: *const f32, t: *const f32, dy: *mut f32, loss: *mut f32, m: i64, stream: *mut c_void) -> wf_status;
    pub fn wf_nn_adam(w: *mut f32, w_bf16: *mut c_void, g: *const f32, m1: *mut f32, m2: *mut f32, n: i64, lr: f32, b1: f32, b2: f32, eps: f32, t: c_int, stream: *mut c_void) -> wf_status;
    pub fn wf_nn_set_tensor_cores(enable: c_int) -> wf_status;
    pub fn wf_nn_tensor_core_timeouts() -> i64;
    pub fn wf_batch_create(n: c_int, descs: *const wf_grid_desc, out: *mut *mut wf_batch) -> wf_status;
    pub fn wf_batch_destroy(b: *mut wf_batch) -> wf_status;
    pub fn wf_batch_size(b: *const wf_batch) -> c_int;
    pub fn wf_batch_handle(b: *mut wf_batch, i: c_int) -> *mut wf_handle;
    pub fn wf_batch_step(b: *mut wf_batch, nsteps: c_int) -> wf_status;
    pub fn wf_batch_sync(b: *mut wf_batch) -> wf_status;
    pub fn wf_batch_get_stream(b: *mut wf_batch, out_stream: *mut *mut c_void) -> wf_status;
    pub fn wf_batch_kernel_launches(b: *const wf_batch) -> i64;
    pub fn wf_batch_get_tiling(b: *const wf_batch, out: *mut wf_tiling) -> wf_status;
    pub fn wf_batch_set_tiling(b: *mut wf_batch, t: *const wf_tiling) -> wf_status;
    pub fn wf_batch_autotune(b: *mut wf_batch, steps: c_int, best: *mut wf_tiling, best_ms: *mut f32) -> wf_status;
    pub fn wf_release_cached_memory(device: c_int) -> wf_status;
    pub fn wf_cached_bytes(device: c_int) -> i64;
    pub fn wf_step_fields_noalloc(fields6: *mut f32, ids: *const u8, table_q16: *const [i32; 4], nx: c_int, ny: c_int, nz: c_int, boundary: *const i32, arith: c_int, nsteps: c_int, stream: *mut c_void) -> wf_status;
    pub fn wf_noalloc_last_error() -> *const c_char;
    pub fn wf_q16_from_f32(v: f32) -> i32;
    pub fn wf_q16_to_f32(q: i32) -> f32;
    pub fn wf_material_coeffs(eps_r: f32, mu_r: f32, sigma: f32, dt: f32, d: f32, out_q16: *mut i32);
    pub fn wf_effective_pml_thickness_blocks(nx: c_int, ny: c_int, nz: c_int, requested_voxels: c_int) -> c_int;
    pub fn wf_pml_profile(n: c_int, grading_order: f32, kappa_max: f32, alpha_max: f32, target_reflection: f32, dt: f32, dx: f32, thickness_voxels: c_int, b: *mut f32, a: *mut f32, inv_kappa: *mut f32);
    pub fn wf_waveform_eval(kind: c_int, p0: f32, p1: f32, t: f32) -> f32;
    pub fn wf_source_values(kind: c_int, p0: f32, p1: f32, amplitude: f32, dt: f32, first_step: c_int, nsteps: c_int, values: *mut f32);
    pub fn wf_probe_first_step(start_recording_at_s: f32, dt: f32) -> c_int;
    pub fn wf_probe_tables(freqs: *const f32, nfreq: c_int, dt: f32, first_step: c_int, nsteps: c_int, cos_tab: *mut f64, sin_tab: *mut f64);
    pub fn wf_spectrum(sum_cos: *const f64, sum_sin: *const f64, n: u64, nfreq: c_int, amplitude: *mut f64, phase_rad: *mut f64);
    pub fn wf_scene_voxelize(text: *const c_char, nx: c_int, ny: c_int, nz: c_int, dt: f32, dx: f32, grid: *mut u8, table: *mut [i32; 4], n_materials: *mut c_int, err: *mut c_char, errlen: c_int) -> wf_status;
    pub fn wf_demo_sphere(nx: c_int, ny: c_int, nz: c_int, grid: *mut u8);
}
