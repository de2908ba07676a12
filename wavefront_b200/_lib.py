"""ctypes binding of libwavefront_gpu.so (include/wavefront_gpu.h).

The library is built in-tree (wavefront_b200/lib/) by wavefront_b200/build.py.
There is no fallback: if the library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# WF_BOUNDS_CHECK=1 loads the bounds-checked variant (device index checks
# that latch an error flag reported by wf_sync as WF_ERR_DEVICE_FLAG)
LIB_PATH = os.path.join(HERE, "lib", "libwavefront_gpu_checked.so"
                        if os.environ.get("WF_BOUNDS_CHECK") == "1" else "libwavefront_gpu.so")

WF_OK, WF_ERR_ARG, WF_ERR_CUDA, WF_ERR_OOM, WF_ERR_TIMEOUT, WF_ERR_DEVICE_FLAG, \
    WF_ERR_STATE, WF_ERR_UNSUPPORTED, WF_ERR_IO = range(9)

# Every symbol include/wavefront_gpu.h declares (checked by tests).
EXPORTS = [
    "wf_create", "wf_destroy", "wf_last_error", "wf_status_string", "wf_set_materials",
    "wf_set_pml", "wf_add_source", "wf_add_probe", "wf_step", "wf_sync", "wf_steps_done",
    "wf_kernel_launches", "wf_storage_info", "wf_set_scene", "wf_get_materials",
    "wf_batch_create", "wf_batch_destroy", "wf_batch_size", "wf_batch_handle", "wf_batch_step",
    "wf_batch_sync", "wf_batch_get_stream", "wf_batch_kernel_launches", "wf_batch_get_tiling",
    "wf_batch_set_tiling", "wf_batch_autotune",
    "wf_set_closure", "wf_set_closure_guard", "wf_band_gather", "wf_band_scatter_add",
    "wf_restrict_state",
    "wf_nn_conv3d_forward", "wf_nn_conv3d_backward_data", "wf_nn_conv3d_backward_weight",
    "wf_nn_gelu_backward", "wf_nn_mse", "wf_nn_adam", "wf_nn_set_tensor_cores",
    "wf_nn_tensor_core_timeouts",
    "wf_probe_sums", "wf_probe_trace", "wf_get_fields", "wf_set_fields",
    "wf_download_blocks", "wf_upload_blocks", "wf_download_blocks_async", "wf_reserve_download",
    "wf_get_psi", "wf_device_fields",
    "wf_snapshot_open", "wf_snapshot_capture", "wf_snapshot_close", "wf_set_test_stall",
    "wf_set_graph_steps",
    "wf_checkpoint_save", "wf_checkpoint_load",
    "wf_set_scene_window", "wf_slab_floats", "wf_slab_pack", "wf_slab_unpack",
    "wf_get_stream", "wf_set_timing", "wf_get_timing", "wf_get_tiling", "wf_set_tiling", "wf_autotune",
    "wf_set_column_tiles", "wf_column_tiles_active", "wf_q16_from_f32", "wf_q16_to_f32",
    "wf_material_coeffs", "wf_effective_pml_thickness_blocks", "wf_pml_profile",
    "wf_waveform_eval", "wf_source_values", "wf_probe_first_step", "wf_probe_tables",
    "wf_spectrum", "wf_scene_voxelize", "wf_demo_sphere",
    "wf_step_fields_noalloc", "wf_noalloc_last_error", "wf_release_cached_memory",
    "wf_cached_bytes",
]


class WfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"wavefront_gpu error {status}: {msg}")
        self.status = status


class GridDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("boundary", C.c_int32 * 3), ("arith", C.c_int32), ("kernel", C.c_int32),
                ("precision", C.c_int32), ("device", C.c_int32), ("stream", C.c_void_p)]


class Tiling(C.Structure):
    _fields_ = [("tile_rows", C.c_int32), ("z_chunk", C.c_int32), ("stages", C.c_int32)]


_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_h = C.c_void_p

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python wavefront_b200/build.py` "
                "(nvcc, sm_100a). There is no CPU fallback.")
        L = C.CDLL(LIB_PATH)
        S = C.c_int
        L.wf_create.argtypes = [C.POINTER(GridDesc), C.POINTER(_h)]
        L.wf_create.restype = S
        L.wf_destroy.argtypes = [_h]
        L.wf_destroy.restype = S
        L.wf_last_error.argtypes = [_h]
        L.wf_last_error.restype = C.c_char_p
        L.wf_status_string.argtypes = [S]
        L.wf_status_string.restype = C.c_char_p
        L.wf_set_materials.argtypes = [_h, _u8p, _i32p]
        L.wf_set_materials.restype = S
        L.wf_set_pml.argtypes = [_h, C.c_int, C.c_int, _f32p, _f32p, _f32p]
        L.wf_set_pml.restype = S
        L.wf_add_source.argtypes = [_h, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_int,
                                    C.POINTER(C.c_int)]
        L.wf_add_source.restype = S
        L.wf_add_probe.argtypes = [_h, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f64p, _f64p,
                                   C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.wf_add_probe.restype = S
        L.wf_step.argtypes = [_h, C.c_int]
        L.wf_step.restype = S
        L.wf_sync.argtypes = [_h]
        L.wf_sync.restype = S
        L.wf_steps_done.argtypes = [_h]
        L.wf_steps_done.restype = C.c_int64
        L.wf_kernel_launches.argtypes = [_h]
        L.wf_kernel_launches.restype = C.c_int64
        L.wf_snapshot_open.argtypes = [_h, C.c_char_p, C.POINTER(C.c_void_p)]
        L.wf_snapshot_open.restype = S
        L.wf_snapshot_capture.argtypes = [C.c_void_p]
        L.wf_snapshot_capture.restype = S
        L.wf_snapshot_close.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        L.wf_snapshot_close.restype = S
        L.wf_set_test_stall.argtypes = [_h, C.c_int]
        L.wf_set_test_stall.restype = S
        L.wf_set_graph_steps.argtypes = [_h, C.c_int]
        L.wf_set_graph_steps.restype = S
        L.wf_checkpoint_save.argtypes = [_h, C.c_char_p]
        L.wf_checkpoint_save.restype = S
        L.wf_checkpoint_load.argtypes = [_h, C.c_char_p]
        L.wf_checkpoint_load.restype = S
        L.wf_storage_info.argtypes = [_h, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_uint64)]
        L.wf_storage_info.restype = S
        L.wf_set_scene.argtypes = [_h, C.c_char_p, C.c_float, C.c_float, _i32p, C.POINTER(C.c_int)]
        L.wf_set_scene.restype = S
        L.wf_get_materials.argtypes = [_h, _u8p]
        L.wf_get_materials.restype = S
        L.wf_set_scene_window.argtypes = [_h, C.c_char_p, C.c_float, C.c_float, C.c_int, C.c_int,
                                          _i32p, C.POINTER(C.c_int)]
        L.wf_set_scene_window.restype = S
        L.wf_slab_floats.argtypes = [_h, C.c_int]
        L.wf_slab_floats.restype = C.c_int64
        L.wf_slab_pack.argtypes = [_h, C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.wf_slab_pack.restype = S
        L.wf_slab_unpack.argtypes = [_h, C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.wf_slab_unpack.restype = S
        L.wf_batch_create.argtypes = [C.c_int, C.POINTER(GridDesc), C.POINTER(_h)]
        L.wf_batch_create.restype = S
        L.wf_batch_destroy.argtypes = [_h]
        L.wf_batch_destroy.restype = S
        L.wf_batch_size.argtypes = [_h]
        L.wf_batch_size.restype = C.c_int
        L.wf_batch_handle.argtypes = [_h, C.c_int]
        L.wf_batch_handle.restype = _h
        L.wf_batch_step.argtypes = [_h, C.c_int]
        L.wf_batch_step.restype = S
        L.wf_batch_sync.argtypes = [_h]
        L.wf_batch_sync.restype = S
        L.wf_batch_get_stream.argtypes = [_h, C.POINTER(C.c_void_p)]
        L.wf_batch_get_stream.restype = S
        L.wf_batch_kernel_launches.argtypes = [_h]
        L.wf_batch_kernel_launches.restype = C.c_int64
        L.wf_batch_get_tiling.argtypes = [_h, C.POINTER(Tiling)]
        L.wf_batch_get_tiling.restype = S
        L.wf_batch_set_tiling.argtypes = [_h, C.POINTER(Tiling)]
        L.wf_batch_set_tiling.restype = S
        L.wf_batch_autotune.argtypes = [_h, C.c_int, C.POINTER(Tiling), _f32p]
        L.wf_batch_autotune.restype = S
        vp = C.c_void_p
        L.wf_set_closure.argtypes = [_h, vp, vp, vp, C.c_float, C.c_float]
        L.wf_set_closure_guard.argtypes = [_h, C.c_int]
        L.wf_band_gather.argtypes = [_h, vp, C.c_float, C.c_float]
        L.wf_band_scatter_add.argtypes = [_h, vp, C.c_float, C.c_float]
        L.wf_restrict_state.argtypes = [_h, _h, C.c_int]
        L.wf_nn_conv3d_forward.argtypes = [vp, vp, vp, vp, vp] + [C.c_int] * 7 + [vp]
        L.wf_nn_conv3d_backward_data.argtypes = [vp, vp, vp, vp] + [C.c_int] * 6 + [vp]
        L.wf_nn_conv3d_backward_weight.argtypes = [vp, vp, vp, vp] + [C.c_int] * 7 + [vp]
        L.wf_nn_gelu_backward.argtypes = [vp, vp, vp, C.c_int64, vp]
        L.wf_nn_mse.argtypes = [vp, vp, vp, vp, C.c_int64, vp]
        L.wf_nn_adam.argtypes = [vp, vp, vp, vp, vp, C.c_int64, C.c_float, C.c_float, C.c_float,
                                 C.c_float, C.c_int, vp]
        L.wf_release_cached_memory.argtypes = [C.c_int]
        L.wf_release_cached_memory.restype = S
        L.wf_cached_bytes.argtypes = [C.c_int]
        L.wf_cached_bytes.restype = C.c_int64
        L.wf_nn_set_tensor_cores.argtypes = [C.c_int]
        L.wf_nn_set_tensor_cores.restype = S
        L.wf_nn_tensor_core_timeouts.argtypes = []
        L.wf_nn_tensor_core_timeouts.restype = C.c_int64
        for name in ("wf_set_closure", "wf_set_closure_guard", "wf_band_gather", "wf_band_scatter_add", "wf_restrict_state",
                     "wf_nn_conv3d_forward", "wf_nn_conv3d_backward_data",
                     "wf_nn_conv3d_backward_weight", "wf_nn_gelu_backward", "wf_nn_mse",
                     "wf_nn_adam"):
            getattr(L, name).restype = S
        L.wf_probe_sums.argtypes = [_h, C.c_int, _f64p, _f64p, C.POINTER(C.c_uint64)]
        L.wf_probe_sums.restype = S
        L.wf_probe_trace.argtypes = [_h, C.c_int, _f32p, C.c_int]
        L.wf_probe_trace.restype = S
        L.wf_get_fields.argtypes = [_h, _f32p]
        L.wf_get_fields.restype = S
        L.wf_set_fields.argtypes = [_h, _f32p]
        L.wf_set_fields.restype = S
        L.wf_download_blocks.argtypes = [_h, C.c_void_p]
        L.wf_download_blocks.restype = S
        L.wf_upload_blocks.argtypes = [_h, C.c_void_p]
        L.wf_upload_blocks.restype = S
        L.wf_download_blocks_async.argtypes = [_h, C.c_void_p]
        L.wf_download_blocks_async.restype = S
        L.wf_reserve_download.argtypes = [_h]
        L.wf_reserve_download.restype = S
        L.wf_get_psi.argtypes = [_h, C.c_int, _f32p]
        L.wf_get_psi.restype = S
        L.wf_device_fields.argtypes = [_h, C.POINTER(C.c_void_p)]
        L.wf_device_fields.restype = S
        L.wf_get_stream.argtypes = [_h, C.POINTER(C.c_void_p)]
        L.wf_get_stream.restype = S
        L.wf_set_timing.argtypes = [_h, C.c_int]
        L.wf_set_timing.restype = S
        L.wf_get_timing.argtypes = [_h, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.wf_get_timing.restype = S
        L.wf_get_tiling.argtypes = [_h, C.POINTER(Tiling)]
        L.wf_get_tiling.restype = S
        L.wf_set_tiling.argtypes = [_h, C.POINTER(Tiling)]
        L.wf_set_tiling.restype = S
        L.wf_autotune.argtypes = [_h, C.c_int, C.POINTER(Tiling), _f32p]
        L.wf_autotune.restype = S
        L.wf_set_column_tiles.argtypes = [_h, C.c_int]
        L.wf_set_column_tiles.restype = S
        L.wf_column_tiles_active.argtypes = [_h]
        L.wf_column_tiles_active.restype = C.c_int
        L.wf_q16_from_f32.argtypes = [C.c_float]
        L.wf_q16_from_f32.restype = C.c_int32
        L.wf_q16_to_f32.argtypes = [C.c_int32]
        L.wf_q16_to_f32.restype = C.c_float
        L.wf_material_coeffs.argtypes = [C.c_float] * 5 + [_i32p]
        L.wf_effective_pml_thickness_blocks.argtypes = [C.c_int] * 4
        L.wf_effective_pml_thickness_blocks.restype = C.c_int
        L.wf_pml_profile.argtypes = [C.c_int] + [C.c_float] * 6 + [C.c_int, _f32p, _f32p, _f32p]
        L.wf_waveform_eval.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float]
        L.wf_waveform_eval.restype = C.c_float
        L.wf_source_values.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                       C.c_int, _f32p]
        L.wf_probe_first_step.argtypes = [C.c_float, C.c_float]
        L.wf_probe_first_step.restype = C.c_int
        L.wf_probe_tables.argtypes = [_f32p, C.c_int, C.c_float, C.c_int, C.c_int, _f64p, _f64p]
        L.wf_spectrum.argtypes = [_f64p, _f64p, C.c_uint64, C.c_int, _f64p, _f64p]
        L.wf_scene_voxelize.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        _u8p, _i32p, C.POINTER(C.c_int), C.c_char_p, C.c_int]
        L.wf_scene_voxelize.restype = S
        L.wf_demo_sphere.argtypes = [C.c_int, C.c_int, C.c_int, _u8p]
        L.wf_step_fields_noalloc.argtypes = [C.c_void_p, C.c_void_p, _i32p, C.c_int, C.c_int,
                                             C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_int,
                                             C.c_void_p]
        L.wf_step_fields_noalloc.restype = S
        L.wf_noalloc_last_error.argtypes = []
        L.wf_noalloc_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(status: int, handle=None) -> None:
    if status != WF_OK:
        msg = lib().wf_last_error(handle)
        raise WfError(status, msg.decode() if msg else "")


def ptr(a, t):
    return a.ctypes.data_as(t)


f32p, f64p, i32p, u8p = _f32p, _f64p, _i32p, _u8p
