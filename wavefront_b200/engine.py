"""The device field grid and the run loop, mirroring src/engine.rs of the reference.

`DeviceFieldGrid` owns one C-ABI handle: the double-buffered SoA field state,
material ids, coefficient table, CPML psi, sources and probes on one GPU.
`run()` keeps engine::run's contract (src/engine.rs:653-819): each step is
H everywhere, E everywhere, sources in order, probes, and an optional
snapshot when step % snapshot_every == 0, handed to a callback in the
reference's FieldBlock byte order (the host writer stays with the caller).
"""
from __future__ import annotations

import ctypes as C
import os
import time
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib as _L
from .layout import GridDims, MaterialGrid, MaterialTable, PmlContext

_BOUNDARY = {"zero": 0, "periodic": 1}
_ARITH = {"exact": 0, "fma": 1}
_KERNEL = {"auto": 0, "fused": 1, "split": 2}
# field storage: FP32 (reference parity) or 16-bit with per-slab power-of-two
# scales (wf_precision)
_PRECISION = {"f32": 0, "bf16": 1, "f16": 2}

# PmlAux array order of src/layout.rs:545-558
PSI_NAMES = ["psi_ez_dx", "psi_ey_dx", "psi_ez_dy", "psi_ex_dy", "psi_ey_dz", "psi_ex_dz",
             "psi_hz_dx", "psi_hy_dx", "psi_hx_dy", "psi_hz_dy", "psi_hy_dz", "psi_hx_dz"]


class DeviceFieldGrid:
    def __init__(self, dims: GridDims, boundary=("zero", "zero", "zero"), arith: str = "exact",
                 kernel: str = "auto", device: int = 0, stream: Optional[int] = None,
                 precision: str = "f32"):
        self.dims = dims
        self.precision = precision
        d = _L.GridDesc()
        d.nx, d.ny, d.nz = dims.nx, dims.ny, dims.nz
        for i, b in enumerate(boundary):
            d.boundary[i] = _BOUNDARY[b]
        d.arith = _ARITH[arith]
        d.kernel = _KERNEL[kernel]
        d.precision = _PRECISION[precision]
        d.device = device
        d.stream = stream
        h = C.c_void_p()
        _L.check(_L.lib().wf_create(C.byref(d), C.byref(h)))
        self._h = h
        self._owned = True
        self.n_sources = 0
        self.n_probes = 0

    @classmethod
    def _member(cls, handle, dims: GridDims) -> "DeviceFieldGrid":
        """A view of a grid owned by a DeviceBatch (closing it frees nothing)."""
        g = cls.__new__(cls)
        g.dims = dims
        g.precision = "f32"
        g._h = C.c_void_p(handle)
        g._owned = False
        g.n_sources = 0
        g.n_probes = 0
        return g

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                _L.lib().wf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, st):
        _L.check(st, self._h)

    # -- scene ---------------------------------------------------------------
    def set_materials(self, grid: MaterialGrid, table: MaterialTable):
        ids = np.ascontiguousarray(grid.ids, np.uint8)
        q = np.ascontiguousarray(table.q16, np.int32)
        self._chk(_L.lib().wf_set_materials(self._h, _L.ptr(ids, _L.u8p), _L.ptr(q, _L.i32p)))

    def set_scene(self, text: str, table: MaterialTable, dt: float, dx: float) -> int:
        """Scene text voxelized on the device (ids start as vacuum 0); the
        registered materials are written into `table`, which becomes the
        coefficient table.  Returns the number of registered materials."""
        q = np.ascontiguousarray(table.q16, np.int32)
        n = C.c_int()
        self._chk(_L.lib().wf_set_scene(self._h, text.encode(), dt, dx, _L.ptr(q, _L.i32p),
                                        C.byref(n)))
        table.q16[:] = q
        return n.value

    def set_scene_window(self, text: str, table: MaterialTable, dt: float, dx: float,
                         nz_global: int, z_offset: int) -> int:
        """set_scene for the planes [z_offset, z_offset + nz) of the scene on
        an nx x ny x nz_global grid (one z slab of a decomposed grid)."""
        q = np.ascontiguousarray(table.q16, np.int32)
        n = C.c_int()
        self._chk(_L.lib().wf_set_scene_window(self._h, text.encode(), dt, dx, nz_global,
                                               z_offset, _L.ptr(q, _L.i32p), C.byref(n)))
        table.q16[:] = q
        return n.value

    def materials(self) -> np.ndarray:
        """The device material ids, nz*ny*nx bytes."""
        out = np.empty(self.dims.voxel_count(), np.uint8)
        self._chk(_L.lib().wf_get_materials(self._h, _L.ptr(out, _L.u8p)))
        return out

    def set_pml(self, ctx: PmlContext):
        for axis in range(3):
            p = ctx.profiles[axis]
            t = ctx.thickness_voxels[axis]
            self._chk(_L.lib().wf_set_pml(self._h, axis, t, _L.ptr(p.b, _L.f32p),
                                          _L.ptr(p.a, _L.f32p), _L.ptr(p.inv_kappa, _L.f32p)))

    def set_pml_axis(self, axis: int, thickness: int, b, a, inv_kappa):
        b, a, k = (np.ascontiguousarray(v, np.float32) for v in (b, a, inv_kappa))
        self._chk(_L.lib().wf_set_pml(self._h, axis, thickness, _L.ptr(b, _L.f32p),
                                      _L.ptr(a, _L.f32p), _L.ptr(k, _L.f32p)))

    def add_source_values(self, x, y, z, comp, values, mode=0) -> int:
        v = np.ascontiguousarray(values, np.float32)
        idx = C.c_int()
        self._chk(_L.lib().wf_add_source(self._h, x, y, z, int(comp), mode, _L.ptr(v, _L.f32p),
                                         len(v), C.byref(idx)))
        self.n_sources += 1
        return idx.value

    def add_probe_tables(self, x, y, z, comp, cos_tab, sin_tab, first_step=0,
                         record_trace=False) -> int:
        c = np.ascontiguousarray(cos_tab, np.float64)
        s = np.ascontiguousarray(sin_tab, np.float64)
        nsteps = c.shape[0]
        nfreq = c.shape[1] if c.ndim == 2 else 0
        idx = C.c_int()
        self._chk(_L.lib().wf_add_probe(self._h, x, y, z, int(comp), nfreq, _L.ptr(c, _L.f64p),
                                        _L.ptr(s, _L.f64p), nsteps, first_step, int(record_trace),
                                        C.byref(idx)))
        self.n_probes += 1
        return idx.value

    # -- stepping -------------------------------------------------------------
    def step(self, n: int = 1):
        self._chk(_L.lib().wf_step(self._h, n))

    def sync(self):
        self._chk(_L.lib().wf_sync(self._h))

    @property
    def steps_done(self) -> int:
        return int(_L.lib().wf_steps_done(self._h))

    def storage_info(self):
        """16-bit storage: (E shifts, H shifts) the next step stores with, per
        8-plane z slab, and the saturation count: one per step, slab and kind
        whose largest stored binary16 magnitude was 65504."""
        nslab = self.dims.nz // 8
        e = (C.c_int * nslab)()
        h = (C.c_int * nslab)()
        ov = C.c_uint64()
        self._chk(_L.lib().wf_storage_info(self._h, e, h, C.byref(ov)))
        return np.array(e[:], np.int32), np.array(h[:], np.int32), int(ov.value)

    @property
    def kernel_launches(self) -> int:
        """Device kernels launched for steps so far (all work classes + tail)."""
        return int(_L.lib().wf_kernel_launches(self._h))

    # -- timing -------------------------------------------------------------
    def stream(self) -> int:
        v = C.c_void_p()
        self._chk(_L.lib().wf_get_stream(self._h, C.byref(v)))
        return int(v.value or 0)

    def set_timing(self, enable: bool):
        self._chk(_L.lib().wf_set_timing(self._h, int(enable)))

    def timing(self):
        """(summed step-kernel milliseconds, launches) since set_timing(True)."""
        ms = C.c_double()
        n = C.c_int64()
        self._chk(_L.lib().wf_get_timing(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    # -- tiling -------------------------------------------------------------
    def tiling(self):
        """(tile_rows, z_chunk, stages) of the fused kernel."""
        t = _L.Tiling()
        self._chk(_L.lib().wf_get_tiling(self._h, C.byref(t)))
        return t.tile_rows, t.z_chunk, t.stages

    def set_tiling(self, tile_rows, z_chunk, stages):
        t = _L.Tiling(tile_rows, z_chunk, stages)
        self._chk(_L.lib().wf_set_tiling(self._h, C.byref(t)))

    def autotune(self, steps: int = 5):
        t = _L.Tiling()
        ms = C.c_float()
        self._chk(_L.lib().wf_autotune(self._h, steps, C.byref(t), C.byref(ms)))
        return (t.tile_rows, t.z_chunk, t.stages), ms.value

    def set_column_tiles(self, enable: bool) -> None:
        """x-CPML slabs as 16-wide column tiles (default) or inside the wide
        tiles; bit-identical results either way."""
        self._chk(_L.lib().wf_set_column_tiles(self._h, int(bool(enable))))

    @property
    def column_tiles(self) -> bool:
        return _L.lib().wf_column_tiles_active(self._h) == 1

    # -- read-back ------------------------------------------------------------
    def fields(self) -> np.ndarray:
        d = self.dims
        out = np.empty((6, d.nz, d.ny, d.nx), np.float32)
        self._chk(_L.lib().wf_get_fields(self._h, _L.ptr(out, _L.f32p)))
        return out

    def set_fields(self, f6):
        a = np.ascontiguousarray(f6, np.float32)
        self._chk(_L.lib().wf_set_fields(self._h, _L.ptr(a, _L.f32p)))

    def download_blocks(self) -> np.ndarray:
        out = np.empty(self.dims.voxel_count() * 6, np.float32)
        self._chk(_L.lib().wf_download_blocks(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def download_blocks_async(self, out) -> None:
        """Starts a FieldBlock download into `out` (a writable buffer of
        6*cells float32, ideally pinned, e.g. a pinned torch tensor's
        numpy view) that overlaps with the following steps; complete once
        sync() returns."""
        a = np.asarray(out)
        if a.dtype != np.float32 or a.size != self.dims.voxel_count() * 6 or not a.flags.c_contiguous:
            raise ValueError("download buffer: contiguous float32, 6 values per voxel")
        self._keep_download = out
        self._chk(_L.lib().wf_download_blocks_async(self._h, a.ctypes.data_as(C.c_void_p)))

    def reserve_download(self) -> None:
        """Allocates the staging buffer of download_blocks_async now."""
        self._chk(_L.lib().wf_reserve_download(self._h))

    def upload_blocks(self, blocks):
        a = np.ascontiguousarray(blocks, np.float32)
        self._chk(_L.lib().wf_upload_blocks(self._h, a.ctypes.data_as(C.c_void_p)))

    def psi(self, which: int) -> np.ndarray:
        d = self.dims
        out = np.empty((d.nz, d.ny, d.nx), np.float32)
        self._chk(_L.lib().wf_get_psi(self._h, which, _L.ptr(out, _L.f32p)))
        return out

    def probe_sums(self, p: int, nfreq: int):
        c = np.zeros(max(nfreq, 1), np.float64)
        s = np.zeros(max(nfreq, 1), np.float64)
        n = C.c_uint64()
        self._chk(_L.lib().wf_probe_sums(self._h, p, _L.ptr(c, _L.f64p), _L.ptr(s, _L.f64p),
                                         C.byref(n)))
        return c[:nfreq], s[:nfreq], int(n.value)

    def probe_trace(self, p: int, n: int) -> np.ndarray:
        out = np.empty(n, np.float32)
        self._chk(_L.lib().wf_probe_trace(self._h, p, _L.ptr(out, _L.f32p), n))
        return out

    def device_field_ptrs(self):
        arr = (C.c_void_p * 6)()
        self._chk(_L.lib().wf_device_fields(self._h, arr))
        return [int(v) for v in arr]

    # -- z-slab copies ---------------------------------------------------------
    def slab_floats(self, nplanes: int) -> int:
        """Floats of the packed state of `nplanes` z planes (wf_slab_floats)."""
        n = int(_L.lib().wf_slab_floats(self._h, nplanes))
        if n < 0:
            raise ValueError(f"bad plane count {nplanes} for nz = {self.dims.nz}")
        return n

    def pack_planes(self, z0: int, nplanes: int, dst_ptr: int, capacity: int) -> None:
        """Enqueues the copy of planes [z0, z0 + nplanes) of the current state
        into the device buffer of `capacity` floats at dst_ptr (wf_slab_pack)."""
        self._chk(_L.lib().wf_slab_pack(self._h, z0, nplanes, C.c_void_p(dst_ptr), capacity))

    def unpack_planes(self, z0: int, nplanes: int, src_ptr: int, capacity: int) -> None:
        """Enqueues the copy of a packed buffer of `capacity` floats into planes
        [z0, z0 + nplanes) of the current state (wf_slab_unpack)."""
        self._chk(_L.lib().wf_slab_unpack(self._h, z0, nplanes, C.c_void_p(src_ptr), capacity))

    def set_graph_steps(self, steps: int) -> None:
        """Steps per captured CUDA graph (even, default 32; wf_set_graph_steps)."""
        self._chk(_L.lib().wf_set_graph_steps(self._h, int(steps)))

    def set_test_stall(self, extra_bytes: int) -> None:
        """Testing aid (wf_set_test_stall): makes every fused step's first TMA
        stage wait run out, so the step reports WF_ERR_TIMEOUT at the next
        sync; 0 turns it off."""
        self._chk(_L.lib().wf_set_test_stall(self._h, int(extra_bytes)))

    # -- checkpoint / resume ----------------------------------------------------
    def checkpoint(self, path) -> None:
        """Saves the complete stepping state (wf_checkpoint_save)."""
        self._chk(_L.lib().wf_checkpoint_save(self._h, os.fsencode(path)))

    def restore(self, path) -> None:
        """Loads a checkpoint into this grid, which must be configured like the
        one that saved it (wf_checkpoint_load); the run then continues bit for
        bit."""
        self._chk(_L.lib().wf_checkpoint_load(self._h, os.fsencode(path)))

    def snapshot_writer(self, path) -> "SnapshotWriter":
        return SnapshotWriter(self, path)


class SnapshotWriter:
    """wave_trajectory.bin writer (src/engine.rs:688-802): each capture()
    appends the current state's FieldBlock bytes; the device-to-host copy and
    the file write overlap the following steps.  Use as a context manager or
    call close()."""

    def __init__(self, grid: DeviceFieldGrid, path):
        self._grid = grid
        self._w = C.c_void_p()
        grid._chk(_L.lib().wf_snapshot_open(grid._h, os.fsencode(path), C.byref(self._w)))
        self.captures = 0

    def capture(self) -> None:
        self._grid._chk(_L.lib().wf_snapshot_capture(self._w))
        self.captures += 1

    def close(self) -> int:
        """Waits for every capture to reach the file; returns the bytes written."""
        if not self._w:
            return 0
        n = C.c_uint64()
        st = _L.lib().wf_snapshot_close(self._w, C.byref(n))
        self._w = C.c_void_p()
        self._grid._chk(st)
        return int(n.value)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class EngineConfig:
    """src/engine.rs:608-615.  With snapshot_every > 0 a snapshot is taken
    after every step whose index is a multiple of it: output_path receives
    them as wave_trajectory.bin through the pinned double-buffered writer,
    and snapshot_sink (if given) receives (step, FieldBlock floats)."""
    num_steps: int
    dt: float
    snapshot_every: int = 0
    snapshot_sink: Optional[Callable[[int, np.ndarray], None]] = None
    output_path: Optional[str] = None


def run(grid: DeviceFieldGrid, sources: Sequence, probes: Sequence, config: EngineConfig,
        quiet: bool = True) -> float:
    """engine::run (src/engine.rs:653-819) on the device.  Returns wall seconds of
    the step loop.  Probe objects receive their sums, count and optional trace."""
    n = config.num_steps
    base_src, base_prb = grid.n_sources, grid.n_probes
    for s in sources:
        grid.add_source_values(s.x, s.y, s.z, s.component, s.values(config.dt, n), s.mode)
    for p in probes:
        c, si = p.tables(config.dt, n)
        grid.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(config.dt),
                              p.record_trace)
    grid.sync()
    t0 = time.perf_counter()
    snap = config.snapshot_sink is not None or config.output_path is not None
    every = max(config.snapshot_every, 1) if snap else 0
    writer = grid.snapshot_writer(config.output_path) if config.output_path is not None else None
    done = 0
    while done < n:
        if every:
            # next step index with step % every == 0 (taken after that step)
            nxt = ((done + every - 1) // every) * every
            chunk = nxt - done + 1 if nxt < n else n - done
        else:
            chunk = n - done
        grid.step(chunk)
        done += chunk
        if every and (done - 1) % every == 0:
            if writer is not None:
                writer.capture()
            if config.snapshot_sink is not None:
                config.snapshot_sink(done - 1, grid.download_blocks())
    if writer is not None:
        writer.close()
    grid.sync()
    wall = time.perf_counter() - t0
    for i, p in enumerate(probes):
        sc, ss, cnt = grid.probe_sums(base_prb + i, len(p.frequencies_hz))
        p.sum_cos, p.sum_sin, p.samples_recorded = sc, ss, cnt
        if p.record_trace:
            p.trace = grid.probe_trace(base_prb + i, n)
    if not quiet:
        d = grid.dims
        print(f"wavefront_b200: {n} steps in {wall:.3f}s ({n / max(wall, 1e-9):.1f} steps/s, "
              f"{d.voxel_count() * n / max(wall, 1e-9) / 1e6:.1f} Mcell/s)")
    return wall


class DeviceBatch:
    """Many independent grids stepped together by one persistent kernel per
    step (wf_batch_*).  grid(i) gives the per-grid handle for setup (scene,
    CPML, sources, probes) and read-back; step() advances every grid."""

    def __init__(self, dims_list: Sequence[GridDims], device: int = 0):
        n = len(dims_list)
        descs = (_L.GridDesc * n)()
        for d, dims in zip(descs, dims_list):
            d.nx, d.ny, d.nz = dims.nx, dims.ny, dims.nz
            d.kernel = _KERNEL["fused"]
            d.device = device
        b = C.c_void_p()
        _L.check(_L.lib().wf_batch_create(n, descs, C.byref(b)))
        self._b = b
        self.grids = [DeviceFieldGrid._member(_L.lib().wf_batch_handle(b, i), dims)
                      for i, dims in enumerate(dims_list)]

    def grid(self, i: int) -> DeviceFieldGrid:
        return self.grids[i]

    def __len__(self):
        return len(self.grids)

    def close(self):
        if getattr(self, "_b", None):
            for g in self.grids:
                g._h = None
            _L.lib().wf_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, n: int = 1):
        _L.check(_L.lib().wf_batch_step(self._b, n))

    def sync(self):
        _L.check(_L.lib().wf_batch_sync(self._b))

    def stream(self) -> int:
        v = C.c_void_p()
        _L.check(_L.lib().wf_batch_get_stream(self._b, C.byref(v)))
        return int(v.value or 0)

    @property
    def kernel_launches(self) -> int:
        return int(_L.lib().wf_batch_kernel_launches(self._b))

    def tiling(self):
        t = _L.Tiling()
        _L.check(_L.lib().wf_batch_get_tiling(self._b, C.byref(t)))
        return t.tile_rows, t.z_chunk, t.stages

    def set_tiling(self, tile_rows, z_chunk, stages):
        t = _L.Tiling(tile_rows, z_chunk, stages)
        _L.check(_L.lib().wf_batch_set_tiling(self._b, C.byref(t)))

    def autotune(self, steps: int = 3):
        t = _L.Tiling()
        ms = C.c_float()
        _L.check(_L.lib().wf_batch_autotune(self._b, steps, C.byref(t), C.byref(ms)))
        return (t.tile_rows, t.z_chunk, t.stages), ms.value
