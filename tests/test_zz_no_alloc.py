"""The allocation-free entry point, wf_step_fields_noalloc.

It exists for callers that cannot call cudaMalloc (device memory owned by
their own pool allocator, or a loop where an allocation is not allowed): they
pass their own device field buffer and material ids, and the library steps
them in place using only a static device array for the next state.

This file is collected last so that a run stopping at its first failure has
already run every other test.  The test builds its device buffers with torch
(the caller's allocations, not the entry point's) and checks the entry point
against the handle-based wf_step, bit for bit as the other parity tests do,
over two calls in a row.
"""
import ctypes as C

import numpy as np
import pytest

import wavefront_b200 as wf
from wavefront_b200 import _lib as L
from wavefront_b200 import configs

pytestmark = pytest.mark.gpu


def _scene():
    dims = wf.GridDims(48, 32, 40)
    dx = 1e-3
    dt = configs.courant_dt(dx)
    grid = wf.MaterialGrid(dims)
    table = wf.MaterialTable.vacuum_filled(dt, dx)
    wf.Scene.parse("sphere 4.0 1.0 0.01 20 16 20 9\nbox 2.0 1.5 0.0 30 4 4 44 28 36\n").voxelize(
        grid, table, dt, dx)
    rng = np.random.default_rng(7)
    init = rng.standard_normal((6, dims.nz, dims.ny, dims.nx)).astype(np.float32)
    return dims, grid, table, init


def _noalloc(dev_fields, dev_ids, table, dims, nsteps, boundary=(0, 0, 0), stream=None):
    b = (C.c_int32 * 3)(*boundary)
    q = np.ascontiguousarray(table.q16, np.int32)
    return L.lib().wf_step_fields_noalloc(C.c_void_p(dev_fields.data_ptr()),
                                          C.c_void_p(dev_ids.data_ptr()), L.ptr(q, L.i32p),
                                          dims.nx, dims.ny, dims.nz, b, 0, nsteps,
                                          C.c_void_p(stream))


@pytest.mark.parametrize("boundary", [(0, 0, 0), (0, 1, 1)])
def test_noalloc_matches_handle_step_on_two_calls(boundary):
    import torch
    dims, grid, table, init = _scene()
    names = ("zero", "periodic")
    h = wf.DeviceFieldGrid(dims, boundary=tuple(names[v] for v in boundary))
    try:
        h.set_materials(grid, table)
        h.set_fields(init)
        dev = torch.from_numpy(init.copy()).cuda()
        ids = torch.from_numpy(grid.ids.copy()).cuda()
        torch.cuda.synchronize()
        for nsteps in (7, 4):  # an odd count (result copied home), then an even one
            h.step(nsteps)
            h.sync()
            st = _noalloc(dev, ids, table, dims, nsteps, boundary)
            assert st == L.WF_OK, L.lib().wf_noalloc_last_error()
            torch.cuda.synchronize()
            want = h.fields()
            got = dev.cpu().numpy()
            assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} cells differ"
    finally:
        h.close()


def test_noalloc_rejects_grids_above_its_limit():
    import torch
    dims = wf.GridDims(72, 64, 64)  # 294912 cells > 262144
    table = wf.MaterialTable.vacuum_filled(1e-12, 1e-3)
    dev = torch.zeros(6 * dims.voxel_count(), device="cuda")
    ids = torch.zeros(dims.voxel_count(), dtype=torch.uint8, device="cuda")
    st = _noalloc(dev, ids, table, dims, 1)
    assert st == L.WF_ERR_ARG
    assert b"exceeds the allocation-free limit of 262144 cells" in L.lib().wf_noalloc_last_error()
