"""The allocation-free entry point, wf_step_fields_noalloc.

It exists for callers that cannot call cudaMalloc (device memory owned by
their own pool allocator, or a loop where an allocation is not allowed): they
pass their own device field buffer and material ids, and the library steps
them in place using only a static device array for the next state.

This file is collected last so that a run stopping at its first failure has
already run every other test.  The test builds its device buffers with torch
(the caller's allocations, not the entry point's) and checks the entry point
against the handle-based wf_step, bit for bit as the other parity tests do,
over two calls in a row, in both arithmetic modes and on a caller's own
stream; and, on its own, against the CPU oracle (so the periodic case meets
the reference's arithmetic directly, not only the handle's split kernels).
Buffers that are not device memory of the current device, and calls on a
stream that is capturing a graph, are refused before anything is launched.
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


def _addr(a):
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


def _noalloc(dev_fields, dev_ids, table, dims, nsteps, boundary=(0, 0, 0), stream=None,
             arith=0):
    b = (C.c_int32 * 3)(*boundary)
    q = np.ascontiguousarray(table.q16, np.int32)
    return L.lib().wf_step_fields_noalloc(C.c_void_p(_addr(dev_fields)),
                                          C.c_void_p(_addr(dev_ids)), L.ptr(q, L.i32p),
                                          dims.nx, dims.ny, dims.nz, b, arith, nsteps,
                                          C.c_void_p(stream))


@pytest.mark.parametrize("boundary,arith,own_stream", [
    ((0, 0, 0), "exact", False), ((0, 1, 1), "exact", False),
    ((0, 0, 0), "fma", True), ((0, 1, 1), "fma", False)])
def test_noalloc_matches_handle_step_on_two_calls(boundary, arith, own_stream):
    import torch
    dims, grid, table, init = _scene()
    names = ("zero", "periodic")
    h = wf.DeviceFieldGrid(dims, boundary=tuple(names[v] for v in boundary), arith=arith)
    try:
        h.set_materials(grid, table)
        h.set_fields(init)
        dev = torch.from_numpy(init.copy()).cuda()
        ids = torch.from_numpy(grid.ids.copy()).cuda()
        torch.cuda.synchronize()
        stream = torch.cuda.Stream() if own_stream else None
        for nsteps in (7, 4):  # an odd count (result copied home), then an even one
            h.step(nsteps)
            h.sync()
            st = _noalloc(dev, ids, table, dims, nsteps, boundary,
                          stream.cuda_stream if stream is not None else None,
                          1 if arith == "fma" else 0)  # WF_ARITH_FMA / WF_ARITH_EXACT
            assert st == L.WF_OK, L.lib().wf_noalloc_last_error()
            if stream is not None:
                stream.synchronize()
            torch.cuda.synchronize()
            want = h.fields()
            got = dev.cpu().numpy()
            assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} cells differ"
    finally:
        h.close()


@pytest.mark.parametrize("boundary", [(0, 0, 0), (1, 0, 1)])
def test_noalloc_matches_the_oracle(boundary):
    """Against the CPU oracle directly (exact arithmetic, bit for bit, +0 and
    -0 equal), over two calls in a row."""
    import torch
    from oracle import oracle as O
    dims, grid, table, init = _scene()
    sim = O.Sim(dims.nx, dims.ny, dims.nz, grid.ids, table.q16, boundary)
    try:
        sim.set_fields(init)
        dev = torch.from_numpy(init.copy()).cuda()
        ids = torch.from_numpy(grid.ids.copy()).cuda()
        torch.cuda.synchronize()
        for nsteps in (5, 6):
            st = _noalloc(dev, ids, table, dims, nsteps, boundary)
            assert st == L.WF_OK, L.lib().wf_noalloc_last_error()
            torch.cuda.synchronize()
            sim.step(nsteps, 4)
            got, want = dev.cpu().numpy(), sim.fields()
            assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} cells differ"
    finally:
        sim.close()


def test_noalloc_refuses_host_buffers_without_launching():
    """A host pointer for the fields or the ids is refused with WF_ERR_ARG
    before any launch: the caller's device fields stay as they were."""
    import torch
    dims, grid, table, init = _scene()
    dev = torch.from_numpy(init.copy()).cuda()
    ids = torch.from_numpy(grid.ids.copy()).cuda()
    host_fields = init.copy()
    host_ids = grid.ids.copy()
    torch.cuda.synchronize()
    st = _noalloc(host_fields, ids, table, dims, 3)
    assert st == L.WF_ERR_ARG and b"fields6" in L.lib().wf_noalloc_last_error()
    assert np.array_equal(host_fields, init)
    st = _noalloc(dev, host_ids, table, dims, 3)
    assert st == L.WF_ERR_ARG and b"ids" in L.lib().wf_noalloc_last_error()
    pinned = torch.from_numpy(init.copy()).pin_memory()  # host memory the GPU can reach
    st = _noalloc(pinned, ids, table, dims, 3)
    assert st == L.WF_ERR_ARG and b"host memory" in L.lib().wf_noalloc_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), init)
    assert np.array_equal(pinned.numpy(), init)


def test_noalloc_refuses_a_capturing_stream():
    """Its coefficient upload reads a host array that lives only for the
    call, so a call on a stream that is capturing a graph is refused."""
    import torch
    dims, grid, table, init = _scene()
    dev = torch.from_numpy(init.copy()).cuda()
    ids = torch.from_numpy(grid.ids.copy()).cuda()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st = _noalloc(dev, ids, table, dims, 2, stream=s.cuda_stream)
        finally:
            g.capture_end()
    assert st == L.WF_ERR_UNSUPPORTED
    assert b"capturing" in L.lib().wf_noalloc_last_error()
    del g
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), init)


def test_noalloc_rejects_grids_above_its_limit():
    import torch
    dims = wf.GridDims(72, 64, 64)  # 294912 cells > 262144
    table = wf.MaterialTable.vacuum_filled(1e-12, 1e-3)
    dev = torch.zeros(6 * dims.voxel_count(), device="cuda")
    ids = torch.zeros(dims.voxel_count(), dtype=torch.uint8, device="cuda")
    st = _noalloc(dev, ids, table, dims, 1)
    assert st == L.WF_ERR_ARG
    assert b"exceeds the allocation-free limit of 262144 cells" in L.lib().wf_noalloc_last_error()
