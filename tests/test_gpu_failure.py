"""GPU: failure paths, exercised without a fault.

wf_set_test_stall makes each fused step CTA expect more bytes on its first
TMA stage than its copies deliver: the copies land, the stage's phase never
completes, and the kernel's bounded wait (about one second) runs out. The
step must then report WF_ERR_TIMEOUT at the next sync, within a bounded
time, and the GPU context must stay usable: a fresh handle on the same device
steps and matches the oracle bit for bit.

The host-side failures: a grid larger than the device (its cudaMalloc
fails, which is not a sticky error) must return WF_ERR_OOM with nothing left
allocated, and a snapshot file whose writes fail (/dev/full) must surface as
WF_ERR_IO from the writer without stalling it.
"""
import os
import time

import numpy as np
import pytest

import wavefront_b200 as wf
from oracle import oracle as O
from wavefront_b200 import _lib as L
from wavefront_b200 import configs

pytestmark = pytest.mark.gpu
NT = min(os.cpu_count() or 1, 32)


def _configure(g, sc, steps):
    for s in sc.sources:
        g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, steps), s.mode)


def test_stalled_stage_reports_timeout_and_context_survives():
    sc = configs.plain_cube_64(steps=4)
    g = configs.device_grid(sc, kernel="fused")
    try:
        _configure(g, sc, 4)
        g.step(1)
        g.sync()  # a normal step first
        g.set_test_stall(16)
        t0 = time.perf_counter()
        g.step(1)
        with pytest.raises(wf.WfError) as e:
            g.sync()
        waited = time.perf_counter() - t0
        assert e.value.status == L.WF_ERR_TIMEOUT
        assert 0.3 < waited < 60.0, waited  # the bound ran out; nothing hung
    finally:
        g.close()

    # the context is intact: a new handle steps and matches the oracle
    h = configs.device_grid(sc, kernel="fused")
    try:
        _configure(h, sc, 4)
        h.step(4)
        h.sync()
        sim = O.sim_from_scenario(sc, steps=4)
        sim.step(4, nthreads=NT)
        got, want = h.fields(), sim.fields()
        assert np.array_equal(got, want)  # == treats +0 and -0 as equal
    finally:
        h.close()


def test_stall_argument_checks():
    sc = configs.plain_cube_64(steps=2)
    g = configs.device_grid(sc, kernel="fused")
    try:
        for bad in (-1, 65537):
            with pytest.raises(wf.WfError) as e:
                g.set_test_stall(bad)
            assert e.value.status == L.WF_ERR_ARG
        g.set_test_stall(0)  # off: a normal step
        _configure(g, sc, 2)
        g.step(2)
        g.sync()
    finally:
        g.close()


def test_device_allocation_failure_is_reported_and_context_survives():
    # 4096^3 cells: 1.6 TB per FP32 state buffer, far beyond any GPU
    with pytest.raises(wf.WfError) as e:
        wf.DeviceFieldGrid(wf.GridDims(4096, 4096, 4096))
    assert e.value.status == L.WF_ERR_OOM
    sc = configs.plain_cube_64(steps=4)
    g = configs.device_grid(sc)
    try:
        _configure(g, sc, 4)
        g.step(4)
        g.sync()
        assert np.abs(g.fields()).max() > 0
    finally:
        g.close()


def test_snapshot_write_failure_surfaces_as_io_error():
    if not os.path.exists("/dev/full"):
        pytest.skip("no /dev/full on this host")
    sc = configs.plain_cube_64(steps=8)
    g = configs.device_grid(sc)
    statuses = []
    try:
        _configure(g, sc, 8)
        w = g.snapshot_writer("/dev/full")
        try:
            for _ in range(3):
                g.step(2)
                w.capture()
        except wf.WfError as err:  # a later capture may see the first failure
            statuses.append(err.status)
        with pytest.raises(wf.WfError) as e:
            w.close()
        statuses.append(e.value.status)
        assert statuses and all(st == L.WF_ERR_IO for st in statuses)
        g.step(1)  # the handle keeps working
        g.sync()
    finally:
        g.close()


def test_device_memory_cache_reuses_and_releases():
    """A destroyed handle's device blocks go to the library's cache and the
    next handle of the same shape takes them back; the cache returns its
    blocks to CUDA on request, and a handle built from reused (dirty)
    blocks still starts from zero fields."""
    lib = L.lib()
    dims = wf.GridDims(64, 64, 64)
    lib.wf_release_cached_memory(-1)
    assert lib.wf_cached_bytes(0) == 0
    g = wf.DeviceFieldGrid(dims)
    g.set_fields(np.ones((6, 64, 64, 64), np.float32))
    g.close()
    cached = lib.wf_cached_bytes(0)
    assert cached >= 2 * 6 * 4 * 64 ** 3  # both state buffers at least
    g = wf.DeviceFieldGrid(dims)
    try:
        assert lib.wf_cached_bytes(0) < cached
        assert not np.any(g.fields())
    finally:
        g.close()
    assert lib.wf_release_cached_memory(-1) == L.WF_OK
    assert lib.wf_cached_bytes(0) == 0
