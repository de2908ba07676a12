"""GPU: the device timeout path, exercised without a fault.

wf_set_test_stall makes each fused step CTA expect more bytes on its first
TMA stage than its copies deliver: the copies land, the stage's phase never
completes, and the kernel's bounded wait (about one second) runs out. The
step must then report WF_ERR_TIMEOUT at the next sync, within a bounded
time, and the GPU context must stay usable: a fresh handle on the same device
steps and matches the oracle bit for bit.
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
