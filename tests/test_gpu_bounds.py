"""GPU: the bounds-checked device build (libwavefront_gpu_checked.so).

compute-sanitizer is not available on the GPU pool, so the library has a
debugging variant compiled with -DWF_BOUNDS_CHECK: every global access of
the step kernels (fused and split: field and psi loads and stores) and of
the step tail (source and probe cells) tests its index against its buffer
and, when it is out of range, latches a device error flag (reported by
wf_sync) and skips the access.  Here the small-grid parity cases run under
that build in a fresh process (the library is chosen when it is loaded):
results must equal the oracle's bit for bit with no flag raised.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r'''
import os, sys
import numpy as np
sys.path.insert(0, os.environ["WF_ROOT"])
import wavefront_b200 as wf
from wavefront_b200 import _lib as L, configs
from oracle import oracle as O
assert L.LIB_PATH.endswith("libwavefront_gpu_checked.so")

def run(sc, steps, prec="f32", arith="exact", **kw):
    g = configs.device_grid(sc, precision=prec, arith=arith, **{k: v for k, v in kw.items() if k == "kernel"})
    if "columns" in kw:
        g.set_column_tiles(kw["columns"])
    for s in sc.sources:
        g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, steps), s.mode)
    for p in sc.probes:
        c, si = p.tables(sc.dt, steps)
        g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(sc.dt))
    g.step(steps)
    g.sync()  # raises on a latched device flag
    f, sums = g.fields(), [g.probe_sums(i, len(p.frequencies_hz)) for i, p in enumerate(sc.probes)]
    psi = [g.psi(w) for w in range(12)] if sc.pml is not None else []
    g.close()
    return f, sums, psi

def check(sc, steps, storage="f32", arith="exact", **kw):
    sim = O.sim_from_scenario(sc, steps=steps, storage=storage, arith=arith)
    sim.step(steps, os.cpu_count() or 1)
    f, sums, psi = run(sc, steps, prec=storage, arith=arith, **kw)
    assert np.array_equal(f, sim.fields()), (sc.name, kw, int(np.count_nonzero(f != sim.fields())))
    for i, p in enumerate(sc.probes):
        oc, os_, on = sim.probe_sums(i, len(p.frequencies_hz))
        assert np.array_equal(sums[i][0], oc) and sums[i][2] == on, (sc.name, i)
    for w, a in enumerate(psi):
        assert np.array_equal(a, sim.psi(w)), (sc.name, kw, w)
    sim.close()

cube = configs.plain_cube_64(steps=120)
check(cube, 120, kernel="fused", columns=True)
check(cube, 120, kernel="fused", columns=False)
check(cube, 120, kernel="split")
check(cube, 60, arith="fma", kernel="fused")
check(configs.plain_cube_64(steps=80, exact_pml=True), 80, kernel="fused")
check(configs.two_spheres(n=64, steps=80), 80, storage="f16", kernel="fused")
check(configs.two_spheres(n=96, steps=60), 60, kernel="fused")
print("BOUNDS_OK")
'''


def test_bounds_checked_build_matches_oracle_without_flags():
    lib = os.path.join(ROOT, "wavefront_b200", "lib", "libwavefront_gpu_checked.so")
    assert os.path.exists(lib), "build the bounds-checked variant (wavefront_b200/build.py)"
    env = dict(os.environ, WF_BOUNDS_CHECK="1", WF_ROOT=ROOT)
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0 and "BOUNDS_OK" in r.stdout, (r.stdout[-2000:], r.stderr[-3000:])
