"""GPU: the reference's kernel-level known answers (src/fdtd.rs:537-628) on
the device, through the C ABI, for the fused and the split kernels: a
uniform field keeps its value wherever all neighbours are inside the domain
(zero curl, unit coefficients), and an identity CPML on every axis (b 1, a 0,
1/kappa 1) gives the plain kernel's fields with psi left at zero.
"""
import numpy as np
import pytest

import wavefront_b200 as wf
from wavefront_b200 import configs

pytestmark = pytest.mark.gpu
N = 32


def _uniform(n=N):
    f = np.empty((6, n, n, n), np.float32)
    for c in range(6):
        f[c] = float(c + 1)
    return f


@pytest.mark.parametrize("kernel", ["fused", "split"])
def test_uniform_field_has_zero_curl(kernel):
    dims = wf.GridDims(N, N, N)
    g = wf.DeviceFieldGrid(dims, kernel=kernel)
    try:
        g.set_materials(wf.MaterialGrid(dims), wf.MaterialTable(np.full((256, 4), 1 << 16)))
        f0 = _uniform()
        g.set_fields(f0)
        g.step(1)
        got = g.fields()
        inner = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
        assert np.array_equal(got[inner].view(np.uint32), f0[inner].view(np.uint32))
        assert not np.array_equal(got, f0)
    finally:
        g.close()


@pytest.mark.parametrize("kernel", ["fused", "split"])
def test_identity_cpml_equals_plain_kernel(kernel):
    steps = 60
    sc = configs.plain_cube_64(steps=steps, pml_cells=0)
    n = sc.dims.nx
    grids = []
    try:
        for identity in (False, True):
            g = configs.device_grid(sc, kernel=kernel)
            grids.append(g)
            if identity:
                for ax in range(3):
                    g.set_pml_axis(ax, 16, np.ones(n), np.zeros(n), np.ones(n))
            for s in sc.sources:
                g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, steps), s.mode)
            g.step(steps)
            g.sync()
        a, b = grids[0].fields(), grids[1].fields()
        assert np.abs(a).max() > 0
        assert np.array_equal(a, b)  # +0 and -0 compare equal
        for w in range(12):
            assert not grids[1].psi(w).any()
    finally:
        for g in grids:
            g.close()
