"""CPU: the reference's kernel-level known answers, on the oracle.

src/fdtd.rs:537-628 pins two facts about the update kernels:
- a spatially uniform field has zero curl, so with da = 1 the H update and
  with ca = 1 the E update leave it unchanged;
- with identity CPML coefficients (b 1, a 0, 1/kappa 1) and zero psi the
  CPML kernel equals the plain kernel.
Here they hold on whole grids: cells whose neighbours are all inside the
domain keep a uniform field exactly through a step, and a run with an
identity CPML shell equals the run without CPML in every field.
test_gpu_known_answers.py checks the same on the device.
"""
import numpy as np

from wavefront_b200 import configs

N = 32
ONE_Q16 = 1 << 16  # Q16.16 of 1.0


def uniform_fields(n=N):
    f = np.empty((6, n, n, n), np.float32)
    for c in range(6):
        f[c] = float(c + 1)
    return f


def interior(a):
    return a[:, 1:-1, 1:-1, 1:-1]


def test_uniform_field_has_zero_curl(oracle):
    table = np.full((256, 4), ONE_Q16, np.int32)  # ca = cb = da = db = 1
    sim = oracle.Sim(N, N, N, None, table)
    f0 = uniform_fields()
    sim.set_fields(f0)
    sim.step(1)
    got = sim.fields()
    assert np.array_equal(interior(got).view(np.uint32), interior(f0).view(np.uint32))
    assert not np.array_equal(got, f0)  # the cells next to the zero outside do change


def test_identity_cpml_equals_plain_kernel(oracle):
    sc = configs.plain_cube_64(steps=60, pml_cells=0)
    plain = oracle.sim_from_scenario(sc)
    shell = oracle.sim_from_scenario(sc)
    n = sc.dims.nx
    ident = (np.ones(n, np.float32), np.zeros(n, np.float32), np.ones(n, np.float32))
    shell.set_pml([ident, ident, ident], [2, 2, 2])
    plain.step(60)
    shell.step(60)
    a, b = plain.fields(), shell.fields()
    assert np.abs(a).max() > 0
    assert np.array_equal(a, b)  # +0 and -0 compare equal
    for w in range(12):
        assert not shell.psi(w).any()  # identity psi stays zero
