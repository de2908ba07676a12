"""GPU parity: the CUDA library against the CPU oracle, through the C ABI.

Bar: bit-exact for the exact-arithmetic build (all six fields, every CPML psi
array, probe sums and counts), with +0 and -0 treated as equal (the CPML
identity correction can flip the sign of a zero, src/fdtd.rs:152-163, and a
signed zero never changes a nonzero value).  The FMA build is held to 1e-6
relative L2 per field.
"""
import csv
import os

import numpy as np
import pytest

import wavefront_b200 as wf
from wavefront_b200 import configs, studies

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
NT = min(os.cpu_count() or 1, 32)


def _assert_fields_equal(got, want, what=""):
    assert got.shape == want.shape
    bad = got != want  # == treats +0 and -0 as equal
    if bad.any():
        idx = np.argwhere(bad)[:5]
        raise AssertionError(f"{what}: {bad.sum()} cells differ, first {idx.tolist()}, "
                             f"got {got[bad][:5]} want {want[bad][:5]}")


def _run_device(sc, steps=None, **kw):
    steps = sc.steps if steps is None else steps
    g = configs.device_grid(sc, **kw)
    for s in sc.sources:
        g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, steps), s.mode)
    for p in sc.probes:
        c, si = p.tables(sc.dt, steps)
        g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(sc.dt), p.record_trace)
    g.step(steps)
    g.sync()
    return g


def _compare(g, sim, sc, psi=True):
    _assert_fields_equal(g.fields(), sim.fields(), "fields")
    for i, p in enumerate(sc.probes):
        nf = len(p.frequencies_hz)
        gc, gs, gn = g.probe_sums(i, nf)
        oc, os_, on = sim.probe_sums(i, nf)
        assert gn == on
        assert np.array_equal(gc, oc) and np.array_equal(gs, os_), (i, gc, oc)
    if psi and sc.pml is not None:
        for w in range(12):
            _assert_fields_equal(g.psi(w), sim.psi(w), wf.PSI_NAMES[w])


@pytest.fixture(scope="module")
def cube64(oracle):
    sc = configs.plain_cube_64()
    sim = oracle.sim_from_scenario(sc)
    sim.step(sc.steps, NT)
    return sc, sim


@pytest.mark.parametrize("kernel,columns", [("fused", True), ("fused", False), ("split", None)])
def test_plain_cube_64_bit_exact(cube64, kernel, columns):
    """64^3 vacuum, CPML 10 -> 16 cells, Ricker at the centre, 500 steps; the
    fused step with the x-CPML slabs as 16-wide column tiles (the default
    here) and inside the wide tiles."""
    sc, sim = cube64
    g = configs.device_grid(sc, kernel=kernel)
    try:
        if columns is not None:
            g.set_column_tiles(columns)
            assert g.column_tiles == columns
        for s in sc.sources:
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, sc.steps))
        for p in sc.probes:
            c, si = p.tables(sc.dt, sc.steps)
            g.add_probe_tables(p.x, p.y, p.z, p.component, c, si)
        g.step(sc.steps)
        g.sync()
        _compare(g, sim, sc)
        assert g.steps_done == 500
    finally:
        g.close()


@pytest.mark.parametrize("tiling", [(4, 16, 3), (8, 64, 4), (8, 7, 3), (16, 1000, 3),
                                    (16, 5, 3), (4, 32, 4), (4, 1000, 3), (8, 1, 4)])
def test_fused_tilings_bit_identical(cube64, tiling):
    """Tiling is a scheduling detail (the GPU analogue of the reference's 1-slab
    vs 4-slab test, src/engine.rs:1008-1099): every tiling gives the oracle's bits."""
    sc, sim = cube64
    g = configs.device_grid(sc, kernel="fused")
    try:
        g.set_tiling(*tiling)
        for s in sc.sources:
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, sc.steps))
        for p in sc.probes:
            c, si = p.tables(sc.dt, sc.steps)
            g.add_probe_tables(p.x, p.y, p.z, p.component, c, si)
        g.step(sc.steps)
        g.sync()
        _compare(g, sim, sc)
    finally:
        g.close()


def _rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_fma_build_within_1e6_relative_l2(oracle):
    """The FMA build on the two-sphere scene (128^3, 200 steps): E fields within
    1e-6 relative L2 of the exact build, and every component whose norm is not
    negligible within 3x the exact build's own distance from the FP64 oracle
    (FMA contraction moves results by about one FP32 rounding per operation;
    components that decay towards zero, or stay near zero like Hz for an Ez
    source, have ill-conditioned relative norms)."""
    sc = configs.two_spheres(n=128, steps=200)
    out = {}
    for arith in ("exact", "fma"):
        g = _run_device(sc, kernel="fused", arith=arith)
        out[arith] = g.fields()
        g.close()
    sim = oracle.sim_from_scenario(sc, dtype="f64")
    sim.step(sc.steps, NT)
    f64 = sim.fields()
    sim.close()
    for c in range(3):
        assert _rel_l2(out["fma"][c], out["exact"][c]) <= 1e-6, c
    top = max(np.linalg.norm(f64[c].ravel()) for c in range(6))
    for c in range(6):
        if np.linalg.norm(f64[c].ravel()) < 1e-6 * top:
            continue
        ref = _rel_l2(out["exact"][c].astype(np.float64), f64[c])
        assert _rel_l2(out["fma"][c], out["exact"][c]) <= 3 * ref + 1e-7, c


@pytest.mark.parametrize("kernel", ["fused", "split"])
@pytest.mark.parametrize("scene", ["cube64", "two_spheres64"])
def test_fma_build_equals_fma_restatement(oracle, kernel, scene):
    """The FMA build computes exactly the fused forms it states:
    psi' = fma(b, psi, a*raw), d = fma(raw, 1/kappa, psi'),
    H' = fma(da, h, -(db*curl)), E' = fma(ca, e, cb*curl): bit for bit against
    the oracle's restatement of those forms (fields, all psi, probe sums)."""
    sc = (configs.plain_cube_64(steps=150) if scene == "cube64"
          else configs.two_spheres(n=64, steps=150))
    sim = oracle.sim_from_scenario(sc, arith="fma")
    sim.step(sc.steps, NT)
    g = _run_device(sc, kernel=kernel, arith="fma")
    try:
        _compare(g, sim, sc)
    finally:
        g.close()
        sim.close()


def test_exact_thin_cpml_10_cells(oracle):
    """Per-cell CPML of 10 cells (not rounded to blocks)."""
    sc = configs.plain_cube_64(steps=300, exact_pml=True)
    assert sc.pml.thickness_voxels == (10, 10, 10)
    sim = oracle.sim_from_scenario(sc)
    sim.step(sc.steps, NT)
    for kernel in ("fused", "split"):
        g = _run_device(sc, kernel=kernel)
        try:
            _compare(g, sim, sc)
        finally:
            g.close()


@pytest.mark.parametrize("shape", [(8, 8, 8), (8, 136, 16), (264, 16, 16), (16, 16, 200)])
def test_extreme_grid_shapes(oracle, shape):
    """The smallest grid, a tile with 2 of its 32 lanes inside the domain, a
    last x tile 8 cells wide, and a long thin z axis: fused under two tilings
    and split, bit for bit (fields, psi, probe sums).  The CPML thickness
    follows the reference's rounding, so grids one block thick get none."""
    nx, ny, nz = shape
    dims = wf.GridDims(nx, ny, nz)
    dx = 1e-3
    dt = configs.courant_dt(dx)
    grid = wf.MaterialGrid(dims)
    table = wf.MaterialTable.vacuum_filled(dt, dx)
    wf.Scene.parse(f"sphere 3.0 1.0 0.01 {nx / 2} {ny / 2} {nz / 2} {min(nx, ny, nz) / 3}\n").voxelize(
        grid, table, dt, dx)
    pml = wf.PmlContext.build(dims, wf.PmlConfig(thickness=8), dt, dx)
    f = float(np.float32(3e8 / (12 * dx)))
    srcs = [wf.Source(nx // 2, ny // 2, nz // 2, wf.FieldComponent.Ez, 1.0,
                      wf.default_waveform("ricker", f)),
            wf.Source(nx - 1, ny - 1, nz - 1, wf.FieldComponent.Ex, 0.5,
                      wf.default_waveform("gaussian", f))]
    prbs = [wf.Probe(nx // 4, ny // 3, nz // 2, wf.ProbeComponent(c), [f], 0.0) for c in (2, 4)]
    sc = configs.Scenario("extreme", dims, dx, dt, grid, table, pml, srcs, prbs, 60)
    sim = oracle.sim_from_scenario(sc)
    sim.step(sc.steps, NT)
    for kernel, tiling in (("fused", (4, 12, 3)), ("fused", (16, 5, 3)), ("split", None)):
        g = configs.device_grid(sc, kernel=kernel)
        try:
            if tiling:
                g.set_tiling(*tiling)
            for s_ in srcs:
                g.add_source_values(s_.x, s_.y, s_.z, s_.component, s_.values(dt, sc.steps))
            for p in prbs:
                c, si = p.tables(dt, sc.steps)
                g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(dt))
            g.step(sc.steps)
            g.sync()
            _compare(g, sim, sc)
        finally:
            g.close()
    sim.close()


def test_ragged_grid_materials_h_probes_and_late_start(oracle):
    """nx not a multiple of the 128-cell tile, ny not a multiple of the tile
    rows (nor of the 32-row column tiles), a thin z axis, a lossy scene,
    several sources and H-component probes with a recording start time;
    fused with and without x-CPML column tiles."""
    dims = wf.GridDims(136, 40, 24)
    dx = 1e-3
    dt = configs.courant_dt(dx)
    grid = wf.MaterialGrid(dims)
    table = wf.MaterialTable.vacuum_filled(dt, dx)
    wf.Scene.parse("sphere 4.0 1.0 0.02 60 20 12 9\nbox 2.5 1.5 0.0 100 3 2 130 30 20\n"
                   "sphere 1.7 1.0 0.0 7 35 20 6\n").voxelize(grid, table, dt, dx)
    pml = wf.PmlContext.build(dims, wf.PmlConfig(thickness=8), dt, dx)
    f = float(np.float32(3e8 / (15 * dx)))
    srcs = [wf.Source(70, 21, 11, wf.FieldComponent.Ez, 1.0, wf.default_waveform("ricker", f)),
            wf.Source(70, 21, 11, wf.FieldComponent.Ez, 0.5, wf.default_waveform("gaussian", f)),
            wf.Source(3, 38, 1, wf.FieldComponent.Ex, 2.0, wf.default_waveform("sinusoid", f)),
            wf.Source(135, 0, 23, wf.FieldComponent.Ey, 1.0, wf.default_waveform("ricker", f))]
    prbs = [wf.Probe(90, 20, 12, wf.ProbeComponent(c), [f, 2 * f], 40 * dt) for c in range(6)]
    sc = configs.Scenario("ragged", dims, dx, dt, grid, table, pml, srcs, prbs, 200)
    sim = oracle.sim_from_scenario(sc)
    sim.step(sc.steps, NT)
    for kernel, tiling, cols in (("fused", (8, 64, 3), True), ("fused", (16, 10, 3), True),
                                 ("fused", (4, 10, 4), True), ("fused", (8, 24, 4), True),
                                 ("fused", (4, 10, 3), False), ("split", None, None)):
        g = configs.device_grid(sc, kernel=kernel)
        try:
            if tiling:
                g.set_tiling(*tiling)
            if cols is not None:
                g.set_column_tiles(cols)
                assert g.column_tiles == cols  # 8-cell x CPML, nx 136: columns apply
            for s in srcs:
                g.add_source_values(s.x, s.y, s.z, s.component, s.values(dt, sc.steps))
            for p in prbs:
                c, si = p.tables(dt, sc.steps)
                g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(dt))
            g.step(sc.steps)
            g.sync()
            _compare(g, sim, sc)
        finally:
            g.close()


def test_two_spheres_128_and_snapshot_bytes(oracle):
    """The headline scene scaled to 128^3 (CPML 16, Gaussian source, 8 probes),
    plus the snapshot byte format (FieldBlock order, src/engine.rs:622-640)."""
    sc = configs.two_spheres(n=128, steps=120)
    sim = oracle.sim_from_scenario(sc)
    sim.step(sc.steps, NT)
    g = _run_device(sc, kernel="fused")
    try:
        _compare(g, sim, sc)
        blk = g.download_blocks()
        assert np.array_equal(blk, sim.blocks())
        # upload the blocks back and continue: identical to continuing directly
        g2 = configs.device_grid(sc, kernel="fused")
        try:
            g2.upload_blocks(blk)
            _assert_fields_equal(g2.fields(), g.fields(), "upload_blocks round trip")
        finally:
            g2.close()
    finally:
        g.close()


def test_full_size_two_spheres_512_matches_oracle(oracle):
    """The headline workload as configured (512^3, 16-cell CPML, Gaussian Ez
    at (256,256,64), 8 Ez probes at z=448, all 1000 steps) against the
    multithreaded oracle, bit for bit: all six fields, the 12 CPML psi arrays
    and every probe's sums and count.  By step 1000 the pulse has crossed
    both sphere interfaces, entered every CPML slab and reached the probe
    line, which the test checks, so none of what is compared is trivially
    zero."""
    sc = configs.two_spheres(n=512, steps=1000)
    sim = oracle.sim_from_scenario(sc)
    sim.step(sc.steps, NT)
    g = _run_device(sc, kernel="fused")
    try:
        _assert_fields_equal(g.fields(), sim.fields(), "fields")
        for i, p in enumerate(sc.probes):
            gc, gs, gn = g.probe_sums(i, 1)
            oc, os_, on = sim.probe_sums(i, 1)
            assert gn == on == sc.steps
            assert np.array_equal(gc, oc) and np.array_equal(gs, os_), (i, gc, oc)
            assert abs(gc[0]) + abs(gs[0]) > 0.0, f"probe {i} at z=448 saw no signal"
        n, t = 512, sc.pml.thickness_voxels[0]
        for w, name in enumerate(wf.PSI_NAMES):
            got = g.psi(w)
            _assert_fields_equal(got, sim.psi(w), name)
            ax = "xyz".index(name[-1])  # psi_*_d{x,y,z}: the axis its slab lies on
            for lo in (0, n - t):
                sl = [slice(None)] * 3
                sl[2 - ax] = slice(lo, lo + t)
                assert np.count_nonzero(got[tuple(sl)]), f"{name}: slab at {lo} stayed zero"
            del got
    finally:
        g.close()
        sim.close()


def test_full_size_properties_linearity_and_paths_agree():
    """512^3, 40 steps: doubling the source amplitude doubles every field bit
    for bit (scaling by 2 is exact in binary floating point and the step is
    linear), and the fused and split kernels agree bit for bit."""
    sc = configs.two_spheres(n=512, steps=40)
    g1 = _run_device(sc, kernel="fused")
    f1 = g1.fields()
    g1.close()
    sc.sources[0].amplitude = 2.0
    g2 = _run_device(sc, kernel="fused")
    f2 = g2.fields()
    g2.close()
    assert np.count_nonzero(f1) > 1000
    _assert_fields_equal(f2, 2.0 * f1, "linearity")
    del f2
    g3 = _run_device(sc, kernel="split")
    f3 = g3.fields()
    g3.close()
    _assert_fields_equal(f3, 2.0 * f1, "split vs fused")


def test_wave_propagates_at_approximately_speed_of_light():
    """src/engine.rs:841-932 on the device."""
    dims = wf.GridDims(64, 64, 64)
    dx, dt = 1.0e-3, 1.5e-12
    g = wf.DeviceFieldGrid(dims)
    try:
        g.set_materials(wf.MaterialGrid(dims), wf.MaterialTable.vacuum_filled(dt, dx))
        f = 3.0e10
        src = wf.Source(32, 32, 32, wf.FieldComponent.Ez, 1.0, wf.Waveform.ricker_wavelet(f, 1.0 / f))
        g.add_source_values(32, 32, 32, 2, src.values(dt, 200))
        g.add_probe_tables(52, 32, 32, 2, np.zeros((200, 0)), np.zeros((200, 0)), 0, True)
        g.step(200)
        g.sync()
        tr = g.probe_trace(0, 200)
        arrival = int(np.argmax(np.abs(tr) > 5.0e-4))
        assert abs(tr[arrival]) > 5.0e-4
        measured = (arrival + 1.0) * dt
        expected = 20.0 * dx / 299792458.0
        assert abs(measured - expected) / expected < 0.20
    finally:
        g.close()


def test_convergence_study_on_gpu_reproduces_reference_csv():
    rows, ms, ts, md = studies.convergence_study()
    with open(os.path.join(GOLD, "convergence_data.csv")) as fh:
        gold = list(csv.DictReader(fh))
    for r, gr in zip(rows, gold):
        assert np.float32(gr["measured_phase_velocity"]) == r[2]
        assert np.float32(gr["theoretical_phase_velocity"]) == r[3]
        assert np.float32(gr["measured_relative_error"]) == r[4]
    assert 1.5 <= ms < 2.6 and md < 0.01


def test_pml_reflection_study_on_gpu_reproduces_reference_csv():
    refl = studies.pml_reflection_study()
    with open(os.path.join(GOLD, "pml_reflection_data.csv")) as fh:
        gold = [float(r["reflection_coeff"]) for r in csv.DictReader(fh)]
    assert list(refl) == gold
    assert all(refl[i + 1] < refl[i] for i in range(3)) and refl[-1] < 1e-2


def test_errors_are_reported_not_crashed():
    dims = wf.GridDims(16, 16, 16)
    g = wf.DeviceFieldGrid(dims)
    try:
        with pytest.raises(wf.WfError, match="outside the domain"):
            g.add_source_values(16, 0, 0, 2, np.zeros(4))
        g.add_source_values(1, 1, 1, 2, np.ones(4, np.float32))
        with pytest.raises(wf.WfError, match="has values for 4 steps"):
            g.step(5)
        g.step(4)
        g.sync()
        with pytest.raises(wf.WfError):
            g.set_tiling(7, 16, 3)
    finally:
        g.close()
    with pytest.raises(wf.WfError, match="zero-field"):
        wf.DeviceFieldGrid(dims, boundary=("periodic", "zero", "zero"), kernel="fused")


def test_autotune_keeps_initial_state():
    sc = configs.two_spheres(n=128, steps=10)
    g = configs.device_grid(sc, kernel="fused")
    try:
        best, ms = g.autotune(steps=2)
        assert ms > 0 and best == g.tiling()
        assert g.steps_done == 0 and not g.fields().any()
    finally:
        g.close()
