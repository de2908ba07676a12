"""CPU: the workload builders match the configurations they stand for.

configs.py builds the measured and tested workloads; these tests pin what
each is: grid, dx and dt (0.99/sqrt(3) Courant, rounded to f32), CPML
thickness after the reference's block rounding (or the exact per-cell
layer), the source (position, component, waveform parameters as
src/main.rs:431-460 derives them from a frequency), the probes and the step
count.  A change to a builder that moves a measured workload fails here.
"""
import numpy as np
import pytest

from wavefront_b200 import configs
from wavefront_b200.layout import material_coeffs
from wavefront_b200.source import FieldComponent

C0 = 299792458.0
EZ = int(FieldComponent.Ez)
DT = float(np.float32(0.99 / np.sqrt(3.0) * 1.0e-3 / C0))


def test_plain_cube_64():
    sc = configs.plain_cube_64()
    assert (sc.dims.nx, sc.dims.ny, sc.dims.nz) == (64, 64, 64)
    assert sc.dx == 1.0e-3 and sc.dt == DT and sc.steps == 500
    assert sc.pml.thickness_voxels == (16, 16, 16)  # 10 requested, rounded to whole blocks
    assert configs.plain_cube_64(exact_pml=True).pml.thickness_voxels == (10, 10, 10)
    f0 = float(np.float32(C0 / (20 * 1.0e-3)))
    (s,) = sc.sources
    assert (s.x, s.y, s.z, int(s.component)) == (32, 32, 32, EZ)
    assert s.waveform.kind == 2 and s.waveform.p0 == f0  # Ricker at f0, t0 = 1/f0
    assert s.waveform.p1 == float(np.float32(1.0) / np.float32(f0))
    (p,) = sc.probes
    assert (p.x, p.y, p.z, int(p.component)) == (48, 32, 32, EZ) and p.frequencies_hz == [f0]
    assert not sc.grid.ids.any()  # vacuum


def test_two_spheres_headline():
    sc = configs.two_spheres(512)
    assert (sc.dims.nx, sc.dims.ny, sc.dims.nz) == (512, 512, 512)
    assert sc.dt == DT and sc.steps == 1000 and sc.pml.thickness_voxels == (16, 16, 16)
    assert configs.two_spheres_text(512).splitlines() == [
        "sphere 4.0 1.0 0.0 160 256 256 80", "sphere 2.25 1.0 0.0 352 256 256 60"]
    f = float(np.float32(C0 / (20 * 1.0e-3)))
    (s,) = sc.sources
    assert (s.x, s.y, s.z, int(s.component)) == (256, 256, 64, EZ)
    spread = np.float32(0.5) / np.float32(f)
    assert s.waveform.kind == 0  # Gaussian: t0 = 4 spread
    assert s.waveform.p1 == float(spread) and s.waveform.p0 == float(np.float32(4.0) * spread)
    assert [(p.x, p.y, p.z) for p in sc.probes] == [(32 + 64 * k, 256, 448) for k in range(8)]
    assert all(int(p.component) == EZ and p.frequencies_hz == [f] for p in sc.probes)
    ids = sc.grid.ids.reshape(512, 512, 512)
    assert ids[256, 256, 160] != 0 and ids[256, 256, 352] != 0 and ids[256, 256, 256] == 0
    assert ids[256, 256, 160] != ids[256, 256, 352]  # two materials


def test_random_spheres_mixed_precision_scene():
    sc = configs.random_spheres(128, device_voxelize=True)
    assert sc.steps == 2000 and sc.pml.thickness_voxels == (16, 16, 16) and sc.grid is None
    lines = sc.scene_text.splitlines()
    assert len(lines) == 32 and sc.scene_text == configs.random_spheres_text(128)
    for ln in lines:
        _, eps, mu, sig, cx, cy, cz, r = ln.split()
        assert 1.0 <= float(eps) <= 8.0 and float(mu) == 1.0 and 0.0 <= float(sig) <= 0.01
        assert all(0.0 <= float(v) < 128 for v in (cx, cy, cz))
        assert 20 * 128 / 1024 <= float(r) <= 120 * 128 / 1024
    (s,) = sc.sources
    assert (s.x, s.y, s.z) == (64, 64, 64) and s.waveform.kind == 1  # sinusoid
    assert s.waveform.p0 == float(np.float32(C0 / (15 * 1.0e-3)))
    assert [(p.x, p.y, p.z) for p in sc.probes] == [(8 + 16 * k, 64, 112) for k in range(8)]
    assert configs.random_spheres_text(128, seed=5) != sc.scene_text


def test_batched_sweep():
    scenes = configs.batched_sweep()
    assert len(scenes) == 256 and all(sc.steps == 800 for sc in scenes)
    assert {sc.dims.nx for sc in scenes} == {32, 48, 64, 96, 128}
    assert all(sc.dims.nx == sc.dims.ny == sc.dims.nz for sc in scenes)
    assert sum(sc.dims.voxel_count() for sc in scenes) == 176_095_232
    for sc in scenes:
        assert sc.pml.thickness_voxels == (10, 10, 10)  # exact per-cell layer
        assert 1 <= len(sc.meta["scene"].splitlines()) <= 4
        (s,) = sc.sources
        n = sc.dims.nx
        assert s.waveform.kind == 2 and all(12 <= v < n - 12 for v in (s.x, s.y, s.z))
        ppw = C0 / (s.waveform.p0 * 1.0e-3)
        assert 15.0 - 1e-3 <= ppw <= 30.0 + 1e-3
        (p,) = sc.probes
        assert all(12 <= v < n - 12 for v in (p.x, p.y, p.z))
    # the same seed gives the same sweep
    again = configs.batched_sweep()
    assert [sc.meta["scene"] for sc in again] == [sc.meta["scene"] for sc in scenes]


def test_demo_sphere_reference_benchmark_shape():
    sc = configs.demo_sphere_cube()
    assert (sc.dims.nx, sc.steps, sc.dt) == (256, 150, 1.5e-12)
    assert sc.pml.thickness_voxels == (8, 8, 8)
    assert sc.grid.ids.reshape(256, 256, 256)[128, 128, 128] == 1  # the eps_r 4 sphere
    np.testing.assert_array_equal(sc.table.q16[1], material_coeffs(4.0, 1.0, 0.0, 1.5e-12, 1e-3))
    assert sc.table.q16[1][1] != sc.table.q16[0][1]  # its Cb differs from vacuum's


@pytest.mark.parametrize("n", [64, 128, 256])
def test_two_spheres_scales_with_the_grid(n):
    sc = configs.two_spheres(n)
    s = n / 512
    assert configs.two_spheres_text(n).splitlines()[0].split()[4:] == [
        f"{160 * s:g}", f"{256 * s:g}", f"{256 * s:g}", f"{80 * s:g}"]
    assert (sc.sources[0].x, sc.sources[0].z) == (n // 2, n // 8)
