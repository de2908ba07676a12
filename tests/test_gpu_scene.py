"""GPU: the device scene voxelizer (wf_set_scene) against the host
voxelizer (wf_scene_voxelize, itself checked against the oracle's
restatement of src/scene.rs:149-230): identical material ids and tables for
spheres, boxes partly outside the grid, overlapping primitives (file order:
a later primitive overwrites), and the reference's parse errors."""
import numpy as np
import pytest

import wavefront_b200 as wf
from wavefront_b200 import configs

pytestmark = pytest.mark.gpu


def _device_ids(dims, text, dt, dx):
    table = wf.MaterialTable.vacuum_filled(dt, dx)
    g = wf.DeviceFieldGrid(dims)
    try:
        n = g.set_scene(text, table, dt, dx)
        return g.materials(), table.q16.copy(), n
    finally:
        g.close()


def _host_ids(dims, text, dt, dx):
    grid = wf.MaterialGrid(dims)
    table = wf.MaterialTable.vacuum_filled(dt, dx)
    wf.Scene.parse(text).voxelize(grid, table, dt, dx)
    return grid.ids, table.q16.copy()


@pytest.mark.parametrize("case", ["two_spheres", "random_spheres", "boxes"])
def test_device_voxelizer_matches_host(case):
    dx = 1e-3
    dt = configs.courant_dt(dx)
    if case == "two_spheres":
        dims, text = wf.GridDims(128, 128, 128), configs.two_spheres_text(128)
    elif case == "random_spheres":
        dims, text = wf.GridDims(128, 96, 136), configs.random_spheres_text(128)
    else:
        dims = wf.GridDims(72, 40, 48)
        text = ("box 2.5 1.5 0.0 -5 3.2 2 30.7 80 20\n"
                "sphere 4.0 1.0 0.02 35.5 20 12 9.25\n"
                "box 3.0 1.0 0.01 50 -1e30 10 1e30 12.5 47.9\n"
                "sphere 2.5 1.5 0.0 70 38 46 13\n"
                "box 4.0 1.0 0.02 10 10 10 10 20 20\n")
    got, gt, n = _device_ids(dims, text, dt, dx)
    want, wt = _host_ids(dims, text, dt, dx)
    assert n >= 1
    assert np.array_equal(gt, wt)
    bad = np.count_nonzero(got != want)
    assert bad == 0, f"{bad} cells differ"
    assert np.any(got)


def test_device_voxelizer_reports_parse_errors():
    g = wf.DeviceFieldGrid(wf.GridDims(16, 16, 16))
    try:
        table = wf.MaterialTable.vacuum_filled(1e-12, 1e-3)
        with pytest.raises(wf.WfError, match="unknown primitive 'cone'"):
            g.set_scene("sphere 2 1 0 8 8 8 3\ncone 1 1 0 1 1 1 1\n", table, 1e-12, 1e-3)
        with pytest.raises(wf.WfError, match="invalid number"):
            g.set_scene("sphere 2 1 0 8 8 x8 3\n", table, 1e-12, 1e-3)
    finally:
        g.close()
