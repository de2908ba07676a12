"""Plain-text scene format and voxelizer, mirroring src/scene.rs of the reference.

Parsing and rasterization run in the library's C++ host code
(wf_scene_voxelize) with the reference's f32 cell-centre test, file-order
overwrite and bit-pattern material de-duplication.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as _L
from .layout import GridDims, MaterialGrid, MaterialTable


class SceneError(ValueError):
    pass


class Scene:
    def __init__(self, text: str):
        self.text = text

    @classmethod
    def load(cls, path) -> "Scene":
        try:
            with open(path) as f:
                return cls.parse(f.read())
        except OSError as e:
            raise SceneError(f"failed to read scene file {path!r}: {e}") from e

    @classmethod
    def parse(cls, text: str) -> "Scene":
        # Validate now (Scene::parse reports line errors before voxelizing).
        grid = np.zeros(8 * 8 * 8, np.uint8)
        tab = np.zeros((256, 4), np.int32)
        _voxelize(text, GridDims(8, 8, 8), grid, tab, 1e-12, 1e-3)
        return cls(text)

    def voxelize(self, grid: MaterialGrid, table: MaterialTable, dt: float, dx: float) -> int:
        """Scene::voxelize, src/scene.rs:149-188; returns the material count."""
        return _voxelize(self.text, grid.dims, grid.ids, table.q16, dt, dx)


def _voxelize(text, dims, ids, q16, dt, dx) -> int:
    err = C.create_string_buffer(512)
    n = C.c_int(0)
    st = _L.lib().wf_scene_voxelize(text.encode(), dims.nx, dims.ny, dims.nz, dt, dx,
                                    _L.ptr(ids, _L.u8p), _L.ptr(q16, _L.i32p), C.byref(n), err, 512)
    if st != _L.WF_OK:
        raise SceneError(err.value.decode())
    return int(n.value)


def demo_sphere(grid: MaterialGrid) -> None:
    """voxelize_demo_sphere, src/main.rs:403-425 (material id 1)."""
    d = grid.dims
    _L.lib().wf_demo_sphere(d.nx, d.ny, d.nz, _L.ptr(grid.ids, _L.u8p))
