"""Host-side layout and setup types, mirroring src/layout.rs of the reference.

All numeric setup work (Q16.16 quantization, material coefficients, CPML
profiles, thickness rounding) runs in the library's C++ host code
(wavefront_b200/csrc/wf_host.cpp) so the tables are bit-identical to the
reference's f32 arithmetic.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as _L

BLOCK_DIM = 8  # src/layout.rs:42
VOXELS_PER_BLOCK = BLOCK_DIM ** 3


@dataclass(frozen=True)
class GridDims:
    """GridDims, src/layout.rs:52-89: every axis a multiple of BLOCK_DIM."""
    nx: int
    ny: int
    nz: int

    def __post_init__(self):
        if any(v <= 0 or v % BLOCK_DIM for v in (self.nx, self.ny, self.nz)):
            raise ValueError(
                f"grid dimensions must be multiples of BLOCK_DIM ({BLOCK_DIM}) so the field grid "
                "tiles exactly with no partial edge blocks")

    def voxel_count(self) -> int:
        return self.nx * self.ny * self.nz

    def block_dims(self):
        return self.nx // BLOCK_DIM, self.ny // BLOCK_DIM, self.nz // BLOCK_DIM

    def block_count(self) -> int:
        bx, by, bz = self.block_dims()
        return bx * by * bz


class FixedQ16_16:
    """Q16.16 coefficient quantization, src/layout.rs:105-126."""

    @staticmethod
    def from_f32(v: float) -> int:
        return int(_L.lib().wf_q16_from_f32(v))

    @staticmethod
    def to_f32(q: int) -> np.float32:
        return np.float32(_L.lib().wf_q16_to_f32(q))


VACUUM = 0  # MaterialId::VACUUM, src/layout.rs:144


def material_coeffs(eps_r, mu_r, sigma, dt, d) -> np.ndarray:
    """MaterialTable::coeffs_from_physical (src/layout.rs:194-208) as Q16.16 {ca,cb,da,db}."""
    out = np.zeros(4, np.int32)
    _L.lib().wf_material_coeffs(eps_r, mu_r, sigma, dt, d, _L.ptr(out, _L.i32p))
    return out


class MaterialTable:
    """256-entry Q16.16 coefficient table, src/layout.rs:167-216."""

    def __init__(self, q16: np.ndarray):
        self.q16 = np.ascontiguousarray(q16, np.int32).reshape(256, 4)

    @classmethod
    def vacuum_filled(cls, dt: float, d: float) -> "MaterialTable":
        t = np.empty((256, 4), np.int32)
        t[:] = material_coeffs(1.0, 1.0, 0.0, dt, d)
        return cls(t)

    def set_material(self, mid: int, eps_r, mu_r, sigma, dt, d) -> None:
        self.q16[mid] = material_coeffs(eps_r, mu_r, sigma, dt, d)

    def get(self, mid: int) -> np.ndarray:
        return self.q16[mid]


class MaterialGrid:
    """One byte per voxel, (z*ny+y)*nx+x order (src/layout.rs:275-364), held in RAM."""

    def __init__(self, dims: GridDims, ids: np.ndarray | None = None):
        self.dims = dims
        self.ids = np.zeros(dims.voxel_count(), np.uint8) if ids is None else \
            np.ascontiguousarray(ids, np.uint8).reshape(-1)
        if self.ids.size != dims.voxel_count():
            raise ValueError("material grid size does not match the requested dimensions")

    def material_at(self, x, y, z) -> int:
        return int(self.ids[(z * self.dims.ny + y) * self.dims.nx + x])

    def set_material_at(self, x, y, z, mid) -> None:
        self.ids[(z * self.dims.ny + y) * self.dims.nx + x] = mid


@dataclass
class PmlConfig:
    """src/layout.rs:403-435."""
    thickness: int = BLOCK_DIM
    grading_order: float = 3.0
    kappa_max: float = 7.0
    alpha_max: float = 0.05
    target_reflection: float = 1.0e-6


@dataclass
class PmlProfile1D:
    """Graded b, a, 1/kappa along one axis, src/layout.rs:462-519."""
    b: np.ndarray
    a: np.ndarray
    inv_kappa: np.ndarray
    thickness_voxels: int

    @classmethod
    def build(cls, n: int, config: PmlConfig, dt: float, dx: float,
              thickness_voxels: int) -> "PmlProfile1D":
        b = np.empty(n, np.float32)
        a = np.empty(n, np.float32)
        k = np.empty(n, np.float32)
        _L.lib().wf_pml_profile(n, config.grading_order, config.kappa_max, config.alpha_max,
                                config.target_reflection, dt, dx, thickness_voxels,
                                _L.ptr(b, _L.f32p), _L.ptr(a, _L.f32p), _L.ptr(k, _L.f32p))
        return cls(b, a, k, thickness_voxels)

    def get(self, i: int):
        return float(self.b[i]), float(self.a[i]), float(self.inv_kappa[i])


def effective_pml_thickness_blocks(dims: GridDims, requested_thickness_voxels: int) -> int:
    """src/layout.rs:525-533."""
    return int(_L.lib().wf_effective_pml_thickness_blocks(dims.nx, dims.ny, dims.nz,
                                                          requested_thickness_voxels))


@dataclass
class PmlContext:
    """The three per-axis profiles of PmlContext::build (src/layout.rs:639-656).

    `thickness_voxels[axis]` is the graded depth the device keeps psi for;
    `build` rounds like the reference (whole blocks), `build_exact` keeps the
    requested per-cell thickness (an extension for thin layers)."""
    profiles: tuple
    thickness_voxels: tuple

    @property
    def profile_x(self):
        return self.profiles[0]

    @property
    def profile_y(self):
        return self.profiles[1]

    @property
    def profile_z(self):
        return self.profiles[2]

    @classmethod
    def build(cls, dims: GridDims, config: PmlConfig, dt: float, dx: float) -> "PmlContext":
        t = effective_pml_thickness_blocks(dims, config.thickness) * BLOCK_DIM
        return cls._make(dims, config, dt, dx, (t, t, t))

    @classmethod
    def build_exact(cls, dims: GridDims, config: PmlConfig, dt: float, dx: float,
                    axes=(True, True, True)) -> "PmlContext":
        n = (dims.nx, dims.ny, dims.nz)
        t = tuple(min(config.thickness, n[i] // 2) if axes[i] else 0 for i in range(3))
        return cls._make(dims, config, dt, dx, t)

    @classmethod
    def _make(cls, dims, config, dt, dx, t):
        n = (dims.nx, dims.ny, dims.nz)
        profs = tuple(PmlProfile1D.build(n[i], config, dt, dx, t[i]) for i in range(3))
        return cls(profs, t)
