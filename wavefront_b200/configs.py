"""Scenario builders for the workloads this project measures and tests.

Each builder returns a `Scenario`: grid dims, dx/dt, material ids + Q16.16
table (voxelized with the reference's scene rules), the CPML context,
sources and probes, the way src/main.rs:508-600 wires a run.

  plain_cube_64       64^3 vacuum, 10-cell CPML request (rounds to 16),
                      Ricker Ez at the centre with 20 cells per wavelength,
                      one Ez probe 16 cells from the source, 500 steps.
  two_spheres(n=512)  two dielectric spheres, 16-cell CPML, Gaussian Ez at
                      (n/2, n/2, n/8), 8 Ez probes on a line at z = 7n/8,
                      1000 steps (the headline throughput workload).
  demo_sphere_cube    the reference's benchmark shape: demo sphere (eps 4)
                      at the centre, 8-cell CPML, dt 1.5 ps, Ricker.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .layout import GridDims, MaterialGrid, MaterialTable, PmlConfig, PmlContext
from .probe import FieldComponent as PC
from .probe import Probe
from .scene import Scene, demo_sphere
from .source import FieldComponent, Source, Waveform, default_waveform

C0 = 299792458.0


def courant_dt(dx: float, factor: float = 0.99) -> float:
    """dt = factor/sqrt(3) * dx / c, rounded to f32 (the engine's dt is f32)."""
    return float(np.float32(factor / np.sqrt(3.0) * dx / C0))


@dataclass
class Scenario:
    name: str
    dims: GridDims
    dx: float
    dt: float
    grid: MaterialGrid
    table: MaterialTable
    pml: Optional[PmlContext]
    sources: List[Source]
    probes: List[Probe]
    steps: int
    meta: dict = field(default_factory=dict)
    # set when the ids are to be rasterized on the device (grid is then None)
    scene_text: Optional[str] = None


def _src(x, y, z, kind, freq, comp=2, amp=1.0, mode=0) -> dict:
    w = default_waveform(kind, freq)
    return {"x": x, "y": y, "z": z, "comp": comp, "amp": amp, "kind": w.kind, "p0": w.p0,
            "p1": w.p1, "mode": mode}


def _prb(x, y, z, freq, comp=2, start=0.0) -> dict:
    return {"x": x, "y": y, "z": z, "comp": comp, "freqs": [freq], "start": start}


def plain_cube_64_desc(steps: int = 500, pml_cells: int = 10, exact_pml: bool = False,
                       n: int = 64) -> dict:
    """Description of plain_cube_64 (plain data: computing it loads no library)."""
    dx = 1.0e-3
    dt = courant_dt(dx)
    f0 = float(np.float32(C0 / (20.0 * dx)))
    c = n // 2
    return {"name": "plain_cube_64", "dims": (n, n, n), "dx": dx, "dt": dt, "scene": None,
            "pml": {"cells": pml_cells, "exact": exact_pml} if pml_cells else None,
            "sources": [_src(c, c, c, "ricker", f0)], "probes": [_prb(c + 16, c, c, f0)],
            "steps": steps, "meta": {"f0": f0}}


def plain_cube_64(steps: int = 500, pml_cells: int = 10, exact_pml: bool = False,
                  n: int = 64) -> Scenario:
    return from_desc(plain_cube_64_desc(steps, pml_cells, exact_pml, n))


def two_spheres_text(n: int) -> str:
    s = n / 512.0
    return (f"sphere 4.0 1.0 0.0 {160 * s:g} {256 * s:g} {256 * s:g} {80 * s:g}\n"
            f"sphere 2.25 1.0 0.0 {352 * s:g} {256 * s:g} {256 * s:g} {60 * s:g}\n")


def two_spheres_desc(n: int = 512, steps: int = 1000, pml_cells: int = 16) -> dict:
    """Description of two_spheres (plain data: computing it loads no library)."""
    dx = 1.0e-3
    dt = courant_dt(dx)
    f = float(np.float32(C0 / (20.0 * dx)))
    zp = (7 * n) // 8
    return {"name": f"two_spheres_{n}", "dims": (n, n, n), "dx": dx, "dt": dt,
            "scene": {"text": two_spheres_text(n)},
            "pml": {"cells": pml_cells, "exact": False} if pml_cells else None,
            "sources": [_src(n // 2, n // 2, n // 8, "gaussian", f)],
            "probes": [_prb(n // 16 + (n // 8) * k, n // 2, zp, f) for k in range(8)],
            "steps": steps, "meta": {"f": f}}


def two_spheres(n: int = 512, steps: int = 1000, pml_cells: int = 16) -> Scenario:
    return from_desc(two_spheres_desc(n, steps, pml_cells))


def random_spheres_text(n: int, count: int = 32, seed: int = 1234) -> str:
    """`count` spheres drawn from numpy's PCG64 stream `seed`, in file order:
    centre U[0,n) per axis, radius U[20,120]*(n/1024) cells, eps_r U[1,8],
    sigma U[0,0.01] S/m, mu_r 1 (a later sphere overwrites an earlier one)."""
    rng = np.random.default_rng(seed)
    lines = []
    for _ in range(count):
        cx, cy, cz = rng.uniform(0.0, n, 3)
        r = rng.uniform(20.0, 120.0) * (n / 1024.0)
        eps = rng.uniform(1.0, 8.0)
        sig = rng.uniform(0.0, 0.01)
        lines.append(f"sphere {eps:.6f} 1.0 {sig:.6f} {cx:.4f} {cy:.4f} {cz:.4f} {r:.4f}")
    return "\n".join(lines) + "\n"


def random_spheres_desc(n: int = 1024, steps: int = 2000, pml_cells: int = 16,
                        seed: int = 1234) -> dict:
    """Description of random_spheres (plain data: computing it loads no library)."""
    dx = 1.0e-3
    dt = courant_dt(dx)
    f = float(np.float32(C0 / (15.0 * dx)))
    c = n // 2
    zp = (7 * n) // 8
    return {"name": f"random_spheres_{n}", "dims": (n, n, n), "dx": dx, "dt": dt,
            "scene": {"text": random_spheres_text(n, seed=seed)},
            "pml": {"cells": pml_cells, "exact": False} if pml_cells else None,
            "sources": [_src(c, c, c, "sinusoid", f)],
            "probes": [_prb(n // 16 + (n // 8) * k, c, zp, f) for k in range(8)],
            "steps": steps, "meta": {"f": f, "seed": seed}}


def random_spheres(n: int = 1024, steps: int = 2000, pml_cells: int = 16,
                   seed: int = 1234, device_voxelize: bool = False) -> Scenario:
    """Mixed-precision workload: 32 seeded random dielectric spheres, 16-cell
    CPML, sinusoid Ez at the centre with 15 cells per wavelength, 8 Ez probes
    on a line at z = 7n/8 (x = n/16 + k*n/8, y = n/2), 2000 steps.  The same
    scene at n = 128 is small enough for the FP64 oracle.  device_voxelize
    leaves the ids to the device voxelizer (device_grid), which at 1024^3
    takes milliseconds instead of the host's minutes."""
    return from_desc(random_spheres_desc(n, steps, pml_cells, seed),
                     device_voxelize=device_voxelize)


def demo_sphere_cube_desc(n: int = 256, steps: int = 150, pml_cells: int = 8) -> dict:
    """Description of demo_sphere_cube (plain data: computing it loads no library)."""
    dx, dt = 1.0e-3, 1.5e-12
    f = float(np.float32(1.0) / (np.float32(20.0) * np.float32(dt)))
    return {"name": f"demo_sphere_{n}", "dims": (n, n, n), "dx": dx, "dt": dt,
            "scene": {"demo_sphere_eps": 4.0},
            "pml": {"cells": pml_cells, "exact": False} if pml_cells else None,
            "sources": [_src(n // 2, n // 2, n // 2, "ricker", f)], "probes": [],
            "steps": steps, "meta": {"f": f}}


def demo_sphere_cube(n: int = 256, steps: int = 150, pml_cells: int = 8) -> Scenario:
    return from_desc(demo_sphere_cube_desc(n, steps, pml_cells))


def from_desc(d: dict, device_voxelize: bool = False) -> Scenario:
    """The Scenario a description stands for, with the library's host code:
    the scene voxelized (or left to the device voxelizer), the Q16.16 table,
    the CPML context (rounded to whole blocks like the reference, or exact),
    the sources and probes."""
    dims = GridDims(*d["dims"])
    dx, dt = d["dx"], d["dt"]
    table = MaterialTable.vacuum_filled(dt, dx)
    grid, text = MaterialGrid(dims), None
    sc_ = d["scene"]
    if sc_ is not None and "text" in sc_:
        if device_voxelize:
            grid, text = None, sc_["text"]
        else:
            Scene.parse(sc_["text"]).voxelize(grid, table, dt, dx)
    elif sc_ is not None and "demo_sphere_eps" in sc_:
        demo_sphere(grid)
        table.set_material(1, sc_["demo_sphere_eps"], 1.0, 0.0, dt, dx)
    pml = None
    if d["pml"] is not None:
        cfg = PmlConfig(thickness=d["pml"]["cells"])
        pml = (PmlContext.build_exact(dims, cfg, dt, dx) if d["pml"]["exact"]
               else PmlContext.build(dims, cfg, dt, dx))
    srcs = [Source(s["x"], s["y"], s["z"], FieldComponent(s["comp"]), s["amp"],
                   Waveform(s["kind"], s["p0"], s["p1"]), s["mode"]) for s in d["sources"]]
    prbs = [Probe(p["x"], p["y"], p["z"], PC(p["comp"]), list(p["freqs"]), p["start"])
            for p in d["probes"]]
    return Scenario(d["name"], dims, dx, dt, grid, table, pml, srcs, prbs, d["steps"],
                    dict(d["meta"]), scene_text=text)


def batched_sweep(n_scenes: int = 256, steps: int = 800, seed: int = 4321,
                  sizes=(32, 48, 64, 96, 128), pml_cells: int = 10) -> List[Scenario]:
    """Batched workload: `n_scenes` independent cubes drawn from numpy's PCG64
    stream `seed`: edge uniform over `sizes`; 1-4 primitives (sphere: centre
    U[0,n), radius U[n/16, n/4]; box: corner U[0,n), extents U[n/8, n/2]),
    eps_r U[1,8], mu_r 1, sigma 0; a 10-cell CPML graded per cell (the
    exact mode: the reference's block rounding would make a 32^3 cube all
    CPML); a Ricker Ez source at a random interior point with 15-30 cells
    per wavelength; one Ez probe at another interior point at the source
    frequency; `steps` steps each."""
    rng = np.random.default_rng(seed)
    dx = 1.0e-3
    dt = courant_dt(dx)
    out = []
    for k in range(n_scenes):
        n = int(rng.choice(sizes))
        lines = []
        for _ in range(int(rng.integers(1, 5))):
            eps = rng.uniform(1.0, 8.0)
            if rng.random() < 0.5:
                c = rng.uniform(0.0, n, 3)
                r = rng.uniform(n / 16.0, n / 4.0)
                lines.append(f"sphere {eps:.6f} 1.0 0.0 {c[0]:.4f} {c[1]:.4f} {c[2]:.4f} {r:.4f}")
            else:
                c = rng.uniform(0.0, n, 3)
                e = rng.uniform(n / 8.0, n / 2.0, 3)
                lines.append(f"box {eps:.6f} 1.0 0.0 {c[0]:.4f} {c[1]:.4f} {c[2]:.4f} "
                             f"{c[0] + e[0]:.4f} {c[1] + e[1]:.4f} {c[2] + e[2]:.4f}")
        text = "\n".join(lines) + "\n"
        lo, hi = pml_cells + 2, n - pml_cells - 2
        sx, sy, sz = (int(v) for v in rng.integers(lo, hi, 3))
        px, py, pz = (int(v) for v in rng.integers(lo, hi, 3))
        ppw = rng.uniform(15.0, 30.0)
        f = float(np.float32(C0 / (ppw * dx)))
        dims = GridDims(n, n, n)
        grid = MaterialGrid(dims)
        table = MaterialTable.vacuum_filled(dt, dx)
        Scene.parse(text).voxelize(grid, table, dt, dx)
        pml = PmlContext.build_exact(dims, PmlConfig(thickness=pml_cells), dt, dx)
        src = Source(sx, sy, sz, FieldComponent.Ez, 1.0, default_waveform("ricker", f))
        prb = Probe(px, py, pz, PC.Ez, [f], 0.0)
        out.append(Scenario(f"batch_{k}_{n}", dims, dx, dt, grid, table, pml, [src], [prb], steps,
                            {"f": f, "scene": text}))
    return out


def device_batch(scenes: List[Scenario], steps: Optional[int] = None, device: int = 0):
    """A DeviceBatch with every scenario's materials, CPML, source values and
    probe tables loaded (tables for `steps` steps, default each scenario's)."""
    from .engine import DeviceBatch
    return load_batch(DeviceBatch([sc.dims for sc in scenes], device=device), scenes, steps)


def load_batch(b, scenes: List[Scenario], steps: Optional[int] = None):
    """Loads every scenario's materials, CPML, source values and probe tables
    into the grids of an allocated DeviceBatch; returns it."""
    for g, sc in zip(b.grids, scenes):
        n = sc.steps if steps is None else steps
        g.set_materials(sc.grid, sc.table)
        if sc.pml is not None:
            g.set_pml(sc.pml)
        for s_ in sc.sources:
            g.add_source_values(s_.x, s_.y, s_.z, s_.component, s_.values(sc.dt, n), s_.mode)
        for p_ in sc.probes:
            c, si = p_.tables(sc.dt, n)
            g.add_probe_tables(p_.x, p_.y, p_.z, p_.component, c, si, p_.first_step(sc.dt))
    return b


def device_grid(sc: Scenario, **kw):
    """A DeviceFieldGrid loaded with the scenario's materials and CPML."""
    from .engine import DeviceFieldGrid
    g = DeviceFieldGrid(sc.dims, **kw)
    if sc.grid is None:
        g.set_scene(sc.scene_text, sc.table, sc.dt, sc.dx)
    else:
        g.set_materials(sc.grid, sc.table)
    if sc.pml is not None:
        g.set_pml(sc.pml)
    return g
