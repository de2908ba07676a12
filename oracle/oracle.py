"""ctypes loader for the CPU oracle (oracle/build/libwforacle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module, as the checker.  The product package
(wavefront_b200) never imports it.

The oracle is a plain-C restatement of the reference FDTD hot path
(src/fdtd.rs, src/engine.rs, src/layout.rs, src/source.rs, src/probe.rs,
src/scene.rs of AndrejRumenovski/wavefront) in the reference's block-major
8^3 AoSoA layout; see wf_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "build", "libwforacle.so")

_lib = None


def build(quiet: bool = True) -> None:
    """Compiles the oracle with its Makefile (gcc, -ffp-contract=off)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


def _declare(L: C.CDLL) -> None:
    L.or_q16_from_f32.argtypes = [C.c_float]
    L.or_q16_from_f32.restype = C.c_int32
    L.or_q16_to_f32.argtypes = [C.c_int32]
    L.or_q16_to_f32.restype = C.c_float
    L.or_material_coeffs.argtypes = [C.c_float] * 5 + [_i32p]
    L.or_effective_pml_thickness_blocks.argtypes = [C.c_int] * 4
    L.or_effective_pml_thickness_blocks.restype = C.c_int
    L.or_pml_profile.argtypes = [C.c_int] + [C.c_float] * 6 + [C.c_int, _f32p, _f32p, _f32p]
    L.or_waveform_eval.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float]
    L.or_waveform_eval.restype = C.c_float
    L.or_source_values.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, _f32p]
    L.or_probe_tables.argtypes = [_f32p, C.c_int, C.c_float, C.c_int, _f64p, _f64p]
    L.or_probe_first_step.argtypes = [C.c_float, C.c_float]
    L.or_probe_first_step.restype = C.c_int
    L.or_scene_voxelize.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                    C.c_float, _u8p, _i32p, C.c_char_p, C.c_int]
    L.or_scene_voxelize.restype = C.c_int
    L.or_demo_sphere.argtypes = [C.c_int, C.c_int, C.c_int, _u8p]
    L.or_convergence_study.argtypes = [_f32p, _f32p, _f32p, _f32p]
    L.or_pml_reflection_study.argtypes = [_f64p]
    for sfx, rp in (("f32", _f32p), ("f64", _f64p)):
        p = f"or_sim_{sfx}_"
        getattr(L, p + "create").argtypes = [C.c_int, C.c_int, C.c_int, _u8p, _i32p, C.POINTER(C.c_int)]
        getattr(L, p + "create").restype = C.c_void_p
        getattr(L, p + "destroy").argtypes = [C.c_void_p]
        getattr(L, p + "set_pml").argtypes = [C.c_void_p, C.POINTER(_f32p), C.POINTER(_f32p),
                                              C.POINTER(_f32p), C.POINTER(C.c_int)]
        getattr(L, p + "add_source").argtypes = [C.c_void_p] + [C.c_int] * 5 + [_f32p, C.c_int]
        getattr(L, p + "add_source").restype = C.c_int
        getattr(L, p + "add_probe").argtypes = [C.c_void_p] + [C.c_int] * 5 + [_f64p, _f64p, C.c_int, C.c_int, C.c_int]
        getattr(L, p + "add_probe").restype = C.c_int
        getattr(L, p + "step").argtypes = [C.c_void_p, C.c_int, C.c_int]
        getattr(L, p + "steps_done").argtypes = [C.c_void_p]
        getattr(L, p + "steps_done").restype = C.c_int
        getattr(L, p + "get_fields").argtypes = [C.c_void_p, rp]
        getattr(L, p + "set_fields").argtypes = [C.c_void_p, rp]
        getattr(L, p + "get_blocks").argtypes = [C.c_void_p, rp]
        getattr(L, p + "get_psi").argtypes = [C.c_void_p, C.c_int, rp]
        getattr(L, p + "probe_sums").argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, C.POINTER(C.c_uint64)]
        getattr(L, p + "probe_trace").argtypes = [C.c_void_p, C.c_int, _f64p]
        getattr(L, p + "set_storage").argtypes = [C.c_void_p, C.c_int]
        getattr(L, p + "set_storage").restype = C.c_int
        getattr(L, p + "set_arith").argtypes = [C.c_void_p, C.c_int]
        getattr(L, p + "set_arith").restype = C.c_int
        getattr(L, p + "storage_overflows").argtypes = [C.c_void_p]
        getattr(L, p + "storage_overflows").restype = C.c_longlong
        getattr(L, p + "get_shifts").argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.or_store_shift.argtypes = [C.c_float]
    L.or_store_shift.restype = C.c_int
    L.or_store16.argtypes = [C.c_float, C.c_int, C.c_int, C.POINTER(C.c_longlong)]
    L.or_store16.restype = C.c_float


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


# ---- setup math ---------------------------------------------------------------

def q16_from_f32(v: float) -> int:
    return int(lib().or_q16_from_f32(v))


def q16_to_f32(q: int) -> np.float32:
    return np.float32(lib().or_q16_to_f32(q))


def material_coeffs(eps_r, mu_r, sigma, dt, d) -> np.ndarray:
    out = np.zeros(4, np.int32)
    lib().or_material_coeffs(eps_r, mu_r, sigma, dt, d, _ptr(out, _i32p))
    return out


def vacuum_table(dt: float, dx: float) -> np.ndarray:
    t = np.zeros((256, 4), np.int32)
    t[:] = material_coeffs(1.0, 1.0, 0.0, dt, dx)
    return t


def effective_pml_thickness_blocks(nx, ny, nz, req) -> int:
    return int(lib().or_effective_pml_thickness_blocks(nx, ny, nz, req))


def pml_profile(n, dt, dx, thickness_voxels, grading_order=3.0, kappa_max=7.0,
                alpha_max=0.05, target_reflection=1e-6):
    b = np.zeros(n, np.float32)
    a = np.zeros(n, np.float32)
    k = np.zeros(n, np.float32)
    lib().or_pml_profile(n, grading_order, kappa_max, alpha_max, target_reflection, dt, dx,
                         thickness_voxels, _ptr(b, _f32p), _ptr(a, _f32p), _ptr(k, _f32p))
    return b, a, k


def waveform_eval(kind: int, p0: float, p1: float, t: float) -> np.float32:
    return np.float32(lib().or_waveform_eval(kind, p0, p1, t))


def source_values(kind, p0, p1, amplitude, dt, nsteps) -> np.ndarray:
    out = np.zeros(nsteps, np.float32)
    lib().or_source_values(kind, p0, p1, amplitude, dt, nsteps, _ptr(out, _f32p))
    return out


def probe_tables(freqs, dt, nsteps):
    f = np.ascontiguousarray(freqs, np.float32)
    c = np.zeros((nsteps, len(f)), np.float64)
    s = np.zeros((nsteps, len(f)), np.float64)
    lib().or_probe_tables(_ptr(f, _f32p), len(f), dt, nsteps, _ptr(c, _f64p), _ptr(s, _f64p))
    return c, s


def probe_first_step(start, dt) -> int:
    return int(lib().or_probe_first_step(start, dt))


def scene_voxelize(text: str, nx, ny, nz, dt, dx, table=None):
    grid = np.zeros(nx * ny * nz, np.uint8)
    if table is None:
        table = vacuum_table(dt, dx)
    table = np.ascontiguousarray(table, np.int32)
    err = C.create_string_buffer(512)
    n = lib().or_scene_voxelize(text.encode(), nx, ny, nz, dt, dx, _ptr(grid, _u8p),
                                _ptr(table, _i32p), err, 512)
    if n < 0:
        raise ValueError(err.value.decode())
    return grid, table, n


def demo_sphere(nx, ny, nz) -> np.ndarray:
    grid = np.zeros(nx * ny * nz, np.uint8)
    lib().or_demo_sphere(nx, ny, nz, _ptr(grid, _u8p))
    return grid


def convergence_study():
    rows = np.zeros((4, 6), np.float32)
    ms, ts, md = C.c_float(), C.c_float(), C.c_float()
    lib().or_convergence_study(_ptr(rows, _f32p), C.byref(ms), C.byref(ts), C.byref(md))
    return rows, np.float32(ms.value), np.float32(ts.value), np.float32(md.value)


def pml_reflection_study() -> np.ndarray:
    out = np.zeros(4, np.float64)
    lib().or_pml_reflection_study(_ptr(out, _f64p))
    return out


# ---- the engine ---------------------------------------------------------------

class Sim:
    """Oracle timestep engine (src/engine.rs run loop without snapshots)."""

    def __init__(self, nx, ny, nz, mat=None, table=None, periodic=(0, 0, 0), dtype="f32"):
        self.sfx = dtype
        self.real = np.float32 if dtype == "f32" else np.float64
        self.rp = _f32p if dtype == "f32" else _f64p
        self.nx, self.ny, self.nz = nx, ny, nz
        L = lib()
        mat = np.zeros(nx * ny * nz, np.uint8) if mat is None else np.ascontiguousarray(mat, np.uint8).ravel()
        table = np.zeros((256, 4), np.int32) if table is None else np.ascontiguousarray(table, np.int32)
        per = (C.c_int * 3)(*periodic)
        self._h = getattr(L, f"or_sim_{dtype}_create")(nx, ny, nz, _ptr(mat, _u8p), _ptr(table, _i32p), per)
        if not self._h:
            raise ValueError("oracle: grid dimensions must be positive multiples of 8")
        self._keep = []

    def _f(self, name):
        return getattr(lib(), f"or_sim_{self.sfx}_{name}")

    def close(self):
        if self._h:
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_pml(self, profiles, shell_blocks):
        """profiles: [(b, a, ik) or None] per axis."""
        arrs = []
        bs = (_f32p * 3)()
        as_ = (_f32p * 3)()
        ks = (_f32p * 3)()
        for ax in range(3):
            if profiles[ax] is None:
                bs[ax] = as_[ax] = ks[ax] = _f32p()
            else:
                b, a, k = (np.ascontiguousarray(v, np.float32) for v in profiles[ax])
                arrs += [b, a, k]
                bs[ax], as_[ax], ks[ax] = _ptr(b, _f32p), _ptr(a, _f32p), _ptr(k, _f32p)
        sb = (C.c_int * 3)(*shell_blocks)
        self._f("set_pml")(self._h, bs, as_, ks, sb)

    def add_source(self, x, y, z, comp, values, mode=0):
        v = np.ascontiguousarray(values, np.float32)
        if self._f("add_source")(self._h, x, y, z, comp, mode, _ptr(v, _f32p), len(v)) != 0:
            raise ValueError("bad source")

    def add_probe(self, x, y, z, comp, cos_tab, sin_tab, nsteps, first_step=0, record_trace=False):
        c = np.ascontiguousarray(cos_tab, np.float64).reshape(nsteps, -1)
        s = np.ascontiguousarray(sin_tab, np.float64).reshape(nsteps, -1)
        nf = c.shape[1] if nsteps else 0
        if self._f("add_probe")(self._h, x, y, z, comp, nf, _ptr(c, _f64p), _ptr(s, _f64p), nsteps,
                                first_step, int(record_trace)) != 0:
            raise ValueError("bad probe")

    def step(self, n=1, nthreads=1):
        self._f("step")(self._h, n, nthreads)

    @property
    def steps_done(self):
        return int(self._f("steps_done")(self._h))

    def fields(self) -> np.ndarray:
        out = np.zeros((6, self.nz, self.ny, self.nx), self.real)
        self._f("get_fields")(self._h, _ptr(out, self.rp))
        return out

    def set_fields(self, f6):
        a = np.ascontiguousarray(f6, self.real)
        self._f("set_fields")(self._h, _ptr(a, self.rp))

    def blocks(self) -> np.ndarray:
        out = np.zeros(self.nx * self.ny * self.nz * 6, self.real)
        self._f("get_blocks")(self._h, _ptr(out, self.rp))
        return out

    def psi(self, which: int) -> np.ndarray:
        out = np.zeros((self.nz, self.ny, self.nx), self.real)
        self._f("get_psi")(self._h, which, _ptr(out, self.rp))
        return out

    def probe_sums(self, p, nfreq):
        c = np.zeros(max(nfreq, 1), np.float64)
        s = np.zeros(max(nfreq, 1), np.float64)
        n = C.c_uint64()
        self._f("probe_sums")(self._h, p, _ptr(c, _f64p), _ptr(s, _f64p), C.byref(n))
        return c[:nfreq], s[:nfreq], int(n.value)

    def probe_trace(self, p, nsteps) -> np.ndarray:
        out = np.zeros(nsteps, np.float64)
        self._f("probe_trace")(self._h, p, _ptr(out, _f64p))
        return out

    def set_arith(self, arith: str):
        """"exact" (the reference's operations) or "fma": the device FMA build's
        fused forms, fma(b, psi, a*raw), fma(raw, 1/kappa, psi'),
        fma(da, h, -(db*curl)), fma(ca, e, cb*curl) (f32, plain storage)."""
        if self._f("set_arith")(self._h, 1 if arith == "fma" else 0) != 0:
            raise ValueError("the FMA restatement needs the f32 oracle with plain storage")

    def set_storage(self, kind: str):
        """16-bit field storage emulation: "f32" (off), "f16" or "bf16" (both
        round to nearest even), or "f16r8" (binary16 plus a residual byte,
        an emulation with no device form, for the error study).  Call after
        the sources are added (their amplitudes enter the shifts)."""
        if self._f("set_storage")(self._h, STORAGE_KINDS[kind]) != 0:
            raise ValueError("storage emulation needs the f32 oracle")

    @property
    def storage_overflows(self) -> int:
        return int(self._f("storage_overflows")(self._h))

    def shifts(self):
        nbz = self.nz // 8
        e = (C.c_int * nbz)()
        h = (C.c_int * nbz)()
        self._f("get_shifts")(self._h, e, h)
        return np.array(e[:], np.int32), np.array(h[:], np.int32)


# "f16r8" (emulation only, no device form): binary16 plus a residual byte
# per value, the byte cost of a compensated store, for the error study
STORAGE_KINDS = {"f32": 0, "f16": 1, "bf16": 2, "f16r8": 3}


def store_shift(bound: float) -> int:
    return int(lib().or_store_shift(bound))


def store16(v: float, kind: str, shift: int) -> float:
    ov = C.c_longlong(0)
    return float(lib().or_store16(v, STORAGE_KINDS[kind], shift, C.byref(ov)))


def tables_from_description(d):
    """Material ids and the Q16.16 table of a workload description (the plain
    dict of wavefront_b200.configs.*_desc), computed by the oracle alone:
    scene text through the oracle's voxelizer (src/scene.rs:149-230), the
    demo sphere through its rasterizer (src/main.rs:403-425), else vacuum."""
    nx, ny, nz = d["dims"]
    dt, dx = d["dt"], d["dx"]
    table = vacuum_table(dt, dx)
    sc = d["scene"]
    if sc is not None and "text" in sc:
        ids, table, _ = scene_voxelize(sc["text"], nx, ny, nz, dt, dx, table)
    elif sc is not None and "demo_sphere_eps" in sc:
        ids = demo_sphere(nx, ny, nz)
        table[1] = material_coeffs(sc["demo_sphere_eps"], 1.0, 0.0, dt, dx)
    else:
        ids = np.zeros(nx * ny * nz, np.uint8)
    return ids, table


def pml_thickness_from_description(d):
    """Graded depth per axis: the reference's whole-block rounding
    (src/layout.rs:525-533) or, in the exact mode, the request capped at
    half the axis."""
    n = d["dims"]
    p = d["pml"]
    if p is None:
        return (0, 0, 0)
    if p["exact"]:
        return tuple(min(p["cells"], v // 2) for v in n)
    t = effective_pml_thickness_blocks(n[0], n[1], n[2], p["cells"]) * 8
    return (t, t, t)


def sim_from_description(d, steps=None, dtype="f32"):
    """An oracle Sim for a workload description (wavefront_b200.configs.*_desc)
    built with the oracle's own C code only: ids and table, CPML profiles,
    source values and probe twiddles.  Nothing here loads the CUDA library."""
    steps = d["steps"] if steps is None else steps
    nx, ny, nz = d["dims"]
    dt, dx = d["dt"], d["dx"]
    ids, table = tables_from_description(d)
    sim = Sim(nx, ny, nz, ids, table, (0, 0, 0), dtype)
    t = pml_thickness_from_description(d)
    if d["pml"] is not None:
        sim.set_pml([pml_profile(n, dt, dx, tv) for n, tv in zip((nx, ny, nz), t)],
                    [(tv + 7) // 8 for tv in t])
    for s in d["sources"]:
        sim.add_source(s["x"], s["y"], s["z"], s["comp"],
                       source_values(s["kind"], s["p0"], s["p1"], s["amp"], dt, steps), s["mode"])
    for p in d["probes"]:
        c, si = probe_tables(p["freqs"], dt, steps)
        sim.add_probe(p["x"], p["y"], p["z"], p["comp"], c, si, steps,
                      probe_first_step(p["start"], dt))
    return sim


def sim_from_scenario(sc, dtype="f32", periodic=(0, 0, 0), steps=None, storage="f32",
                      arith="exact"):
    """Builds an oracle Sim for a wavefront_b200.configs.Scenario, computing every
    table (CPML profiles, source values, probe twiddles) with the oracle's own
    C code; only the scenario's description and its material ids are shared.
    storage "f16"/"bf16" turns on the 16-bit storage emulation (f32 only);
    arith "fma" restates the device FMA build (f32, plain storage)."""
    steps = sc.steps if steps is None else steps
    d = sc.dims
    sim = Sim(d.nx, d.ny, d.nz, sc.grid.ids, sc.table.q16, periodic, dtype)
    if sc.pml is not None:
        n = (d.nx, d.ny, d.nz)
        profs, shell = [], []
        for ax in range(3):
            t = sc.pml.thickness_voxels[ax]
            profs.append(pml_profile(n[ax], sc.dt, sc.dx, t))
            shell.append((t + 7) // 8)
        sim.set_pml(profs, shell)
    for s in sc.sources:
        w = s.waveform
        sim.add_source(s.x, s.y, s.z, int(s.component),
                       source_values(w.kind, w.p0, w.p1, s.amplitude, sc.dt, steps), s.mode)
    for p in sc.probes:
        c, si = probe_tables(p.frequencies_hz, sc.dt, steps)
        sim.add_probe(p.x, p.y, p.z, int(p.component), c, si, steps,
                      probe_first_step(p.start_recording_at_s, sc.dt), p.record_trace)
    if storage != "f32":
        sim.set_storage(storage)
    if arith != "exact":
        sim.set_arith(arith)
    return sim
