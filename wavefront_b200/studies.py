"""The reference's validation studies, driven through the GPU library.

  convergence_study()     examples/convergence_study.rs:204-369
  pml_reflection_study()  examples/pml_reflection_study.rs:237-387

Both drive a 1D plane wave in an nx x 8 x 8 vacuum domain with periodic Y/Z
(the split kernels handle periodic axes), a hard Ez sheet source and a probe
trace, then post-process in the reference's f32/f64 arithmetic (libm for
sinf/asinf/log10f, as the reference's f32 methods call).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from .engine import DeviceFieldGrid
from .layout import GridDims, MaterialGrid, MaterialTable, PmlConfig, PmlProfile1D
from .source import HARD_SHEET_X, FieldComponent, Source, Waveform

_libm = ctypes.CDLL("libm.so.6")
for _fn in ("sinf", "asinf", "log10f"):
    getattr(_libm, _fn).argtypes = [ctypes.c_float]
    getattr(_libm, _fn).restype = ctypes.c_float

F = np.float32
C0 = F(299792458.0)
PI_F = F(np.pi)


def _round_half_away(x: float) -> float:
    r = math.floor(abs(x))
    if abs(x) - r >= 0.5:
        r += 1.0
    return math.copysign(r, x)


def _nx8(v: int) -> int:
    return (v + 7) // 8 * 8


def plane_wave_trace(nx: int, dx, dt, freq, x_source: int, x_probe: int, steps: int,
                     pml_voxels: int, device: int = 0) -> np.ndarray:
    """run_plane_wave of both studies on the GPU; returns the f32 Ez trace."""
    dims = GridDims(nx, 8, 8)
    g = DeviceFieldGrid(dims, boundary=("zero", "periodic", "periodic"), kernel="split",
                        device=device)
    try:
        g.set_materials(MaterialGrid(dims), MaterialTable.vacuum_filled(float(dt), float(dx)))
        if pml_voxels > 0:
            tb = min((pml_voxels + 7) // 8, (nx // 8) // 2)
            p = PmlProfile1D.build(nx, PmlConfig(thickness=pml_voxels), float(dt), float(dx), tb * 8)
            if tb > 0:
                g.set_pml_axis(0, tb * 8, p.b, p.a, p.inv_kappa)
        src = Source(x_source, 0, 0, FieldComponent.Ez, 1.0, Waveform.sinusoid(float(freq)),
                     HARD_SHEET_X)
        g.add_source_values(src.x, 0, 0, 2, src.values(float(dt), steps), HARD_SHEET_X)
        g.add_probe_tables(x_probe, 0, 0, 2, np.zeros((steps, 0)), np.zeros((steps, 0)), 0, True)
        g.step(steps)
        g.sync()
        return g.probe_trace(0, steps)
    finally:
        g.close()


def _quadrature(trace, dt, omega: float, skip):
    sc = ss = 0.0
    count = 0
    for i, v in enumerate(trace):
        t = F(F(i) + F(1.0)) * dt
        if t > skip:
            ph = omega * float(t)
            sc += float(v) * math.cos(ph)
            ss += float(v) * math.sin(ph)
            count += 1
    return 2.0 * sc / count, 2.0 * ss / count


def _theory_v(dx, dt, f):
    omega = F(F(2.0) * PI_F) * f
    rhs = F(dx / F(C0 * dt)) * F(_libm.sinf(F(omega * dt) / F(2.0)))
    k = F(F(2.0) / dx) * F(_libm.asinf(rhs))
    return F(omega / k)


def _slope(xs, ys):
    lx = [F(_libm.log10f(x)) for x in xs]
    ly = [F(_libm.log10f(y)) for y in ys]
    n = F(len(lx))
    mx = F(sum(lx, F(-0.0)) / n)
    my = F(sum(ly, F(-0.0)) / n)
    cov = F(-0.0)
    var = F(-0.0)
    for a, b in zip(lx, ly):
        cov = F(cov + F(F(a - mx) * F(b - my)))
    for a in lx:
        d = F(a - mx)
        var = F(var + F(d * d))
    return F(cov / var)


def convergence_study(device: int = 0):
    """Returns (rows[4][6] f32, measured_slope, theory_slope, max_discrepancy)."""
    freq = F(3.0e10)
    wl = F(C0 / freq)
    courant = F(0.4)
    periods = F(8.0)
    rows = np.zeros((4, 6), np.float32)
    for r, ppw in enumerate([F(10.0), F(15.0), F(20.0), F(30.0)]):
        dx = F(wl / ppw)
        dt = F(F(courant * dx) / C0)
        period_s = F(F(1.0) / freq)
        period_steps = F(ppw / courant)
        n_vox = int(_round_half_away(float(F(periods * ppw))))
        x_source = 3 * n_vox
        x_probe = x_source + n_vox
        nx = _nx8(7 * n_vox)
        steps = int(math.ceil(float(F(F(periods + F(12.0)) * period_steps))))
        expected = F(F(F(n_vox) * dx) / C0)
        omega = 2.0 * math.pi * float(freq)
        trace = plane_wave_trace(nx, dx, dt, freq, x_source, x_probe, steps, 0, device)
        skip = F(expected + F(F(5.0) * period_s))
        a, b = _quadrature(trace, dt, omega, skip)
        raw_delay = math.atan2(-a, b) / omega
        k = _round_half_away((float(expected) - raw_delay) / float(period_s))
        measured = F(raw_delay + k * float(period_s))
        mv = F(F(F(n_vox) * dx) / measured)
        tv = _theory_v(dx, dt, freq)
        rows[r] = [dx, ppw, mv, tv, F(abs(F(mv - C0)) / C0), F(abs(F(tv - C0)) / C0)]
    ms = _slope(rows[:, 0], rows[:, 4])
    ts = _slope(rows[:, 0], rows[:, 5])
    md = F(0.0)
    for r in range(4):
        md = max(md, F(abs(F(rows[r, 4] - rows[r, 5]))))
    return rows, ms, ts, md


def pml_reflection_study(device: int = 0) -> np.ndarray:
    """|R| for 1, 2, 4, 8 block CPML layers (f64)."""
    freq = F(3.0e10)
    wl = F(C0 / freq)
    ppw = F(20.0)
    dx = F(wl / ppw)
    dt = F(F(F(0.4) * dx) / C0)
    period_s = F(F(1.0) / freq)
    probe_off = int(_round_half_away(float(F(F(3.0) * ppw))))
    right_gap = int(_round_half_away(float(F(F(2.0) * ppw))))
    out = np.zeros(4)
    for r, tb in enumerate([1, 2, 4, 8]):
        T = tb * 8
        xs_t = T + int(_round_half_away(float(F(F(2.0) * ppw))))
        xp_t = xs_t + probe_off
        face = xp_t + right_gap
        nx_t = _nx8(face + T)
        inc_delay = F(F(F(probe_off) * dx) / C0)
        rt_s = F(F(F(2 * (face - xp_t)) * dx) / C0)
        skip = F(F(inc_delay + rt_s) + F(F(6.0) * period_s))
        steps = int(math.ceil(float(F(F(skip + F(F(10.0) * period_s)) / dt)))) + 4
        tt = plane_wave_trace(nx_t, dx, dt, freq, xs_t, xp_t, steps, T, device)
        req = int(math.ceil(float(F(F(F(F(F(steps) * dt) + F(F(2.0) * period_s)) * C0) / dx)))) + 8
        xp_r = req + probe_off
        xs_r = xp_r - probe_off
        nx_r = _nx8(xp_r + req)
        rt = plane_wave_trace(nx_r, dx, dt, freq, xs_r, xp_r, steps, 0, device)
        omega = 2.0 * math.pi * float(freq)
        a, b = _quadrature(rt, dt, omega, skip)
        inc = math.sqrt(a * a + b * b)
        a, b = _quadrature((tt - rt).astype(np.float32), dt, omega, skip)
        out[r] = math.sqrt(a * a + b * b) / inc
    return out
