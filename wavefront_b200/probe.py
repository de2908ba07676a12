"""Running-DFT probes, mirroring src/probe.rs of the reference.

The device accumulates sum += (f64)v * cos/sin(omega*t) in FP64, in step
order, from host-computed twiddle tables (glibc cos/sin of the same f64
phase the reference computes), so sums are bit-identical to
Probe::accumulate (src/probe.rs:126-138).
"""
from __future__ import annotations

import enum
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as _L


class FieldComponent(enum.IntEnum):
    """src/probe.rs:29-37."""
    Ex = 0
    Ey = 1
    Ez = 2
    Hx = 3
    Hy = 4
    Hz = 5


@dataclass(frozen=True)
class FrequencyResponse:
    freq_hz: float
    amplitude: float
    phase_rad: float


@dataclass
class Probe:
    x: int
    y: int
    z: int
    component: FieldComponent
    frequencies_hz: list
    start_recording_at_s: float = 0.0
    record_trace: bool = False
    sum_cos: np.ndarray = field(default=None, repr=False)
    sum_sin: np.ndarray = field(default=None, repr=False)
    samples_recorded: int = 0
    trace: np.ndarray = field(default=None, repr=False)

    def __post_init__(self):
        n = len(self.frequencies_hz)
        self.sum_cos = np.zeros(n, np.float64)
        self.sum_sin = np.zeros(n, np.float64)

    def first_step(self, dt: float) -> int:
        return int(_L.lib().wf_probe_first_step(self.start_recording_at_s, dt))

    def tables(self, dt: float, nsteps: int):
        """cos/sin(omega_f * (double)t_s) for s in [0, nsteps), shape (nsteps, nfreq)."""
        f = np.ascontiguousarray(self.frequencies_hz, np.float32)
        nf = len(f)
        c = np.zeros((nsteps, max(nf, 1)), np.float64)
        s = np.zeros((nsteps, max(nf, 1)), np.float64)
        if nf:
            _L.lib().wf_probe_tables(_L.ptr(f, _L.f32p), nf, dt, 0, nsteps, _L.ptr(c, _L.f64p),
                                     _L.ptr(s, _L.f64p))
        return c[:, :nf].copy(), s[:, :nf].copy()

    def spectrum(self):
        """Probe::spectrum, src/probe.rs:143-167."""
        n = max(self.samples_recorded, 1)
        out = []
        for f, sc, ss in zip(self.frequencies_hz, self.sum_cos, self.sum_sin):
            a = 2.0 * sc / n
            b = 2.0 * ss / n
            out.append(FrequencyResponse(float(np.float32(f)), math.sqrt(a * a + b * b),
                                         math.atan2(a, b)))
        return out

    def position(self):
        return self.x, self.y, self.z
