"""Time-domain sources, mirroring src/source.rs of the reference.

The waveform is evaluated on the host in f32 (glibc expf/sinf, as the
reference does) for every step of a run and uploaded; the device only adds
the tabulated value, after the E update (src/engine.rs:769-772).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass

import numpy as np

from . import _lib as _L


class FieldComponent(enum.IntEnum):
    """Components a source can drive (src/source.rs:19-25)."""
    Ex = 0
    Ey = 1
    Ez = 2


@dataclass(frozen=True)
class Waveform:
    """Waveform enum of src/source.rs:28-60: kind 0 Gaussian, 1 Sinusoid, 2 Ricker."""
    kind: int
    p0: float
    p1: float = 0.0

    @classmethod
    def gaussian_pulse(cls, t0: float, spread: float) -> "Waveform":
        return cls(0, t0, spread)

    @classmethod
    def sinusoid(cls, freq_hz: float) -> "Waveform":
        return cls(1, freq_hz, 0.0)

    @classmethod
    def ricker_wavelet(cls, peak_freq_hz: float, t0: float) -> "Waveform":
        return cls(2, peak_freq_hz, t0)

    def evaluate(self, t: float) -> np.float32:
        return np.float32(_L.lib().wf_waveform_eval(self.kind, self.p0, self.p1, t))


SOFT = 0
HARD_SHEET_X = 1


@dataclass
class Source:
    """A point soft source (src/source.rs:62-96); mode HARD_SHEET_X is the
    validation studies' hard Ez sheet over the whole (y,z) plane at x."""
    x: int
    y: int
    z: int
    component: FieldComponent
    amplitude: float
    waveform: Waveform
    mode: int = SOFT

    def values(self, dt: float, nsteps: int, first_step: int = 0) -> np.ndarray:
        """amplitude * evaluate(((s as f32) + 1) * dt) for s in [first, first+nsteps)."""
        out = np.empty(nsteps, np.float32)
        w = self.waveform
        _L.lib().wf_source_values(w.kind, w.p0, w.p1, self.amplitude, dt, first_step, nsteps,
                                  _L.ptr(out, _L.f32p))
        return out


def default_waveform(kind: str, freq_hz: float) -> Waveform:
    """Waveform parameters the CLI derives from a frequency (src/main.rs:431-460)."""
    f = np.float32(freq_hz)
    if kind == "sinusoid":
        return Waveform.sinusoid(float(f))
    if kind == "ricker":
        return Waveform.ricker_wavelet(float(f), float(np.float32(1.0) / f))
    if kind == "gaussian":
        spread = np.float32(0.5) / f
        return Waveform.gaussian_pulse(float(np.float32(4.0) * spread), float(spread))
    raise ValueError(f"unknown waveform kind {kind}")
