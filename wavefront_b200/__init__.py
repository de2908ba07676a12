"""wavefront_b200: B200-native (sm_100a) FDTD timestep hot path for wavefront.

The CUDA library (wavefront_b200/lib/libwavefront_gpu.so, C ABI in
include/wavefront_gpu.h) replaces the reference engine's per-step work:
step_all_slabs (Yee H/E updates with CPML), Source::inject and
Probe::accumulate.  This package mirrors the reference's host API
(src/layout.rs, src/source.rs, src/probe.rs, src/scene.rs, src/engine.rs)
on top of it.
"""
from .layout import (BLOCK_DIM, VOXELS_PER_BLOCK, FixedQ16_16, GridDims, MaterialGrid,
                     MaterialTable, PmlConfig, PmlContext, PmlProfile1D,
                     effective_pml_thickness_blocks, material_coeffs)
from .source import FieldComponent, Source, Waveform, default_waveform
from .probe import FrequencyResponse, Probe
from .probe import FieldComponent as ProbeComponent
from .scene import Scene, SceneError, demo_sphere
from .engine import DeviceBatch, DeviceFieldGrid, EngineConfig, PSI_NAMES, SnapshotWriter, run
from ._lib import WfError, lib

__all__ = [
    "BLOCK_DIM", "VOXELS_PER_BLOCK", "FixedQ16_16", "GridDims", "MaterialGrid", "MaterialTable",
    "PmlConfig", "PmlContext", "PmlProfile1D", "effective_pml_thickness_blocks",
    "material_coeffs", "FieldComponent", "Source", "Waveform", "default_waveform",
    "FrequencyResponse", "Probe", "ProbeComponent", "Scene", "SceneError", "demo_sphere",
    "DeviceBatch", "DeviceFieldGrid", "EngineConfig", "PSI_NAMES", "SnapshotWriter", "run", "WfError", "lib",
]
