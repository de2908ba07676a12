"""GPU: trajectory snapshots and checkpoint / resume.

1. engine.run with output_path writes wave_trajectory.bin: one FieldBlock
   snapshot (src/engine.rs:617-640) after every step whose index is a
   multiple of snapshot_every, appended back to back; each equals the oracle's
   blocks at that step bit for bit (FP32, and binary16 and bfloat16 against
   the storage emulation), and voxels read the way src/bin/wavefront-view.rs:280-305
   reads them equal the oracle's fields.
2. The writer overlaps stepping: captures taken between steps on a larger
   grid equal wf_download_blocks at the same steps.
3. A checkpoint taken mid-run and loaded into a second, identically
   configured grid continues bit for bit (fields, all psi, probe sums and
   traces, 16-bit shifts and saturation count).
4. A checkpoint of another configuration is refused before anything changes;
   a damaged one is reported.
"""
import os

import numpy as np
import pytest

import wavefront_b200 as wf
from oracle import oracle as O
from wavefront_b200 import _lib as L
from wavefront_b200 import configs
from wavefront_b200.engine import EngineConfig, run

pytestmark = pytest.mark.gpu
NT = min(os.cpu_count() or 1, 32)
BLOCK_FLOATS = 6 * 512  # FieldBlock: ex..hz x 8^3


def _eq(got, want, what):
    bad = got != want  # +0 == -0
    if bad.any():
        idx = np.argwhere(bad)[:5]
        raise AssertionError(f"{what}: {bad.sum()} values differ, first {idx.tolist()}, "
                             f"got {got[bad][:5]} want {want[bad][:5]}")


def _configure(g, sc, steps, trace=False):
    for s in sc.sources:
        g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, steps), s.mode)
    for p in sc.probes:
        c, si = p.tables(sc.dt, steps)
        g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(sc.dt), trace)


def _read_component(snap, dims, x, y, z, field):
    """src/bin/wavefront-view.rs:280-305 on one snapshot's floats."""
    nbx, nby = dims.nx // 8, dims.ny // 8
    b = ((z // 8) * nby + y // 8) * nbx + x // 8
    local = ((z % 8) * 8 + y % 8) * 8 + x % 8
    return snap[b * BLOCK_FLOATS + field * 512 + local]


@pytest.mark.parametrize("prec", ["f32", "f16", "bf16"])
def test_trajectory_file_matches_oracle(tmp_path, prec):
    steps, every = 40, 10
    sc = configs.plain_cube_64(steps=steps)
    path = tmp_path / "wave_trajectory.bin"
    g = configs.device_grid(sc, precision=prec)
    try:
        run(g, sc.sources, [], EngineConfig(num_steps=steps, dt=sc.dt, snapshot_every=every,
                                            output_path=str(path)))
    finally:
        g.close()
    sim = O.sim_from_scenario(sc, steps=steps, storage=prec)
    want = []
    for s in range(steps):
        sim.step(1, nthreads=NT)
        if s % every == 0:
            want.append((sim.blocks().copy(), sim.fields().copy()))
    raw = np.fromfile(path, np.float32)
    n_floats = sc.dims.voxel_count() * 6
    assert raw.size == len(want) * n_floats  # no header, snapshots back to back
    rng = np.random.default_rng(3)
    for k, (blocks, fields) in enumerate(want):
        snap = raw[k * n_floats:(k + 1) * n_floats]
        _eq(snap, blocks.ravel(), f"snapshot {k}")
        for _ in range(20):
            x, y, z = (int(v) for v in rng.integers(0, 64, 3))
            c = int(rng.integers(0, 6))
            v = _read_component(snap, sc.dims, x, y, z, c)
            assert v == fields[c, z, y, x] or (v == 0 and fields[c, z, y, x] == 0)


def test_writer_overlaps_stepping(tmp_path):
    sc = configs.random_spheres(n=128, steps=60, pml_cells=16)
    path = tmp_path / "traj.bin"
    g = configs.device_grid(sc)
    ref = configs.device_grid(sc)
    try:
        for grid in (g, ref):
            _configure(grid, sc, 61)
        want = []
        with g.snapshot_writer(path) as w:
            for _ in range(5):
                g.step(12)
                w.capture()  # no sync: the copy and the write overlap the next steps
                ref.step(12)
                want.append(ref.download_blocks())
            g.step(1)
            nbytes = w.close()
        n = sc.dims.voxel_count() * 6
        assert nbytes == 5 * n * 4 == os.path.getsize(path)
        raw = np.fromfile(path, np.float32)
        for k in range(5):
            _eq(raw[k * n:(k + 1) * n], want[k], f"capture {k}")
    finally:
        g.close()
        ref.close()


@pytest.mark.parametrize("prec", ["f32", "f16", "bf16"])
def test_checkpoint_resume_is_bit_exact(tmp_path, prec):
    steps = 90
    sc = configs.random_spheres(n=64, steps=steps, pml_cells=10)
    path = tmp_path / "state.ckpt"
    a = configs.device_grid(sc, precision=prec)
    b = configs.device_grid(sc, precision=prec)
    try:
        for g in (a, b):
            _configure(g, sc, steps, trace=True)
        a.step(50)
        a.checkpoint(path)
        a.step(40)
        b.restore(path)
        assert b.steps_done == 50
        b.step(40)
        a.sync()
        b.sync()
        _eq(b.fields(), a.fields(), "fields")
        for w in range(12):
            _eq(b.psi(w), a.psi(w), wf.PSI_NAMES[w])
        for i, p in enumerate(sc.probes):
            nf = len(p.frequencies_hz)
            ac, as_, an = a.probe_sums(i, nf)
            bc, bs, bn = b.probe_sums(i, nf)
            assert an == bn and np.array_equal(ac, bc) and np.array_equal(as_, bs)
            assert np.array_equal(a.probe_trace(i, steps), b.probe_trace(i, steps))
        if prec != "f32":
            ae, ah, ao = a.storage_info()
            be, bh, bo = b.storage_info()
            assert np.array_equal(ae, be) and np.array_equal(ah, bh) and ao == bo
    finally:
        a.close()
        b.close()


def test_checkpoint_refuses_other_configurations_and_damage(tmp_path):
    sc = configs.plain_cube_64(steps=20)
    path = tmp_path / "s.ckpt"
    g = configs.device_grid(sc)
    other = configs.device_grid(configs.plain_cube_64(steps=20, n=40))
    no_pml = configs.device_grid(configs.plain_cube_64(steps=20, pml_cells=0))
    try:
        _configure(g, sc, 20)
        g.step(7)
        g.checkpoint(path)
        before = g.fields()
        for wrong in (other, no_pml):
            with pytest.raises(wf.WfError) as e:
                wrong.restore(path)
            assert e.value.status == L.WF_ERR_ARG
        data = bytearray(path.read_bytes())
        data[len(data) // 2] ^= 0x40
        bad = tmp_path / "bad.ckpt"
        bad.write_bytes(bytes(data))
        h = configs.device_grid(sc)
        try:
            _configure(h, sc, 20)
            with pytest.raises(wf.WfError) as e:
                h.restore(bad)
            assert e.value.status == L.WF_ERR_IO
            h.restore(path)
            _eq(h.fields(), before, "restored fields")
        finally:
            h.close()
    finally:
        for x in (g, other, no_pml):
            x.close()


def test_async_download_overlaps_stepping_and_equals_the_oracle():
    """wf_download_blocks_async: the FieldBlock bytes of the state at the
    call, copied while later steps run (two downloads in flight order
    themselves on the staging buffer), equal the oracle's blocks at those
    steps; 16-bit storage is refused."""
    import torch
    sc = configs.two_spheres(n=64, steps=40)
    sim = O.sim_from_scenario(sc)
    g = configs.device_grid(sc, kernel="fused")
    try:
        for s in sc.sources:
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, sc.steps))
        bufs = [torch.empty(sc.dims.voxel_count() * 6, dtype=torch.float32).pin_memory()
                for _ in range(2)]
        g.step(3)
        g.download_blocks_async(bufs[0].numpy())
        g.step(9)
        g.download_blocks_async(bufs[1].numpy())
        g.step(20)
        g.sync()
        sim.step(3, NT)
        want3 = sim.blocks()
        sim.step(9, NT)
        want12 = sim.blocks()
        _eq(bufs[0].numpy(), want3, "download after 3 steps")
        _eq(bufs[1].numpy(), want12, "download after 12 steps")
        sim.step(20, NT)
        _eq(g.fields(), sim.fields(), "fields after the downloads")
    finally:
        g.close()
        sim.close()
    h = wf.DeviceFieldGrid(wf.GridDims(16, 16, 16), precision="f16")
    try:
        with pytest.raises(wf.WfError):
            h.reserve_download()
    finally:
        h.close()
