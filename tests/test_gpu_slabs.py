"""GPU: the z-slab decomposition in one process against the whole grid.

A grid split into 2-4 z slabs (SlabDomain: one handle per slab on one device,
each on its own stream, ghost blocks moved every 8 steps by the pack/unpack
kernels)
must give the whole grid's fields and probe sums, with +0 and -0 treated as
equal (the slabs holding the z CPML run its interior-valued profile on their
other side, where the correction can flip the sign of a zero).  The scenes
have CPML on every axis, so the x and y psi of the ghost planes move too,
and sources on ghost planes.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from wavefront_b200 import configs  # noqa: E402
from wavefront_b200 import slabs as S  # noqa: E402
from wavefront_b200._lib import WF_ERR_UNSUPPORTED, WfError  # noqa: E402
from wavefront_b200.engine import DeviceFieldGrid  # noqa: E402
from wavefront_b200.source import FieldComponent, Source, default_waveform  # noqa: E402

pytestmark = pytest.mark.gpu
STEPS = 61


def _eq(got, want, what):
    bad = got != want
    assert not bad.any(), f"{what}: {bad.sum()} cells differ, first {np.argwhere(bad)[:4].tolist()}"


def _scene(n=128, device_voxelize=False):
    if device_voxelize:
        sc = configs.random_spheres(n, steps=STEPS, device_voxelize=True)
    else:
        sc = configs.two_spheres(n, steps=STEPS)
    f = sc.meta["f"]
    # sources on planes that are ghost planes of the 2- and 4-way plans
    sc.sources.append(Source(40, 50, 60, FieldComponent.Ex, 0.25, default_waveform("ricker", f)))
    sc.sources.append(Source(70, 61, 66, FieldComponent.Ey, -0.5, default_waveform("ricker", f)))
    return sc


def _whole(sc, **kw):
    g = configs.device_grid(sc, **kw)
    for s in sc.sources:
        g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, STEPS), s.mode)
    for p in sc.probes:
        c, si = p.tables(sc.dt, STEPS)
        g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(sc.dt))
    g.step(STEPS)
    g.sync()
    return g


def _check(sc, parts, **kw):
    whole = _whole(sc, **kw)
    want = whole.fields()
    assert np.abs(want).max() > 0
    d = S.SlabDomain(sc, parts, steps=STEPS, **kw)
    try:
        d.step(3)
        d.step(STEPS - 3)
        assert d.exchanges == (STEPS - 1) // S.GHOST
        _eq(d.fields(), want, f"fields, {parts} slabs")
        _eq(d.download_blocks(), whole.download_blocks(), f"FieldBlock snapshot, {parts} slabs")
        for i, p in enumerate(sc.probes):
            nf = len(p.frequencies_hz)
            gc, gs, gn = d.probe_sums(i, nf)
            wc, ws, wn = whole.probe_sums(i, nf)
            assert gn == wn and np.array_equal(gc, wc) and np.array_equal(gs, ws), i
    finally:
        d.close()
        whole.close()


@pytest.mark.parametrize("parts", [2, 3, 4])
def test_slab_domain_equals_whole_grid(parts):
    _check(_scene(), parts)


def test_slab_domain_split_kernel():
    _check(_scene(), 2, kernel="split")


def test_slab_domain_fma_build():
    _check(_scene(), 3, arith="fma")


def test_scene_window_voxelizer_and_device_scene():
    sc = _scene(device_voxelize=True)
    whole = DeviceFieldGrid(sc.dims)
    whole.set_scene(sc.scene_text, sc.table, sc.dt, sc.dx)
    ids = whole.materials().reshape(sc.dims.nz, -1)
    whole.close()
    for s in S.plan(sc.dims.nz, 3, 16):
        g = DeviceFieldGrid(configs.GridDims(sc.dims.nx, sc.dims.ny, s.nz))
        g.set_scene_window(sc.scene_text, configs.MaterialTable(sc.table.q16.copy()), sc.dt,
                           sc.dx, sc.dims.nz, s.lo)
        assert np.array_equal(g.materials().reshape(s.nz, -1), ids[s.lo:s.hi])
        g.close()
    _check(sc, 3)


def test_pack_unpack_round_trip_moves_fields_and_psi():
    sc = configs.two_spheres(64, steps=20)
    a = _whole(sc)
    b = configs.device_grid(sc)
    import torch
    n = a.slab_floats(8)
    nx = ny = 64
    row_x = ny * ((32 + 3) // 4 * 4)  # x psi: 2 x 16 slab positions per row
    assert n == 6 * 8 * nx * ny + 4 * 8 * row_x + 4 * 8 * 32 * nx
    buf = torch.empty(n, dtype=torch.float32, device="cuda")
    a.pack_planes(24, 8, buf.data_ptr(), n)
    b.unpack_planes(8, 8, buf.data_ptr(), n)
    a.sync()
    b.sync()
    fa, fb = a.fields(), b.fields()
    assert np.array_equal(fb[:, 8:16].view(np.uint32), fa[:, 24:32].view(np.uint32))
    assert not fb[:, :8].any() and not fb[:, 16:].any()
    for w in (0, 1, 2, 3, 6, 7, 8, 9):  # x and y psi arrays
        pa, pb = a.psi(w), b.psi(w)
        assert np.array_equal(pb[8:16].view(np.uint32), pa[24:32].view(np.uint32)), w
    a.close()
    b.close()


def test_slab_copies_reject_bad_arguments():
    import torch
    g = DeviceFieldGrid(configs.GridDims(32, 32, 32), precision="f16")
    buf = torch.empty(1 << 16, dtype=torch.float32, device="cuda")
    cap = buf.numel()
    with pytest.raises(WfError) as e:
        g.pack_planes(0, 8, buf.data_ptr(), cap)
    assert e.value.status == WF_ERR_UNSUPPORTED
    g.close()
    g = DeviceFieldGrid(configs.GridDims(32, 32, 32))
    with pytest.raises(WfError):
        g.pack_planes(30, 8, buf.data_ptr(), cap)  # past nz
    with pytest.raises(WfError):
        g.pack_planes(0, 8, buf.data_ptr() + 4, cap - 1)  # not 16-byte aligned
    need = g.slab_floats(8)
    for bad in (need - 4, 0):  # a buffer smaller than the planes need
        with pytest.raises(WfError) as e:
            g.unpack_planes(0, 8, buf.data_ptr(), bad)
        assert "floats" in str(e.value)
    g.pack_planes(0, 8, buf.data_ptr(), need)
    with pytest.raises(ValueError):
        g.slab_floats(0)
    text = "sphere 4.0 1.0 0.0 16 16 16 6\n"
    table = configs.MaterialTable.vacuum_filled(1e-12, 1e-3)
    for nz_global, off in ((24, 0), (64, 40), (64, -8)):  # window outside the global grid
        with pytest.raises(WfError):
            g.set_scene_window(text, table, 1e-12, 1e-3, nz_global, off)
    g.set_scene_window(text, table, 1e-12, 1e-3, 64, 32)  # planes 32..63: the sphere misses
    assert not g.materials().any()
    g.close()


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        r = S.SlabRank(_scene(), steps=STEPS)
        r.step(5)
        r.step(STEPS - 5)
        f = r.gather_fields()
        pr = r.gather_probe_sums(1)
        if rank == 0:
            np.savez(out, fields=f, exchanges=r.exchanges,
                     **{f"p{k}": np.array([v[0][0], v[1][0], v[2]]) for k, v in pr.items()})
        r.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_slab_ranks_gloo_host_staging_on_one_gpu(tmp_path, world):
    """SlabRank in separate processes (gloo, blocks staged through pinned
    host buffers), every rank's slab on the one GPU: the gathered fields and
    probe sums equal the whole grid's.  No kernel waits on another rank: the
    exchange happens on the host between launches."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "ranks.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world,
                       start_method="spawn", join=True)
    got = np.load(out)
    sc = _scene()
    whole = _whole(sc)
    try:
        assert int(got["exchanges"]) == (STEPS - 1) // S.GHOST
        _eq(got["fields"], whole.fields(), f"fields, {world} ranks")
        for i in range(len(sc.probes)):
            c, si, n = whole.probe_sums(i, 1)
            assert np.array_equal(got[f"p{i}"], np.array([c[0], si[0], n])), i
    finally:
        whole.close()


def test_graph_steps_change_only_the_launch_grouping():
    sc = configs.two_spheres(64, steps=50)
    out = []
    for gs in (None, 8, 2):
        g = configs.device_grid(sc)
        if gs:
            g.set_graph_steps(gs)
        for s in sc.sources:
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, 50), s.mode)
        g.step(21)
        g.step(29)
        g.sync()
        out.append(g.fields())
        if gs == 8:
            for bad in (0, 3, 2048):
                with pytest.raises(WfError):
                    g.set_graph_steps(bad)
        g.close()
    assert np.abs(out[0]).max() > 0
    for f in out[1:]:
        assert np.array_equal(f.view(np.uint32), out[0].view(np.uint32))


def test_slab_domain_checkpoint_resumes_bit_exactly(tmp_path):
    sc = _scene()
    ref = S.SlabDomain(sc, 3, steps=STEPS)
    try:
        ref.step(STEPS)
        want, want_blocks = ref.fields(), ref.download_blocks()
    finally:
        ref.close()
    for cut in (24, 29):  # right after an exchange period, and in the middle of one
        a = S.SlabDomain(sc, 3, steps=STEPS)
        try:
            a.step(cut)
            paths = a.checkpoint(str(tmp_path / f"ck{cut}"))
        finally:
            a.close()
        assert len(paths) == 3
        b = S.SlabDomain(sc, 3, steps=STEPS)
        try:
            b.restore(str(tmp_path / f"ck{cut}"))
            b.step(STEPS - cut)
            assert np.array_equal(b.fields().view(np.uint32), want.view(np.uint32))
            assert np.array_equal(b.download_blocks().view(np.uint32), want_blocks.view(np.uint32))
        finally:
            b.close()
