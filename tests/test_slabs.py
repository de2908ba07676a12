"""CPU: the z-slab decomposition's plan, per-slab setup and rank exchange.

`plan` and `slab_spec` are host logic.  The exchange runs as gloo process
groups of 2 and 3 ranks; each rank's slab state is the oracle (the oracle
restates the reference's step, so the decomposition is checked against the
whole grid stepped by the same oracle): fields and probe sums of the
decomposed run must equal the whole grid's bit for bit.  The device
transport (pack/unpack kernels, one process) is covered by
test_gpu_slabs.py.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from wavefront_b200 import slabs as S  # noqa: E402
from wavefront_b200.configs import Scenario, courant_dt, two_spheres  # noqa: E402
from wavefront_b200.layout import (GridDims, MaterialGrid, MaterialTable, PmlConfig,  # noqa: E402
                                   PmlContext)
from wavefront_b200.probe import FieldComponent as PC  # noqa: E402
from wavefront_b200.probe import Probe  # noqa: E402
from wavefront_b200.scene import Scene  # noqa: E402
from wavefront_b200.source import FieldComponent, Source, default_waveform  # noqa: E402

STEPS = 29  # three exchanges and a partial period


def test_plan_splits_whole_blocks_with_ghosts():
    p = S.plan(512, 3, pml_z=16)
    assert [(s.z0, s.z1) for s in p] == [(0, 176), (176, 344), (344, 512)]
    assert [(s.lo, s.hi) for s in p] == [(0, 184), (168, 352), (336, 512)]
    assert all(s.nz % 8 == 0 for s in p)
    one = S.plan(64, 1, pml_z=16)[0]
    assert (one.z0, one.z1, one.lo, one.hi) == (0, 64, 0, 64)
    assert S.plan(64, 8)[3].owns(24) and S.plan(64, 8)[3].holds(16)


@pytest.mark.parametrize("nz,parts,pml", [(60, 2, 0), (64, 9, 0), (64, 0, 0), (64, 4, 16)])
def test_plan_rejects_bad_splits(nz, parts, pml):
    with pytest.raises(ValueError):
        S.plan(nz, parts, pml_z=pml)


def _scenario(nx=16, nz=64, pml=8, steps=STEPS):
    """Small z-CPML-only scene whose box, sources and probes straddle the slab
    boundaries of 2- and 3-way plans (ghost-plane source at z = 30)."""
    dims = GridDims(nx, nx, nz)
    dx = 1.0e-3
    dt = courant_dt(dx)
    f = float(np.float32(299792458.0 / (12.0 * dx)))
    grid = MaterialGrid(dims)
    table = MaterialTable.vacuum_filled(dt, dx)
    Scene.parse("box 3.0 1.0 0.001 2 3 20 13 12 45\n").voxelize(grid, table, dt, dx)
    cpml = PmlContext.build_exact(dims, PmlConfig(thickness=pml), dt, dx, axes=(False, False, True))
    srcs = [Source(8, 8, 30, FieldComponent.Ez, 1.0, default_waveform("ricker", f)),
            Source(5, 9, 12, FieldComponent.Ex, -0.5, default_waveform("gaussian", f))]
    probes = [Probe(8, 8, 33, PC.Ez, [f], 0.0), Probe(4, 4, 5, PC.Hy, [f, 2 * f], 0.0),
              Probe(9, 7, 23, PC.Ex, [f], 0.0)]
    return Scenario("slab_test", dims, dx, dt, grid, table, cpml, srcs, probes, steps)


def test_slab_spec_routes_sources_probes_and_z_cpml():
    sc = _scenario()
    p = S.plan(64, 2, pml_z=8)
    a, b = (S.slab_spec(sc, s, STEPS) for s in p)
    # z = 30 is owned by slab 0 and is in slab 1's lower ghost block [24, 32)
    assert [src[2] for src in a.sources] == [30, 12]
    assert [src[2] for src in b.sources] == [30 - 24]
    assert [pr[0] for pr in a.probes] == [1, 2] and [pr[0] for pr in b.probes] == [0]
    assert a.pml[0] is None and a.pml[1] is None
    t, bb, aa, kk = a.pml[2]
    assert t == 8 and len(bb) == a.dims.nz
    np.testing.assert_array_equal(bb, sc.pml.profiles[2].b[0:40])
    np.testing.assert_array_equal(kk[-8:], np.ones(8, np.float32))  # interior values
    np.testing.assert_array_equal(b.pml[2][1], sc.pml.profiles[2].b[24:64])
    assert a.ids.size == 16 * 16 * 40
    mid = S.slab_spec(sc, S.plan(64, 3, pml_z=8)[1], STEPS)
    assert mid.pml[2] is None  # middle slab: no z CPML


def test_slab_spec_sheet_source_reaches_every_slab():
    sc = _scenario()
    sc.sources.append(Source(3, 0, 0, FieldComponent.Ez, 1.0, default_waveform("sinusoid", 1e10),
                             mode=1))
    for s in S.plan(64, 3, pml_z=8):
        spec = S.slab_spec(sc, s, 4)
        assert spec.sources[-1][5] == 1 and spec.sources[-1][2] == 0


class OracleSlabState:
    """A slab stepped by the oracle, with the state interface SlabRank uses
    (the packed layout here is the six field components only: the test
    scene has no x or y CPML)."""

    def __init__(self, spec):
        import torch
        from oracle import oracle as O
        self.torch = torch
        d = spec.dims
        self.spec = spec
        self.sim = O.Sim(d.nx, d.ny, d.nz, spec.ids, spec.table.q16)
        profs, shell = [None] * 3, [0, 0, 0]
        for ax, p in enumerate(spec.pml):
            if p is not None:
                profs[ax] = p[1:]
                shell[ax] = (p[0] + 7) // 8
        if any(shell):
            self.sim.set_pml(profs, shell)
        for (x, y, z, comp, vals, mode) in spec.sources:
            self.sim.add_source(x, y, z, comp, vals, mode)
        self.probe_index = {}
        for k, (gi, x, y, z, comp, c, si, first, trace) in enumerate(spec.probes):
            self.sim.add_probe(x, y, z, comp, c, si, c.shape[0], first, trace)
            self.probe_index[gi] = k

    def step(self, n):
        self.sim.step(n)

    def floats(self, nplanes):
        return 6 * nplanes * self.spec.dims.ny * self.spec.dims.nx

    def pack(self, z0, n, out):
        f = self.sim.fields()
        out.copy_(self.torch.from_numpy(np.ascontiguousarray(f[:, z0:z0 + n]).ravel()))

    def unpack(self, z0, n, src):
        f = self.sim.fields()
        d = self.spec.dims
        f[:, z0:z0 + n] = src.numpy().reshape(6, n, d.ny, d.nx)
        self.sim.set_fields(f)

    def owned_fields(self):
        s = self.spec.slab
        return self.sim.fields()[:, s.z0 - s.lo:s.z1 - s.lo]

    def probe_sums(self, gi, nfreq):
        return self.sim.probe_sums(self.probe_index[gi], nfreq)

    def owned_blocks(self):
        return S.owned_block_range(self.sim.blocks(), self.spec)

    def close(self):
        self.sim.close()


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        sc = _scenario()
        r = S.SlabRank(sc, make_state=OracleSlabState)
        r.step(5)
        r.step(STEPS - 5)  # the exchange period carries across calls
        f = r.gather_fields()
        blk = r.gather_blocks()
        pr = r.gather_probe_sums(2)
        if rank == 0:
            np.savez(out, fields=f, blocks=blk, exchanges=r.exchanges,
                     **{f"p{k}_{i}": v[i] for k, v in pr.items() for i in range(2)},
                     **{f"n{k}": v[2] for k, v in pr.items()})
        r.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_equal_the_whole_grid(oracle, tmp_path, world):
    import torch.multiprocessing as mp
    out = str(tmp_path / "slabs.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world,
                       start_method="spawn", join=True)
    got = np.load(out)
    sc = _scenario()
    whole = oracle.Sim(16, 16, 64, sc.grid.ids, sc.table.q16)
    p = sc.pml.profiles[2]
    whole.set_pml([None, None, (p.b, p.a, p.inv_kappa)], [0, 0, 1])
    for s in sc.sources:
        whole.add_source(s.x, s.y, s.z, int(s.component), s.values(sc.dt, STEPS), s.mode)
    for pb in sc.probes:
        c, si = pb.tables(sc.dt, STEPS)
        whole.add_probe(pb.x, pb.y, pb.z, int(pb.component), c, si, STEPS, pb.first_step(sc.dt))
    whole.step(STEPS)
    ref = whole.fields()
    assert np.abs(ref).max() > 0
    assert int(got["exchanges"]) == 3
    np.testing.assert_array_equal(got["fields"].view(np.uint32), ref.view(np.uint32))
    # the snapshot assembled from the slabs' owned block layers is the whole grid's
    np.testing.assert_array_equal(got["blocks"].view(np.uint32), whole.blocks().view(np.uint32))
    for k, pb in enumerate(sc.probes):
        nf = len(pb.frequencies_hz)
        c, si, n = whole.probe_sums(k, nf)
        assert int(got[f"n{k}"]) == n == STEPS
        np.testing.assert_array_equal(got[f"p{k}_0"][:nf], c)
        np.testing.assert_array_equal(got[f"p{k}_1"][:nf], si)


def test_two_spheres_plan_keeps_cpml_off_ghosts():
    sc = two_spheres(128, steps=8)
    for parts in (2, 3, 4):
        for s in S.plan(128, parts, 16):
            spec = S.slab_spec(sc, s, 8)
            if spec.pml[2] is not None:
                t = spec.pml[2][0]
                k = spec.pml[2][3]
                # the ghost planes carry the profile's interior values
                ghost = slice(0, s.z0 - s.lo) if s.lo > 0 else slice(s.z1 - s.lo, s.nz)
                np.testing.assert_array_equal(k[ghost], 1.0)
                assert t == 16


def test_plan_properties_over_random_splits():
    """Every plan covers [0, nz) with disjoint owned ranges of whole blocks,
    holds at most GHOST planes beyond them on each inner side, keeps every
    held range inside the grid, and keeps the z CPML off all ghost blocks."""
    rng = np.random.default_rng(7)
    checked = 0
    for _ in range(400):
        nz = 8 * int(rng.integers(1, 160))
        parts = int(rng.integers(1, 12))
        t = int(rng.choice([0, 8, 10, 16, 32]))
        try:
            p = S.plan(nz, parts, pml_z=t)
        except ValueError:
            continue
        checked += 1
        assert p[0].z0 == 0 and p[-1].z1 == nz
        for a, b in zip(p, p[1:]):
            assert a.z1 == b.z0
        for s in p:
            assert s.z0 % 8 == 0 and s.z1 % 8 == 0 and s.z1 - s.z0 >= 8
            assert s.lo == max(s.z0 - S.GHOST, 0) and s.hi == min(s.z1 + S.GHOST, nz)
            assert 0 <= s.lo and s.hi <= nz and s.nz % 8 == 0
            if len(p) > 1 and t:
                for z in list(range(s.lo, s.z0)) + list(range(s.z1, s.hi)):
                    assert t <= z < nz - t  # a ghost plane is never a real z-CPML plane
    assert checked > 200
