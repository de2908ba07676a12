"""Z-slab decomposition of one grid: one handle per slab, ghost blocks between.

The reference splits its grid into z slabs of whole blocks for its rayon
threads (src/engine.rs:8-13), all in one address space, each thread reading
its neighbours' planes directly.  Here a slab is a separate grid (on its own
GPU, or several on one GPU) that holds its own planes [z0, z1) plus a ghost
block of GHOST planes on each inner side, [lo, hi).

Why the ghost blocks stay exact for GHOST steps: H(k) reads E(k) and E(k+1),
E(k) reads H(k) and H(k-1).  A slab's outer ghost planes see zero fields
beyond [lo, hi) where the whole grid has real ones, so each step the wrong
values advance one plane inward from lo and from hi - 1.  After s steps the
planes [lo, lo + s) and [hi - s, hi) may be wrong; the owned planes read
the ghost planes next to them, z0 - 1 and z1, which stay exact while
s <= GHOST.  So every GHOST steps each slab receives both ghost blocks
(the six field components and the x and y CPML psi of those planes) from
its neighbours' owned planes, and runs GHOST more steps.  Sources on a
ghost plane are applied by both slabs that hold it (the ghost must evolve
exactly); probes only by the owner.

z CPML: the slab holding a real z-CPML layer gets the global profile sliced
to its planes, with the same thickness, so its other z side carries the
profile's interior values (b 1, a 0, 1/kappa 1): psi stays exactly +0 there
and the curl passes through unchanged.  `plan` keeps the real layer off
every ghost block, so z psi never has to move between slabs.

Transports: `SlabDomain` runs all slabs in one process on one device, each
on its own CUDA stream, moving ghost blocks with the pack/unpack kernels
through device staging buffers; `SlabRank` runs one slab per rank of a
torch.distributed group and moves ghost blocks with batched point-to-point
sends (NCCL over NVLink between GPUs).  FP32 storage only.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from .layout import GridDims, MaterialGrid, MaterialTable

GHOST = 8  # planes per ghost block, and steps between exchanges
_HARD_SHEET_X = 1  # WF_SRC_HARD_SHEET_X: writes every (y, z) of its plane x


@dataclass(frozen=True)
class Slab:
    index: int
    z0: int  # first owned plane of the whole grid
    z1: int  # one past the last owned plane
    lo: int  # first plane held (z0 - GHOST, or 0)
    hi: int  # one past the last plane held (z1 + GHOST, or nz)

    @property
    def nz(self) -> int:
        return self.hi - self.lo

    def owns(self, z: int) -> bool:
        return self.z0 <= z < self.z1

    def holds(self, z: int) -> bool:
        return self.lo <= z < self.hi


def plan(nz: int, parts: int, pml_z: int = 0) -> List[Slab]:
    """Splits nz planes into `parts` slabs of whole 8-plane blocks, the first
    nz/8 % parts slabs one block larger.  With more than one slab the first
    and last must own at least pml_z + GHOST planes, so that no ghost block
    reaches a real z-CPML plane."""
    if nz <= 0 or nz % 8:
        raise ValueError("nz must be a positive multiple of 8")
    blocks = nz // 8
    if parts < 1 or parts > blocks:
        raise ValueError(f"cannot split {blocks} z blocks into {parts} slabs")
    base, extra = divmod(blocks, parts)
    out, z = [], 0
    for i in range(parts):
        z1 = z + 8 * (base + (1 if i < extra else 0))
        out.append(Slab(i, z, z1, max(z - GHOST, 0), min(z1 + GHOST, nz)))
        z = z1
    if parts > 1 and pml_z > 0:
        for s in (out[0], out[-1]):
            if s.z1 - s.z0 < pml_z + GHOST:
                raise ValueError(f"slab {s.index} owns {s.z1 - s.z0} planes; with a {pml_z}-plane "
                                 f"z CPML the end slabs need at least {pml_z + GHOST}")
    return out


@dataclass
class SlabSpec:
    """Everything one slab's grid is loaded with, in slab coordinates."""
    slab: Slab
    dims: GridDims
    ids: Optional[np.ndarray]       # nz*ny*nx material ids, or None (scene window)
    scene_text: Optional[str]
    table: MaterialTable
    pml: list                       # per axis (thickness, b, a, inv_kappa) or None
    sources: list = field(default_factory=list)  # (x, y, z, comp, values, mode)
    probes: list = field(default_factory=list)   # (global index, x, y, z, comp, cos, sin, first, trace)


def slab_spec(sc, slab: Slab, steps: int) -> SlabSpec:
    """The slab's share of a Scenario: its planes of the material ids (or the
    scene text for a device window), the CPML profiles (x, y whole; z sliced),
    every source on a plane it holds (sheet sources everywhere) and every
    probe on a plane it owns, with tables for `steps` steps."""
    d = sc.dims
    dims = GridDims(d.nx, d.ny, slab.nz)
    ids = None
    if sc.grid is not None:
        plane = d.nx * d.ny
        ids = np.ascontiguousarray(sc.grid.ids[slab.lo * plane:slab.hi * plane])
    table = MaterialTable(np.array(sc.table.q16, np.int32, copy=True))
    pml = [None, None, None]
    if sc.pml is not None:
        for ax in range(3):
            p = sc.pml.profiles[ax]
            t = int(sc.pml.thickness_voxels[ax])
            if t == 0:
                continue
            if ax < 2:
                pml[ax] = (t, p.b, p.a, p.inv_kappa)
            elif slab.lo < t or slab.hi > d.nz - t:
                sl = slice(slab.lo, slab.hi)
                pml[ax] = (t, p.b[sl].copy(), p.a[sl].copy(), p.inv_kappa[sl].copy())
    spec = SlabSpec(slab, dims, ids, None if ids is not None else sc.scene_text, table, pml)
    for s in sc.sources:
        vals = s.values(sc.dt, steps)
        if s.mode == _HARD_SHEET_X:
            spec.sources.append((s.x, s.y, 0, int(s.component), vals, s.mode))
        elif slab.holds(s.z):
            spec.sources.append((s.x, s.y, s.z - slab.lo, int(s.component), vals, s.mode))
    for i, p in enumerate(sc.probes):
        if slab.owns(p.z):
            c, si = p.tables(sc.dt, steps)
            spec.probes.append((i, p.x, p.y, p.z - slab.lo, int(p.component), c, si,
                                p.first_step(sc.dt), bool(p.record_trace)))
    return spec


class DeviceSlabState:
    """A slab's grid on the device (DeviceFieldGrid) behind the interface the
    transports use: step, floats/pack/unpack of plane ranges into torch
    device tensors, owned fields and probe sums."""

    def __init__(self, spec: SlabSpec, nz_global: int, sc, stream: int, device: int = 0,
                 arith: str = "exact", kernel: str = "auto"):
        from .engine import DeviceFieldGrid
        self.spec = spec
        g = DeviceFieldGrid(spec.dims, arith=arith, kernel=kernel, device=device, stream=stream)
        self.grid = g
        if spec.ids is not None:
            g.set_materials(MaterialGrid(spec.dims, spec.ids), spec.table)
        else:
            g.set_scene_window(spec.scene_text, spec.table, sc.dt, sc.dx, nz_global,
                               spec.slab.lo)
        for ax, p in enumerate(spec.pml):
            if p is not None:
                g.set_pml_axis(ax, *p)
        for (x, y, z, comp, vals, mode) in spec.sources:
            g.add_source_values(x, y, z, comp, vals, mode)
        self.probe_index = {}
        for (gi, x, y, z, comp, c, si, first, trace) in spec.probes:
            self.probe_index[gi] = g.add_probe_tables(x, y, z, comp, c, si, first, trace)

    def step(self, n: int) -> None:
        self.grid.step(n)

    def floats(self, nplanes: int) -> int:
        return self.grid.slab_floats(nplanes)

    @staticmethod
    def _device_buffer(t):
        """(pointer, capacity in floats) of a contiguous float32 CUDA tensor."""
        import torch
        if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("slab buffers are contiguous float32 CUDA tensors")
        return t.data_ptr(), t.numel()

    def pack(self, z0: int, nplanes: int, out) -> None:
        self.grid.pack_planes(z0, nplanes, *self._device_buffer(out))

    def unpack(self, z0: int, nplanes: int, src) -> None:
        self.grid.unpack_planes(z0, nplanes, *self._device_buffer(src))

    def owned_fields(self) -> np.ndarray:
        s = self.spec.slab
        return self.grid.fields()[:, s.z0 - s.lo:s.z1 - s.lo]

    def probe_sums(self, global_index: int, nfreq: int):
        return self.grid.probe_sums(self.probe_index[global_index], nfreq)

    def owned_blocks(self) -> np.ndarray:
        """The owned planes in the reference's FieldBlock order
        (src/engine.rs:622-640): whole 8-plane block layers, so the slice of
        the slab's own block stream that the whole grid's stream holds at
        block layers [z0/8, z1/8)."""
        return owned_block_range(self.grid.download_blocks(), self.spec)

    def close(self) -> None:
        self.grid.close()


def owned_block_range(blocks: np.ndarray, spec: "SlabSpec") -> np.ndarray:
    """The owned block layers of a slab's FieldBlock stream (6 x 512 floats
    per block, blocks ordered (bz, by, bx))."""
    d, s = spec.dims, spec.slab
    per_layer = (d.nx // 8) * (d.ny // 8) * 6 * 512
    return blocks[(s.z0 - s.lo) // 8 * per_layer:(s.z1 - s.lo) // 8 * per_layer]


def _pml_z(sc) -> int:
    """The scenario's z-CPML thickness (0 without CPML)."""
    return int(sc.pml.thickness_voxels[2]) if sc.pml is not None else 0


class SlabDomain:
    """All slabs of a grid in this process on one device, each slab on a CUDA
    stream of its own so that the slabs' steps run concurrently.  step(n)
    runs every slab in lockstep, exchanging ghost blocks every GHOST steps
    through the pack/unpack kernels: a block is packed on its owner's stream
    into a staging buffer of its own, and the receiving slab's stream waits
    for that before unpacking (and the next pack into the buffer waits for
    the unpack).  `stream` is the domain's own stream: every step(n) starts
    after the work already on it and ends with it waiting for every slab, so
    events recorded on it bracket the domain's work.  fields() and
    probe_sums() read the owning slabs.  Results equal the whole grid's bit
    for bit."""

    def __init__(self, sc, parts: int, steps: Optional[int] = None, device: int = 0,
                 arith: str = "exact", kernel: str = "auto"):
        import torch
        self.sc = sc
        steps = sc.steps if steps is None else steps
        self.slabs = plan(sc.dims.nz, parts, _pml_z(sc))
        self._torch = torch
        self.stream = torch.cuda.Stream(device=device)
        self.streams = [torch.cuda.Stream(device=device) for _ in self.slabs]
        self.states = [DeviceSlabState(slab_spec(sc, s, steps), sc.dims.nz, sc,
                                       st.cuda_stream, device, arith, kernel)
                       for s, st in zip(self.slabs, self.streams)]
        for s in self.states:
            s.grid.set_graph_steps(GHOST)  # every step call is one exchange period
        n = self.states[0].floats(GHOST) if parts > 1 else 4
        with torch.cuda.stream(self.stream):
            # per neighbouring pair: [block moving down, block moving up]
            self._bufs = [[torch.empty(n, dtype=torch.float32, device=f"cuda:{device}")
                           for _ in range(2)] for _ in range(parts - 1)]
        self._unpacked = [[None, None] for _ in range(parts - 1)]
        self._since = 0  # steps since the last exchange
        self.exchanges = 0

    def _move(self, pair: int, way: int, src: int, z_src: int, dst: int, z_dst: int) -> None:
        torch = self._torch
        buf = self._bufs[pair][way]
        s_src, s_dst = self.streams[src], self.streams[dst]
        if self._unpacked[pair][way] is not None:  # the buffer's last unpack is done
            s_src.wait_event(self._unpacked[pair][way])
        self.states[src].pack(z_src, GHOST, buf)
        packed = torch.cuda.Event()
        packed.record(s_src)
        s_dst.wait_event(packed)
        self.states[dst].unpack(z_dst, GHOST, buf)
        done = torch.cuda.Event()
        done.record(s_dst)
        self._unpacked[pair][way] = done

    def exchange(self) -> None:
        """Refreshes every ghost block from its owner."""
        for i in range(len(self.states) - 1):
            sa, sb = self.slabs[i], self.slabs[i + 1]
            # i+1's lowest owned block -> i's upper ghost block
            self._move(i, 0, i + 1, sb.z0 - sb.lo, i, sa.z1 - sa.lo)
            # i's highest owned block -> i+1's lower ghost block
            self._move(i, 1, i, sa.z1 - GHOST - sa.lo, i + 1, 0)
        self.exchanges += 1

    def step(self, n: int = 1) -> None:
        torch = self._torch
        start = torch.cuda.Event()
        start.record(self.stream)
        for st in self.streams:
            st.wait_event(start)
        while n > 0:
            if self._since == GHOST:
                if len(self.states) > 1:
                    self.exchange()
                self._since = 0
            k = min(GHOST - self._since, n)
            for s in self.states:
                s.step(k)
            self._since += k
            n -= k
        for st in self.streams:
            ev = torch.cuda.Event()
            ev.record(st)
            self.stream.wait_event(ev)

    def sync(self) -> None:
        self.stream.synchronize()
        for st in self.streams:
            st.synchronize()
        for s in self.states:
            s.grid.sync()

    def fields(self) -> np.ndarray:
        self.sync()
        return np.concatenate([s.owned_fields() for s in self.states], axis=1)

    def probe_sums(self, p: int, nfreq: int):
        self.sync()
        for s in self.states:
            if p in s.probe_index:
                return s.probe_sums(p, nfreq)
        raise IndexError(f"no probe {p}")

    def download_blocks(self) -> np.ndarray:
        """The whole grid's snapshot in FieldBlock order: each slab's owned
        block layers, in slab order (the bytes wave_trajectory.bin holds)."""
        self.sync()
        return np.concatenate([s.owned_blocks() for s in self.states])

    def checkpoint(self, prefix: str) -> list:
        """Saves every slab's complete state (ghost blocks included) to
        `prefix`.slab<i> (wf_checkpoint_save); returns the paths."""
        self.sync()
        paths = [f"{prefix}.slab{i}" for i in range(len(self.states))]
        for st, path in zip(self.states, paths):
            st.grid.checkpoint(path)
        return paths

    def restore(self, prefix: str) -> None:
        """Loads the slabs saved by checkpoint(prefix) into this domain, which
        must be set up like the one that saved them.  The exchange phase
        follows from the step count: an exchange is due before every step
        whose index is a positive multiple of GHOST."""
        self.sync()
        for i, st in enumerate(self.states):
            st.grid.restore(f"{prefix}.slab{i}")
        done = self.states[0].grid.steps_done
        if any(st.grid.steps_done != done for st in self.states):
            raise ValueError("the slab checkpoints are from different steps")
        self._since = (done - 1) % GHOST + 1 if done > 0 else 0

    def close(self) -> None:
        self.sync()
        for s in self.states:
            s.close()
        self.states = []


class SlabRank:
    """This rank's slab of a grid split over the ranks of a torch.distributed
    group (one process per GPU).  step(n) exchanges ghost blocks with the two
    neighbouring ranks every GHOST steps through batched point-to-point
    sends and receives of packed device buffers; every rank calls step with
    the same n.  `make_state(spec)` builds the slab's state (default: a
    DeviceSlabState on the current CUDA device, on a stream of its own that
    the exchange's copies and communication are ordered on as well).

    With an NCCL group the packed device buffers travel as they are.  With
    another backend (gloo) a device slab's blocks are staged through pinned
    host buffers: packed on the device, copied to the host, sent, received,
    copied back and unpacked, all ordered on the slab's stream."""

    def __init__(self, sc, group=None, steps: Optional[int] = None,
                 make_state: Optional[Callable] = None, arith: str = "exact",
                 kernel: str = "auto"):
        import torch
        import torch.distributed as dist
        self._dist, self._torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        steps = sc.steps if steps is None else steps
        self.slabs = plan(sc.dims.nz, self.world, _pml_z(sc))
        self.slab = self.slabs[self.rank]
        spec = slab_spec(sc, self.slab, steps)
        self.stream = None
        if make_state is None:
            dev = torch.cuda.current_device()
            self.stream = torch.cuda.Stream(dev)
            self.state = DeviceSlabState(spec, sc.dims.nz, sc, self.stream.cuda_stream, dev,
                                         arith, kernel)
            self.state.grid.set_graph_steps(GHOST)  # every step call is one exchange period
            where = torch.device("cuda", dev)
        else:
            self.state = make_state(spec)
            where = torch.device("cpu")
        n = self.state.floats(GHOST)
        with self._on_stream():
            self._bufs = [torch.empty(n, dtype=torch.float32, device=where) for _ in range(4)]
        # host staging for a device slab in a group whose backend is not NCCL
        self._host = None
        if where.type == "cuda" and dist.get_backend(group) != "nccl":
            self._host = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(4)]
        self._since = 0
        self.exchanges = 0

    def _on_stream(self):
        """Makes the slab's stream torch's current stream (a device slab), so
        that torch copies and NCCL calls are ordered with its kernels."""
        import contextlib
        return self._torch.cuda.stream(self.stream) if self.stream is not None \
            else contextlib.nullcontext()

    def _peer(self, r: int) -> int:
        return r if self.group is None else self._dist.get_global_rank(self.group, r)

    def exchange(self) -> None:
        with self._on_stream():
            self._exchange()
        self.exchanges += 1

    def _exchange(self) -> None:
        dist, s = self._dist, self.slab
        send_lo, recv_lo, send_hi, recv_hi = self._bufs
        wire = self._host or self._bufs  # what travels: device or pinned host buffers
        lower, upper = self.rank > 0, self.rank < self.world - 1
        if lower:
            self.state.pack(s.z0 - s.lo, GHOST, send_lo)
        if upper:
            self.state.pack(s.z1 - GHOST - s.lo, GHOST, send_hi)
        if self._host:  # device -> host on the slab's stream, then wait for it
            for k, on in ((0, lower), (2, upper)):
                if on:
                    wire[k].copy_(self._bufs[k], non_blocking=True)
            self.stream.synchronize()
        ops = []
        if lower:
            ops += [dist.P2POp(dist.isend, wire[0], self._peer(self.rank - 1), self.group),
                    dist.P2POp(dist.irecv, wire[1], self._peer(self.rank - 1), self.group)]
        if upper:
            ops += [dist.P2POp(dist.isend, wire[2], self._peer(self.rank + 1), self.group),
                    dist.P2POp(dist.irecv, wire[3], self._peer(self.rank + 1), self.group)]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if self._host:  # host -> device, ordered before the unpacks on the same stream
            for k, on in ((1, lower), (3, upper)):
                if on:
                    self._bufs[k].copy_(wire[k], non_blocking=True)
        if lower:
            self.state.unpack(0, GHOST, recv_lo)
        if upper:
            self.state.unpack(s.z1 - s.lo, GHOST, recv_hi)

    def step(self, n: int = 1) -> None:
        while n > 0:
            if self._since == GHOST:
                if self.world > 1:
                    self.exchange()
                self._since = 0
            k = min(GHOST - self._since, n)
            self.state.step(k)
            self._since += k
            n -= k

    def gather_fields(self, dst: int = 0) -> Optional[np.ndarray]:
        """The whole grid's fields on rank `dst` (None elsewhere)."""
        part = self.state.owned_fields()
        got = [None] * self.world if self.rank == dst else None
        self._dist.gather_object(part, got, dst=self._peer(dst), group=self.group)
        return np.concatenate(got, axis=1) if self.rank == dst else None

    def gather_blocks(self, dst: int = 0) -> Optional[np.ndarray]:
        """The whole grid's snapshot in FieldBlock order on rank `dst` (None
        elsewhere)."""
        part = self.state.owned_blocks()
        got = [None] * self.world if self.rank == dst else None
        self._dist.gather_object(part, got, dst=self._peer(dst), group=self.group)
        return np.concatenate(got) if self.rank == dst else None

    def gather_probe_sums(self, nfreq: int, dst: int = 0) -> Optional[dict]:
        """{global probe index: (cos sums, sin sums, samples)} on rank `dst`."""
        mine = {p: self.state.probe_sums(p, nfreq) for p in self.state.probe_index}
        got = [None] * self.world if self.rank == dst else None
        self._dist.gather_object(mine, got, dst=self._peer(dst), group=self.group)
        if self.rank != dst:
            return None
        out = {}
        for d in got:
            out.update(d)
        return out

    def close(self) -> None:
        self.state.close()
