"""The learned thin-CPML boundary closure: data, training and use.

A grid with a thin CPML (4 cells) reflects more than one with a thick CPML
(16 cells).  The closure is a per-face 3-layer 3D conv network (3x3x3
kernels, 10 -> 16 -> 16 -> 6 channels, GELU, no bias, bfloat16 weights, FP32
accumulation) that reads the 8-cell band next to each face -- the six fields
and the four psi terms of the face's normal axis -- after every step kernel
and adds a correction to the band's fields (wf_set_closure).

Training data come from plain thick-CPML runs ("teachers", 64^3 with a
16-cell CPML, random Ricker or Gaussian sources, random dielectric
inclusions eps_r U[1,6]).  At sampled steps the teacher's state is
restricted to a thin-CPML "student" (40^3: the teacher's 32^3 interior plus
4 cells on each side, wf_restrict_state), the student takes one step, and
the teacher's next state, restricted the same way, minus the student's is
the correction the network learns (teacher forcing on one step).  The
network's forward and backward passes and the Adam updates run in the
library's own CUDA kernels (wf_nn_*); torch only allocates device memory.

The plain CPML stays the fallback (no closure set) and the judge of the
closure's reflection error (reflection_test).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _lib as _L
from .configs import C0, courant_dt
from .engine import DeviceFieldGrid
from .layout import GridDims, MaterialGrid, MaterialTable, PmlConfig, PmlContext
from .probe import FieldComponent as PC
from .scene import Scene
from .source import FieldComponent, default_waveform

ETA0 = 376.730313668  # free-space impedance: H-side values are scaled by it
BAND = 8
CHANNELS = [(10, 16), (16, 16), (16, 6)]  # (cin, cout) per layer
TEACHER_N, STUDENT_N, OFFSET = 64, 40, 12
THICK, THIN = 16, 4


def _torch():
    import torch
    return torch


def _p(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _chk(st: int):
    _L.check(st)


class ClosureNet:
    """Per-face weights on the device: FP32 masters, bfloat16 copies (what
    the forward pass and wf_set_closure read) and Adam moments."""

    def __init__(self, device: int = 0, seed: int = 0, gain_e: float = 1.0, gain_h: float = ETA0):
        torch = _torch()
        g = torch.Generator().manual_seed(seed)
        self.dev = torch.device("cuda", device)
        self.w, self.wb, self.m1, self.m2, self.dw = [], [], [], [], []
        for layer, (ci, co) in enumerate(CHANNELS):
            scale = math.sqrt(2.0 / (ci * 27)) * (0.01 if layer == 2 else 1.0)
            w = (torch.randn(6, co, ci, 27, generator=g) * scale).to(self.dev)
            self.w.append(w)
            self.wb.append(w.to(torch.bfloat16))
            self.m1.append(torch.zeros_like(w))
            self.m2.append(torch.zeros_like(w))
            self.dw.append(torch.zeros_like(w))
        self.t = 0
        self.gain_e, self.gain_h = gain_e, gain_h

    def _stream(self):
        return C.c_void_p(_torch().cuda.current_stream(self.dev).cuda_stream)

    def forward(self, x, face):
        """x [n][10][8][h][w] -> (y [n][6][8][h][w], cache for backward)."""
        torch = _torch()
        n, _, D, H, W = x.shape
        zs, acts = [], [x]
        a = x
        for layer, (ci, co) in enumerate(CHANNELS):
            last = layer == len(CHANNELS) - 1
            out = torch.empty(n, co, D, H, W, device=self.dev)
            z = None if last else torch.empty_like(out)
            _chk(_L.lib().wf_nn_conv3d_forward(_p(a), _p(self.wb[layer]), _p(face),
                                               _p(z) if z is not None else None, _p(out),
                                               n, ci, co, D, H, W, 0 if last else 1, self._stream()))
            zs.append(z)
            acts.append(out)
            a = out
        return a, (zs, acts, face)

    def backward(self, dy, cache):
        """Accumulates the weight gradients of dy into self.dw (zeroed first)."""
        torch = _torch()
        zs, acts, face = cache
        for d in self.dw:
            d.zero_()
        g = dy
        for layer in range(len(CHANNELS) - 1, -1, -1):
            ci, co = CHANNELS[layer]
            x = acts[layer]
            n, _, D, H, W = x.shape
            _chk(_L.lib().wf_nn_conv3d_backward_weight(_p(x), _p(g), _p(face), _p(self.dw[layer]),
                                                       n, ci, co, D, H, W, 6, self._stream()))
            if layer == 0:
                break
            dx = torch.empty(n, ci, D, H, W, device=self.dev)
            _chk(_L.lib().wf_nn_conv3d_backward_data(_p(g), _p(self.wb[layer]), _p(face), _p(dx),
                                                     n, ci, co, D, H, W, self._stream()))
            dz = torch.empty_like(dx)
            _chk(_L.lib().wf_nn_gelu_backward(_p(dx), _p(zs[layer - 1]), _p(dz), dx.numel(),
                                              self._stream()))
            g = dz

    def loss_grad(self, y, t):
        torch = _torch()
        dy = torch.empty_like(y)
        loss = torch.zeros(1, device=self.dev)
        _chk(_L.lib().wf_nn_mse(_p(y), _p(t), _p(dy), _p(loss), y.numel(), self._stream()))
        return loss, dy

    def adam_step(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.t += 1
        for w, wb, g, m1, m2 in zip(self.w, self.wb, self.dw, self.m1, self.m2):
            _chk(_L.lib().wf_nn_adam(_p(w), _p(wb), _p(g), _p(m1), _p(m2), w.numel(), lr, b1, b2, eps,
                                     self.t, self._stream()))

    def train_step(self, x, t, face, lr: float = 1e-3) -> float:
        y, cache = self.forward(x, face)
        loss, dy = self.loss_grad(y, t)
        self.backward(dy, cache)
        self.adam_step(lr)
        return loss

    def attach(self, grid: DeviceFieldGrid, alpha: float = 1.0, guard: bool = False):
        """The network as grid's closure (applied after every step kernel),
        its correction scaled by alpha (folded into the last layer); guard
        scales each face's correction so that it cannot raise the band's
        energy (wf_set_closure_guard)."""
        torch = _torch()
        w3 = self.wb[2] if alpha == 1.0 else (self.w[2] * alpha).to(torch.bfloat16)
        _chk(_L.lib().wf_set_closure(grid._h, _p(self.wb[0]), _p(self.wb[1]), _p(w3),
                                     self.gain_e, self.gain_h))
        _chk(_L.lib().wf_set_closure_guard(grid._h, 1 if guard else 0))

    @staticmethod
    def detach(grid: DeviceFieldGrid):
        _chk(_L.lib().wf_set_closure(grid._h, None, None, None, 1.0, 1.0))

    def state(self) -> dict:
        return {"w": [w.cpu().numpy() for w in self.w], "gain_e": self.gain_e,
                "gain_h": self.gain_h, "t": self.t}

    def load_state(self, st: dict):
        torch = _torch()
        for k, w in enumerate(st["w"]):
            self.w[k].copy_(torch.from_numpy(np.asarray(w, np.float32)))
            self.wb[k].copy_(self.w[k].to(torch.bfloat16))
        self.gain_e, self.gain_h, self.t = st["gain_e"], st["gain_h"], st["t"]


# ---- training data --------------------------------------------------------------


@dataclass
class Run:
    text: str
    comp: int
    kind: str
    freq: float
    src: tuple


def random_run(rng: np.random.Generator, dx: float) -> Run:
    """One teacher run: 1-3 dielectric inclusions (eps_r U[1,6]) and a Ricker
    or Gaussian source (15-30 cells per wavelength) inside the student's
    interior; the source stays out of the 8-cell bands (the student has no
    source, so a source inside a band would put its injection into the
    residual the network learns)."""
    lines = []
    lo, hi = OFFSET + THIN + 2, TEACHER_N - OFFSET - THIN - 2
    slo, shi = OFFSET + BAND + 1, TEACHER_N - OFFSET - BAND - 1
    for _ in range(int(rng.integers(1, 4))):
        eps = rng.uniform(1.0, 6.0)
        c = rng.uniform(lo, hi, 3)
        if rng.random() < 0.5:
            lines.append(f"sphere {eps:.5f} 1.0 0.0 {c[0]:.3f} {c[1]:.3f} {c[2]:.3f} "
                         f"{rng.uniform(2.0, 8.0):.3f}")
        else:
            e = rng.uniform(3.0, 12.0, 3)
            lines.append(f"box {eps:.5f} 1.0 0.0 {c[0]:.3f} {c[1]:.3f} {c[2]:.3f} "
                         f"{c[0] + e[0]:.3f} {c[1] + e[1]:.3f} {c[2] + e[2]:.3f}")
    f = float(np.float32(C0 / (rng.uniform(15.0, 30.0) * dx)))
    src = tuple(int(v) for v in rng.integers(slo, shi, 3))
    return Run("\n".join(lines) + "\n", int(rng.integers(0, 3)), str(rng.choice(["ricker", "gaussian"])),
               f, src)


def truncated_profiles(n: int, dt: float, dx: float):
    """The thin layer's CPML: on each axis of an n-cell grid, the THIN cells
    next to each face carry the innermost THIN cells of the THICK-cell
    grading of the grid (n + 2 (THICK - THIN)) that the thin grid is the
    interior of; identity (b=1, a=0, 1/kappa=1) elsewhere.  The closure then
    stands in for the missing outer THICK - THIN cells."""
    cut = THICK - THIN
    nt = n + 2 * cut
    ctx = PmlContext.build_exact(GridDims(nt, nt, nt), PmlConfig(thickness=THICK), dt, dx)
    out = []
    for ax in range(3):
        p = ctx.profiles[ax]
        out.append(tuple(np.ascontiguousarray(v[cut:cut + n], np.float32)
                         for v in (p.b, p.a, p.inv_kappa)))
    return out


def graded_profiles(n: int, dt: float, dx: float):
    """The plain thin CPML: a THIN-cell layer graded over its own THIN cells
    (PmlContext::build's grading, src/layout.rs:471-513, per cell)."""
    ctx = PmlContext.build_exact(GridDims(n, n, n), PmlConfig(thickness=THIN), dt, dx)
    return [tuple(np.ascontiguousarray(v, np.float32) for v in (p.b, p.a, p.inv_kappa))
            for p in ctx.profiles]


def set_thin_cpml(grid: DeviceFieldGrid, dt: float, dx: float, profile: str = "truncated"):
    """The thin layer on every face: "truncated" (the innermost THIN cells of
    the THICK grading) or "graded" (a plain THIN-cell CPML)."""
    n = grid.dims.nx
    profs = truncated_profiles(n, dt, dx) if profile == "truncated" else graded_profiles(n, dt, dx)
    for ax, (b, a, ik) in enumerate(profs):
        grid.set_pml_axis(ax, THIN, b, a, ik)


def _grids(run: Run, dx: float, dt: float, steps: int, device: int, profile: str = "truncated"):
    tdims, sdims = GridDims(TEACHER_N, TEACHER_N, TEACHER_N), GridDims(STUDENT_N, STUDENT_N, STUDENT_N)
    tgrid = MaterialGrid(tdims)
    table = MaterialTable.vacuum_filled(dt, dx)
    Scene.parse(run.text).voxelize(tgrid, table, dt, dx)
    ids = tgrid.ids.reshape(TEACHER_N, TEACHER_N, TEACHER_N)
    sl = slice(OFFSET, OFFSET + STUDENT_N)
    sgrid = MaterialGrid(sdims, ids[sl, sl, sl].copy())
    teacher = DeviceFieldGrid(tdims, kernel="fused", device=device)
    teacher.set_materials(tgrid, table)
    teacher.set_pml(PmlContext.build_exact(tdims, PmlConfig(thickness=THICK), dt, dx))
    wf = default_waveform(run.kind, run.freq)
    from .source import Source
    s = Source(run.src[0], run.src[1], run.src[2], FieldComponent(run.comp), 1.0, wf)
    teacher.add_source_values(s.x, s.y, s.z, s.component, s.values(dt, steps))
    students = []
    for _ in range(2):
        st = DeviceFieldGrid(sdims, kernel="fused", device=device)
        st.set_materials(sgrid, table)
        set_thin_cpml(st, dt, dx, profile)
        students.append(st)
    return teacher, students


def generate(n_runs: int, steps: int = 160, first: int = 30, every: int = 10, crop: int = 16,
             seed: int = 1, device: int = 0, net: Optional["ClosureNet"] = None, max_lead: int = 12,
             guard: bool = False, profile: str = "truncated"):
    """Teacher-forced one-step samples: returns (X [M][10][8][c][c],
    R [M][6][8][c][c], face [M] int32, 1.0) on the device.  H-side values
    are times ETA0, and every sample is divided by the RMS of the E channels
    of its whole face band -- the normalization the closure applies at run
    time.  One random c x c crop per face and sampled step.

    With `net`, each sample is taken after the student has run a random
    1..max_lead steps with `net` as its closure from the teacher's state
    (the last of them without the closure, whose input is the sample): the
    target is the teacher's state at the same time, so the network also
    learns to pull a drifting student back (a DAgger-style round).  guard
    runs those closure steps with the energy guard on.  profile is the
    student's thin layer (set_thin_cpml)."""
    torch = _torch()
    dev = torch.device("cuda", device)
    rng = np.random.default_rng(seed)
    dx = 1.0e-3
    dt = courant_dt(dx)
    n = STUDENT_N
    band = torch.empty(6, 10, BAND, n, n, device=dev)
    band2 = torch.empty_like(band)
    xs, rs, fs = [], [], []
    for _ in range(n_runs):
        run = random_run(rng, dx)
        teacher, (s1, s2) = _grids(run, dx, dt, steps + 1, device, profile)
        try:
            done = 0
            for k in range(first, steps, every):
                lead = int(rng.integers(1, max_lead + 1)) if net is not None else 1
                lead = min(lead, k - done + 1)  # the teacher cannot step back
                teacher.step(k - lead + 1 - done)
                done = k - lead + 1
                _chk(_L.lib().wf_restrict_state(teacher._h, s1._h, OFFSET))
                if lead > 1:
                    net.attach(s1, guard=guard)
                    for _ in range(lead - 1):
                        s1.step(1)
                        teacher.step(1)
                        done += 1
                    ClosureNet.detach(s1)
                s1.step(1)
                teacher.step(1)
                done += 1
                _chk(_L.lib().wf_restrict_state(teacher._h, s2._h, OFFSET))
                _chk(_L.lib().wf_band_gather(s1._h, _p(band), 1.0, ETA0))
                _chk(_L.lib().wf_band_gather(s2._h, _p(band2), 1.0, ETA0))
                s1.sync()
                s2.sync()
                for f in range(6):
                    sf = float(torch.sqrt(torch.mean(band[f, :3] ** 2)).item()) + 1e-30
                    u0, v0 = (int(v) for v in rng.integers(0, n - crop + 1, 2))
                    xs.append(band[f, :, :, u0:u0 + crop, v0:v0 + crop] / sf)
                    rs.append((band2[f, :6, :, u0:u0 + crop, v0:v0 + crop]
                               - band[f, :6, :, u0:u0 + crop, v0:v0 + crop]) / sf)
                    fs.append(f)
        finally:
            teacher.close()
            s1.close()
            s2.close()
    X = torch.stack(xs)
    R = torch.stack(rs)
    F = torch.tensor(fs, dtype=torch.int32, device=dev)
    return X, R, F, 1.0


def train(X, R, F, rms: float, iters: int = 3000, batch: int = 64, lr: float = 3e-4,
          seed: int = 0, device: int = 0, log_every: int = 0, net: Optional[ClosureNet] = None):
    """Adam on the MSE of the predicted correction, targets normalized to
    unit RMS during training (the scale is folded into the last layer
    afterwards), learning rate on a cosine from lr to lr/30; returns (net,
    [(iteration, loss on normalized targets)])."""
    torch = _torch()
    r_scale = float(torch.sqrt(torch.mean(R * R)).item()) or 1.0
    if net is None:
        net = ClosureNet(device=device, seed=seed, gain_e=1.0 / rms, gain_h=ETA0 / rms)
    else:  # continue: back to the normalized-target units of training
        net.w[2].div_(r_scale)
        net.wb[2].copy_(net.w[2].to(torch.bfloat16))
    Rn = R / r_scale
    g = torch.Generator(device=X.device).manual_seed(seed)
    losses = []
    for it in range(iters):
        lr_it = lr / 30.0 + 0.5 * (lr - lr / 30.0) * (1.0 + math.cos(math.pi * it / max(iters - 1, 1)))
        idx = torch.randint(0, X.shape[0], (batch,), generator=g, device=X.device)
        loss = net.train_step(X[idx].contiguous(), Rn[idx].contiguous(), F[idx].contiguous(), lr_it)
        if log_every and (it % log_every == 0 or it == iters - 1):
            losses.append((it, float(loss.item())))
    net.w[2].mul_(r_scale)
    net.wb[2].copy_(net.w[2].to(torch.bfloat16))
    return net, losses


def residual_loss(net: Optional[ClosureNet], X, R, F, batch: int = 256) -> float:
    """Mean squared residual left after the net's correction (no net: R itself)."""
    torch = _torch()
    tot, cnt = 0.0, 0
    for i in range(0, X.shape[0], batch):
        r = R[i:i + batch]
        if net is not None:
            y, _ = net.forward(X[i:i + batch].contiguous(), F[i:i + batch].contiguous())
            r = r - y
        tot += float(torch.sum(r * r).item())
        cnt += r.numel()
    return tot / cnt


# ---- evaluation -------------------------------------------------------------------


def reflection_test(interior: int = 48, steps: int = 260, net: Optional[ClosureNet] = None,
                    cpml: int = THIN, device: int = 0, seed: int = 3, alpha: float = 1.0,
                    truncated: bool = False, guard: bool = False) -> dict:
    """Reflection of the boundary of an interior^3 region with a `cpml`-cell
    CPML (plus `net` as its closure), against a reference run in a domain
    large enough that nothing returns within `steps`: a Ricker Ez source
    (20 cells per wavelength) off-centre, Ez traces recorded 3 cells inside
    the interior next to three faces, an edge and a corner.  Returns the max
    over probes of max_t |trace - reference| / max_t |reference| and the
    traces' relative L2."""
    dx = 1.0e-3
    dt = courant_dt(dx)
    f = float(np.float32(C0 / (20.0 * dx)))
    wf = default_waveform("ricker", f)
    rng = np.random.default_rng(seed)
    src_i = tuple(int(v) for v in (interior // 2 + rng.integers(-3, 4, 3)))
    probes_i = [(3, interior // 2, interior // 2), (interior // 2, interior - 4, interior // 2),
                (interior // 2, interior // 2, 3), (3, 3, interior // 2), (3, 3, 3)]
    margin = int(math.ceil(steps * 0.58)) + 8
    from .source import Source

    def run(n_total: int, off: int, pml, closure: bool):
        dims = GridDims(n_total, n_total, n_total)
        g = DeviceFieldGrid(dims, kernel="fused", device=device)
        try:
            g.set_materials(MaterialGrid(dims), MaterialTable.vacuum_filled(dt, dx))
            if pml == "truncated":
                set_thin_cpml(g, dt, dx)
            elif pml is not None:
                g.set_pml(pml)
            s = Source(src_i[0] + off, src_i[1] + off, src_i[2] + off, FieldComponent.Ez, 1.0, wf)
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(dt, steps))
            for p in probes_i:
                g.add_probe_tables(p[0] + off, p[1] + off, p[2] + off, PC.Ez,
                                   np.zeros((steps, 0)), np.zeros((steps, 0)), 0, record_trace=True)
            if closure:
                net.attach(g, alpha, guard)
            g.step(steps)
            g.sync()
            return np.stack([g.probe_trace(i, steps) for i in range(len(probes_i))]).astype(np.float64)
        finally:
            g.close()

    n_ref = interior + 2 * margin
    n_ref += (-n_ref) % 8
    ref = run(n_ref, margin, None, False)
    n_b = interior + 2 * cpml
    n_b += (-n_b) % 8
    dims_b = GridDims(n_b, n_b, n_b)
    pml = "truncated" if truncated else PmlContext.build_exact(dims_b, PmlConfig(thickness=cpml), dt, dx)
    got = run(n_b, cpml, pml, net is not None)
    peak = np.max(np.abs(ref), axis=1)
    err = np.max(np.abs(got - ref), axis=1) / peak
    l2 = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return {"max_rel_error": float(err.max()), "per_probe": err.tolist(),
            "trace_rel_l2": float(l2.max()), "cpml": cpml, "closure": net is not None,
            "profile": "innermost cells of the 16-cell grading" if truncated else "graded over the layer",
            "interior": interior, "steps": steps}
