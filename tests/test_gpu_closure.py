"""GPU: the learned thin-CPML closure.

1. The network's CUDA training kernels (forward, backward to the weights,
   bfloat16 weights, FP32 accumulation) against the numpy restatement in
   oracle/closure_oracle.py, float64 with the same bfloat16-rounded weights.
2. The closure applied inside a step equals the explicit pipeline (band
   gather, per-face RMS normalization, three convs, scatter) run by hand.
3. Training on teacher-forced samples reduces the one-step residual on
   held-out runs.
4. Ablation: the trained closure on the thin layer (the innermost 4 cells
   of the 16-cell grading) against the same thin layer without it, with the
   plain CPML judging both through the reflection test.
"""
import ctypes as C
import types

import numpy as np
import pytest

import wavefront_b200 as wf
from oracle import closure_oracle as CO
from wavefront_b200 import _lib as L
from wavefront_b200 import closure as CL
from wavefront_b200 import configs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_training_kernels_match_numpy():
    rng = np.random.default_rng(0)
    n, D, H, W = 3, 8, 6, 7
    face = np.array([0, 3, 5], np.int32)
    x = rng.standard_normal((n, 10, D, H, W)).astype(np.float32)
    t = (rng.standard_normal((n, 6, D, H, W)) * 0.1).astype(np.float32)
    net = CL.ClosureNet(seed=1)
    net.w[2].mul_(300.0)  # a last layer that matters
    net.wb[2].copy_(net.w[2].to(torch.bfloat16))
    ws = [CO.bf16_round(w.cpu().numpy()) for w in net.w]
    loss_o, dws_o, y_o = CO.net_loss_and_grads(x.astype(np.float64), t.astype(np.float64), ws, face, 6)
    dev = net.dev
    y, cache = net.forward(torch.from_numpy(x).to(dev), torch.from_numpy(face).to(dev))
    loss, dy = net.loss_grad(y, torch.from_numpy(t).to(dev))
    net.backward(dy, cache)
    torch.cuda.synchronize()
    assert np.abs(y.cpu().numpy() - y_o).max() <= 1e-5 * np.abs(y_o).max()
    assert abs(loss.item() - loss_o) <= 1e-5 * loss_o
    for k in range(3):
        g, go = net.dw[k].cpu().numpy(), dws_o[k]
        assert np.abs(g - go).max() <= 1e-5 * np.abs(go).max(), k


@pytest.mark.parametrize("shape", [(2, 10, 16, 8, 6, 7), (3, 16, 16, 8, 37, 65), (6, 16, 6, 8, 9, 33),
                                   (1, 3, 5, 5, 4, 61)])
def test_tensor_core_convs_match_the_oracle(shape):
    """The tcgen05 implicit-GEMM convolutions (forward with GELU and the
    pre-activation, and the gradient with respect to the input) against the
    float64 restatement with the same bfloat16 weights, within 1e-5 of the
    largest magnitude; tile edges in every direction (30-column, 4-row and
    4-plane tiles), channel counts below 16 and a depth below a tile."""
    n, ci, co, D, H, W = shape
    rng = np.random.default_rng(sum(shape))
    face = (np.arange(n) * 5 % 6).astype(np.int32)
    x = rng.standard_normal((n, ci, D, H, W)).astype(np.float32)
    dz = rng.standard_normal((n, co, D, H, W)).astype(np.float32)
    w = CO.bf16_round((rng.standard_normal((6, co, ci, 27)) * 0.2).astype(np.float32))
    dev = torch.device("cuda", 0)
    wb = torch.from_numpy(w.astype(np.float32)).to(dev).to(torch.bfloat16)
    fx, tf, tdz = (torch.from_numpy(v).to(dev) for v in (x, face, dz))
    z = torch.empty(n, co, D, H, W, device=dev)
    a = torch.empty_like(z)
    din = torch.empty(n, ci, D, H, W, device=dev)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.lib().wf_nn_set_tensor_cores(1) == L.WF_OK
    L.check(L.lib().wf_nn_conv3d_forward(CL._p(fx), CL._p(wb), CL._p(tf), CL._p(z), CL._p(a),
                                         n, ci, co, D, H, W, 1, st))
    L.check(L.lib().wf_nn_conv3d_backward_data(CL._p(tdz), CL._p(wb), CL._p(tf), CL._p(din),
                                               n, ci, co, D, H, W, st))
    torch.cuda.synchronize()
    assert L.lib().wf_nn_tensor_core_timeouts() == 0
    zo = CO.conv_fwd(x.astype(np.float64), w.astype(np.float64), face)
    ao = CO.gelu(zo)
    do = CO.conv_bwd_data(dz.astype(np.float64), w.astype(np.float64), face, ci)
    for got, want, what in ((z, zo, "pre-activation"), (a, ao, "GELU output"), (din, do, "input gradient")):
        g = got.cpu().numpy()
        err = np.abs(g - want).max() / np.abs(want).max()
        assert err <= 1e-5, (what, err)


def test_tensor_core_and_cuda_core_convs_agree():
    """The two kernel sets behind wf_nn_set_tensor_cores agree to 1e-5 of the
    largest magnitude on a closure-sized band (6 faces, 10 -> 16 channels):
    both accumulate the 270 products of a voxel in FP32, in different orders
    (measured: 2e-6 of the largest output), and both stay within the same 1e-5
    of the float64 restatement."""
    rng = np.random.default_rng(3)
    n, ci, co, D, H, W = 6, 10, 16, 8, 48, 48
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(rng.standard_normal((n, ci, D, H, W)).astype(np.float32)).to(dev)
    wb = (torch.from_numpy(rng.standard_normal((6, co, ci, 27)).astype(np.float32)) * 0.2).to(dev).to(torch.bfloat16)
    face = torch.arange(6, dtype=torch.int32, device=dev)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    outs = []
    try:
        for on in (1, 0):
            L.lib().wf_nn_set_tensor_cores(on)
            out = torch.empty(n, co, D, H, W, device=dev)
            L.check(L.lib().wf_nn_conv3d_forward(CL._p(x), CL._p(wb), CL._p(face), None, CL._p(out),
                                                 n, ci, co, D, H, W, 1, st))
            outs.append(out)
    finally:
        L.lib().wf_nn_set_tensor_cores(1)
    torch.cuda.synchronize()
    err = (outs[0] - outs[1]).abs().max().item() / outs[1].abs().max().item()
    assert err <= 1e-5, err


@pytest.mark.parametrize("n", [16, 24, 32])
def test_closure_in_step_equals_explicit_pipeline(n):
    """One step with the closure attached against the same step without it
    followed by the closure's pipeline by hand (random fields, thin layer).
    From 32 cells the step runs the packed tensor-core path; narrower grids
    keep the FP32-in path."""
    dx = 1.0e-3
    sc = types.SimpleNamespace(dx=dx, dt=configs.courant_dt(dx))
    net = CL.ClosureNet(seed=2)
    net.w[2].mul_(50.0)
    net.wb[2].copy_(net.w[2].to(torch.bfloat16))
    dims = wf.GridDims(n, n, n)
    rng = np.random.default_rng(5)
    f0 = (rng.standard_normal((6, n, n, n)) * 0.01).astype(np.float32)
    g1 = wf.DeviceFieldGrid(dims, kernel="fused")
    g2 = wf.DeviceFieldGrid(dims, kernel="fused")
    try:
        for g in (g1, g2):
            g.set_materials(wf.MaterialGrid(dims), wf.MaterialTable.vacuum_filled(sc.dt, sc.dx))
            CL.set_thin_cpml(g, sc.dt, sc.dx)
            g.set_fields(f0)
        net.attach(g1)
        g1.step(1)
        g2.step(1)
        g2.sync()
        P = 8 * n * n
        X = torch.empty(6, 10, 8, n, n, device=net.dev)
        L.check(L.lib().wf_band_gather(g2._h, CL._p(X), net.gain_e, net.gain_h))
        torch.cuda.synchronize()
        s = torch.sqrt(torch.sum(X[:, :3].reshape(6, -1) ** 2, dim=1) / (3 * P)) + 1e-30
        Xs = X / s.view(6, 1, 1, 1, 1)
        faces = torch.arange(6, dtype=torch.int32, device=net.dev)
        y, _ = net.forward(Xs.contiguous(), faces)
        Y = (y * s.view(6, 1, 1, 1, 1)).contiguous()
        torch.cuda.synchronize()  # Y comes from torch's stream; the scatter runs on the handle's
        L.check(L.lib().wf_band_scatter_add(g2._h, CL._p(Y), net.gain_e, net.gain_h))
        torch.cuda.synchronize()
        got, want = g1.fields(), g2.fields()
        # the per-face RMS is reduced in a different order here, so the
        # corrections may differ in their last bits: bound the difference by
        # 1e-6 of the largest field value
        assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
        assert not np.array_equal(got, f0)
    finally:
        g1.close()
        g2.close()


def test_tensor_core_closure_step_matches_cuda_core_step():
    """The in-step closure on the tensor cores with packed operands (one TMA
    box per tile, weights pre-arranged, the next layer's split written by the
    epilogue) against the same step with the CUDA-core convolutions, over
    three steps from random fields on a 48^3 grid (tile edges in x and y)."""
    dims = wf.GridDims(48, 48, 48)
    sc = configs.plain_cube_64(steps=1, n=48)
    net = CL.ClosureNet(seed=7)
    net.w[2].mul_(50.0)
    net.wb[2].copy_(net.w[2].to(torch.bfloat16))
    rng = np.random.default_rng(8)
    f0 = (rng.standard_normal((6, 48, 48, 48)) * 0.01).astype(np.float32)
    out = []
    try:
        for tc in (1, 0):
            L.lib().wf_nn_set_tensor_cores(tc)
            g = wf.DeviceFieldGrid(dims, kernel="fused")
            try:
                g.set_materials(wf.MaterialGrid(dims), wf.MaterialTable.vacuum_filled(sc.dt, sc.dx))
                CL.set_thin_cpml(g, sc.dt, sc.dx)
                g.set_fields(f0)
                net.attach(g)
                g.step(3)
                g.sync()
                out.append(g.fields())
            finally:
                g.close()
    finally:
        L.lib().wf_nn_set_tensor_cores(1)
    assert L.lib().wf_nn_tensor_core_timeouts() == 0
    assert not np.array_equal(out[0], f0)
    assert np.abs(out[0] - out[1]).max() <= 1e-5 * np.abs(out[1]).max()


def test_energy_guard_in_step_and_never_raises_band_energy():
    """With the guard on, a step equals the explicit pipeline with the guard
    applied by hand, and each face's correction can only lower the energy of
    its band's six fields (sum of squares in the gained units)."""
    n = 32
    sc = configs.plain_cube_64(steps=1, n=n)
    net = CL.ClosureNet(seed=4)
    net.w[2].mul_(400.0)  # a correction large enough that the guard must act
    net.wb[2].copy_(net.w[2].to(torch.bfloat16))
    dims = wf.GridDims(32, 32, 32)
    rng = np.random.default_rng(6)
    f0 = (rng.standard_normal((6, 32, 32, 32)) * 0.01).astype(np.float32)
    g1 = wf.DeviceFieldGrid(dims, kernel="fused")
    g2 = wf.DeviceFieldGrid(dims, kernel="fused")
    try:
        for g in (g1, g2):
            g.set_materials(wf.MaterialGrid(dims), wf.MaterialTable.vacuum_filled(sc.dt, sc.dx))
            CL.set_thin_cpml(g, sc.dt, sc.dx)
            g.set_fields(f0)
        net.attach(g1, guard=True)
        g1.step(1)
        g2.step(1)
        g2.sync()
        P = 8 * n * n
        X = torch.empty(6, 10, 8, n, n, device=net.dev)
        L.check(L.lib().wf_band_gather(g2._h, CL._p(X), net.gain_e, net.gain_h))
        torch.cuda.synchronize()
        s = torch.sqrt(torch.sum(X[:, :3].reshape(6, -1) ** 2, dim=1) / (3 * P)) + 1e-30
        Xs = (X / s.view(6, 1, 1, 1, 1)).contiguous()
        faces = torch.arange(6, dtype=torch.int32, device=net.dev)
        y, _ = net.forward(Xs, faces)
        Y = y * s.view(6, 1, 1, 1, 1)
        F = X[:, :6]
        a = torch.sum((F * Y).reshape(6, -1).double(), dim=1)
        b = torch.sum((Y * Y).reshape(6, -1).double(), dim=1)
        grow = 2 * a + b > 0
        lam = torch.where(grow, torch.clamp(-2 * a / torch.clamp(b, min=1e-300), 0, 1),
                          torch.ones_like(a))
        assert bool(grow.any())  # the guard has work to do in this case
        Yg = (Y * lam.view(6, 1, 1, 1, 1).float()).contiguous()
        e_before = torch.sum((F * F).reshape(6, -1).double(), dim=1)
        e_after = torch.sum(((F + Yg) ** 2).reshape(6, -1).double(), dim=1)
        assert bool(torch.all(e_after <= e_before * (1 + 1e-6)))
        torch.cuda.synchronize()  # Yg comes from torch's stream; the scatter runs on the handle's
        L.check(L.lib().wf_band_scatter_add(g2._h, CL._p(Yg), net.gain_e, net.gain_h))
        torch.cuda.synchronize()
        got, want = g1.fields(), g2.fields()
        assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    finally:
        g1.close()
        g2.close()


@pytest.fixture(scope="module")
def trained():
    X, R, F, _ = CL.generate(96, seed=1)
    Xv, Rv, Fv, _ = CL.generate(8, seed=99)
    net, _ = CL.train(X, R, F, 1.0, iters=4000, lr=3e-4)
    return net, (X, R, F), (Xv, Rv, Fv)


def test_training_reduces_the_one_step_residual(trained):
    net, _, (Xv, Rv, Fv) = trained
    none, with_net = CL.residual_loss(None, Xv, Rv, Fv), CL.residual_loss(net, Xv, Rv, Fv)
    print(f"\nheld-out one-step residual: without {none:.3e}, with the network {with_net:.3e}")
    assert with_net < none / 3.0


def test_ablation_closure_on_the_thin_layer(trained):
    """Reflection-test error (max over probes of max_t |E - E_ref| / max|E_ref|)
    of the thin layer with the trained closure (correction gain 0.5) against
    the same thin layer without it; the plain CPMLs for reference."""
    net = trained[0]
    thin = CL.reflection_test(truncated=True)
    closed = CL.reflection_test(net=net, alpha=0.5, truncated=True)
    steep4 = CL.reflection_test(cpml=4)
    thick16 = CL.reflection_test(cpml=16)
    print(f"\nthin layer alone {thin['max_rel_error']:.3f}, with closure {closed['max_rel_error']:.3f}; "
          f"plain 4-cell CPML {steep4['max_rel_error']:.3f}, 16-cell CPML {thick16['max_rel_error']:.4f}")
    assert np.isfinite(closed["max_rel_error"])
    assert closed["max_rel_error"] < 0.5 * thin["max_rel_error"]
