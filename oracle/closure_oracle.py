"""CPU restatement of the learned boundary closure's network (numpy, float64).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the CUDA training kernels
(wf_nn_conv3d_forward / backward_data / backward_weight, GELU backward, MSE,
Adam) of the library.  The network has no counterpart in the reference
(AndrejRumenovski/wavefront); its definition is the library's:

  tensors [n][c][d][h][w]; 3x3x3 convolution, stride 1, zero padding, no
  bias, weights [faces][cout][cin][27] with tap t = (dd+1)*9 + (dy+1)*3 +
  (dx+1) reading in[p + (dd, dy, dx)]; sample i uses the weights of face[i];
  GELU(z) = 0.5 z (1 + erf(z / sqrt 2)).
"""
from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf)
OFFS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def _shift(x, dd, dy, dx):
    """y[..., d, h, w] = x[..., d+dd, h+dy, w+dx] (zero outside)."""
    out = np.zeros_like(x)
    D, H, W = x.shape[-3:]
    sd = slice(max(0, -dd), min(D, D - dd))
    sh = slice(max(0, -dy), min(H, H - dy))
    sw = slice(max(0, -dx), min(W, W - dx))
    td = slice(max(0, dd), min(D, D + dd))
    th = slice(max(0, dy), min(H, H + dy))
    tw = slice(max(0, dx), min(W, W + dx))
    out[..., sd, sh, sw] = x[..., td, th, tw]
    return out


def conv_fwd(x, w, face):
    """x [n][ci][D][H][W], w [F][co][ci][27] -> [n][co][D][H][W]."""
    n = x.shape[0]
    co = w.shape[1]
    out = np.zeros((n, co) + x.shape[2:], np.float64)
    for i in range(n):
        wf = w[face[i]]
        for t, (dd, dy, dx) in enumerate(OFFS):
            xs = _shift(x[i], dd, dy, dx)  # [ci][D][H][W]
            out[i] += np.einsum("oc,cdhw->odhw", wf[:, :, t], xs)
    return out


def conv_bwd_data(dz, w, face, ci):
    n = dz.shape[0]
    out = np.zeros((n, ci) + dz.shape[2:], np.float64)
    for i in range(n):
        wf = w[face[i]]
        for t, (dd, dy, dx) in enumerate(OFFS):
            g = _shift(dz[i], -dd, -dy, -dx)  # g[p] = dz[p - off]
            out[i] += np.einsum("oc,odhw->cdhw", wf[:, :, t], g)
    return out


def conv_bwd_weight(x, dz, face, nface):
    n, ci = x.shape[:2]
    co = dz.shape[1]
    dw = np.zeros((nface, co, ci, 27), np.float64)
    for i in range(n):
        for t, (dd, dy, dx) in enumerate(OFFS):
            xs = _shift(x[i], dd, dy, dx)
            dw[face[i], :, :, t] += np.einsum("odhw,cdhw->oc", dz[i], xs)
    return dw


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def net_loss_and_grads(x, t, ws, face, nface):
    """The closure network (10->16 GELU ->16 GELU ->6) with MSE loss against
    t: returns (loss, [dw1, dw2, dw3], y)."""
    z1 = conv_fwd(x, ws[0], face)
    a1 = gelu(z1)
    z2 = conv_fwd(a1, ws[1], face)
    a2 = gelu(z2)
    y = conv_fwd(a2, ws[2], face)
    m = y.size
    loss = float(np.sum((y - t) ** 2) / m)
    dy = 2.0 * (y - t) / m
    dw3 = conv_bwd_weight(a2, dy, face, nface)
    da2 = conv_bwd_data(dy, ws[2], face, a2.shape[1])
    dz2 = da2 * gelu_grad(z2)
    dw2 = conv_bwd_weight(a1, dz2, face, nface)
    da1 = conv_bwd_data(dz2, ws[1], face, a1.shape[1])
    dz1 = da1 * gelu_grad(z1)
    dw1 = conv_bwd_weight(x, dz1, face, nface)
    return loss, [dw1, dw2, dw3], y


def bf16_round(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)
