"""CPU oracle for the learned coarse-grid correction network.

TEST INFRASTRUCTURE ONLY.  The tests compare the CUDA network kernels
(``gpu-to_b200/csrc/kernels_learned.cu``) against this numpy restatement and
check its analytic gradients against finite differences; the product never
imports it.

The network has no counterpart in the reference (GPU-TO solves with a plain
V-cycle); its definition is this project's:

* input  [4, X, Z, Y] on the level-2 node grid (node order of the solver: x
  slowest, y fastest): a density feature and the three components of the
  scaled level-2 residual;
* three 3x3x3 convolutions 4 -> 16 -> 32 -> 64 with bias and ReLU, zero
  padding at the grid boundary, then a 1x1x1 convolution 64 -> 3 with bias;
* weights are stored in FP32 and used rounded to BF16 (round to nearest
  even); activations and sums are FP32.

Flat parameter layout (shared with the CUDA side): for each layer, the
weights w[co][ci][tap] and then the biases b[co]; tap = 9 (dx+1) + 3 (dz+1)
+ (dy+1) for offsets dx, dz, dy in {-1, 0, 1}.
"""
from __future__ import annotations

import numpy as np

CHANNELS = (4, 16, 32, 64, 3)
KSIZE = (3, 3, 3, 1)


def layer_shapes():
    out = []
    for l in range(4):
        ci, co, k = CHANNELS[l], CHANNELS[l + 1], KSIZE[l]
        out.append(((co, ci, k ** 3), (co,)))
    return out


def num_params():
    return sum(int(np.prod(w)) + b[0] for w, b in layer_shapes())


def unpack(theta):
    """Flat parameter vector -> [(w, b)] views."""
    out, o = [], 0
    for ws, bs in layer_shapes():
        nw = int(np.prod(ws))
        out.append((theta[o:o + nw].reshape(ws), theta[o + nw:o + nw + bs[0]]))
        o += nw + bs[0]
    return out


def bf16_round(a):
    """Round float32 values to the nearest BF16 value (ties to even)."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def _taps(k):
    if k == 1:
        return [(0, 0, 0)]
    return [(dx, dz, dy) for dx in (-1, 0, 1) for dz in (-1, 0, 1) for dy in (-1, 0, 1)]


def _shift(x, d):
    """y[..., i, k, j] = x[..., i+dx, k+dz, j+dy], zero outside."""
    dx, dz, dy = d
    y = np.zeros_like(x)
    X, Z, Y = x.shape[-3:]
    sx = slice(max(0, -dx), X - max(0, dx))
    sz = slice(max(0, -dz), Z - max(0, dz))
    sy = slice(max(0, -dy), Y - max(0, dy))
    tx = slice(max(0, dx), X - max(0, -dx))
    tz = slice(max(0, dz), Z - max(0, -dz))
    ty = slice(max(0, dy), Y - max(0, -dy))
    y[..., sx, sz, sy] = x[..., tx, tz, ty]
    return y


def conv(x, w, b, k):
    """out[co] = b[co] + sum_ci sum_tap w[co, ci, tap] x[ci](node + offset)."""
    out = np.broadcast_to(b[:, None, None, None], (w.shape[0],) + x.shape[1:]).astype(x.dtype).copy()
    for t, d in enumerate(_taps(k)):
        xs = _shift(x, d)
        out += np.tensordot(w[:, :, t], xs, axes=(1, 0))
    return out


def conv_bwd(x, w, k, gy):
    """Gradients of conv: (d input, d weights, d bias) given d output gy."""
    gx = np.zeros_like(x)
    gw = np.zeros_like(w)
    for t, d in enumerate(_taps(k)):
        xs = _shift(x, d)
        gw[:, :, t] = np.tensordot(gy, xs, axes=([1, 2, 3], [1, 2, 3]))
        back = np.tensordot(w[:, :, t], gy, axes=(0, 0))          # [ci, ...] at node + 0
        gx += _shift(back, (-d[0], -d[1], -d[2]))
    gb = gy.sum(axis=(1, 2, 3))
    return gx, gw, gb


def forward(x, theta, round_weights=True, dtype=np.float32):
    """Network output and the activations the backward pass needs."""
    acts = [x.astype(dtype)]
    h = acts[0]
    for l, (w, b) in enumerate(unpack(theta)):
        w = bf16_round(w) if round_weights else w
        h = conv(h, w.astype(dtype), b.astype(dtype), KSIZE[l])
        if l < 3:
            h = np.maximum(h, 0)
        acts.append(h)
    return h, acts


def loss(y, t, m):
    """Masked mean square error and its gradient w.r.t. y."""
    den = max(float(m.sum()), 1.0)
    r = (y - t) * m
    return float((r * r).sum() / den), 2.0 * r / den


def backward(acts, theta, gy, round_weights=True):
    """Gradient of the loss w.r.t. the flat parameters, given d output gy."""
    dtype = acts[0].dtype
    grads = []
    g = gy.astype(dtype)
    layers = unpack(theta)
    for l in range(3, -1, -1):
        w, _ = layers[l]
        w = (bf16_round(w) if round_weights else w).astype(dtype)
        if l < 3:
            g = g * (acts[l + 1] > 0)
        gx, gw, gb = conv_bwd(acts[l], w, KSIZE[l], g)
        grads.append((gw, gb))
        g = gx
    flat = []
    for gw, gb in reversed(grads):
        flat += [gw.reshape(-1), gb]
    return np.concatenate(flat)


def init_params(seed=0):
    """He-normal weights (the last layer scaled down), zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (ws, bs) in enumerate(layer_shapes()):
        fan_in = ws[1] * ws[2]
        std = np.sqrt(2.0 / fan_in) * (0.1 if l == 3 else 1.0)
        parts += [rng.standard_normal(int(np.prod(ws))) * std, np.zeros(bs[0])]
    return np.concatenate(parts).astype(np.float32)
