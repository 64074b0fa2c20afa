"""CPU restatement of the learned-conduction network.  TEST INFRASTRUCTURE
ONLY: the product path (lare3d_b200.surrogate) never imports this module.

The network has no counterpart in the reference; this file is the CPU
oracle its device kernels (lare3d_b200/csrc/surrogate.cu) are checked
against: the same 4-layer valid 3-D convolution with ReLU, the same MSE
loss on channel 0, and the backward pass written out by hand (backward-data
as a full convolution with tap-flipped, transposed weights; weight gradient
as a sum over voxels of dy x^T per tap).

All arithmetic is float64.  With ``rounding=True`` the values are rounded to
bfloat16 at the points where the device kernels store bfloat16 (inputs,
weights, activations, output gradients), so that a comparison measures the
kernels' FP32 accumulation and not the storage format.
"""
from __future__ import annotations

import numpy as np

# (cin padded, cout of the master weights, cin used, cout used by the forward)
LAYERS = ((16, 32, 7, 32), (32, 32, 32, 32), (32, 32, 32, 32), (32, 16, 32, 1))
TAPS = [(t // 9, (t // 3) % 3, t % 3) for t in range(27)]   # t = (dz*3 + dy)*3 + dx


def bf16(a):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    u = ((u + r) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def conv(x, w, bias=None, pad=0, relu=False, mask=None):
    """y[b,o,co] = sum_{t,ci} w[t,co,ci] x[b, o + d(t) - pad, ci] (+ bias, ReLU, mask).
    x: [nb, d, d, d, cin]; w: [27, cout, cin]."""
    if pad:
        x = np.pad(x, ((0, 0), (pad, pad), (pad, pad), (pad, pad), (0, 0)))
    nb, d = x.shape[0], x.shape[1]
    do = d - 2
    y = np.zeros((nb, do, do, do, w.shape[1]))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += x[:, dz:dz + do, dy:dy + do, dx:dx + do, :] @ w[t].T
    if bias is not None:
        y = y + bias
    if relu:
        y = np.maximum(y, 0.0)
    if mask is not None:
        y = y * (mask > 0)
    return y


def flip(w):
    """Backward-data weights: wb[t'] = w[26 - t'].T, [27, cin, cout]."""
    return np.stack([w[26 - t].T for t in range(27)])


def wgrad(dy, x):
    """Weight and bias gradients of a valid conv (x has edge dout + 2)."""
    do = dy.shape[1]
    dw = np.stack([np.einsum("bzyxo,bzyxi->oi", dy, x[:, dz:dz + do, dy_:dy_ + do, dx:dx + do, :])
                   for (dz, dy_, dx) in TAPS])
    return dw, dy.sum(axis=(0, 1, 2, 3))


def init_params(seed=0):
    """He-normal weights on the used channels, zero padding and biases; the
    last layer is scaled by 0.1.  Returns lists W[l] [27, cout, cin], b[l]."""
    rng = np.random.default_rng(seed)
    W, B = [], []
    for l, (cin, cout, cin_r, _cf) in enumerate(LAYERS):
        cout_r = 1 if l == len(LAYERS) - 1 else cout
        std = np.sqrt(2.0 / (27.0 * cin_r)) * (0.1 if l == len(LAYERS) - 1 else 1.0)
        w = np.zeros((27, cout, cin), np.float32)
        w[:, :cout_r, :cin_r] = (rng.standard_normal((27, cout_r, cin_r)) * std).astype(np.float32)
        W.append(w)
        B.append(np.zeros(cout, np.float32))
    return W, B


def forward(W, B, x, rounding=True):
    """Activations [x, a1, a2, a3] and the FP32-like output [nb, p, p, p, 8]."""
    q = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    acts = [q(x)]
    a = acts[0]
    for l in range(3):
        a = q(conv(a, q(W[l]), B[l].astype(np.float64), relu=True))
        acts.append(a)
    cf = LAYERS[3][3]
    out = conv(a, q(W[3][:, :cf, :]), B[3][:cf].astype(np.float64))
    return acts, out


def loss_and_grads(W, B, x, target, rounding=True):
    """MSE of channel 0 against target [nb, p, p, p] and the gradients of
    every weight and bias, as the device's backward pass computes them."""
    q = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    acts, out = forward(W, B, x, rounding)
    count = target.size
    diff = out[..., 0] - target
    loss = float(np.mean(diff * diff))
    cpad = LAYERS[3][1]
    dy = np.zeros(out.shape[:4] + (cpad,))
    dy[..., 0] = 2.0 * diff / count
    dy = q(dy)
    dW, dB = [None] * 4, [None] * 4
    for l in (3, 2, 1, 0):
        dW[l], dB[l] = wgrad(dy, acts[l])
        if l > 0:
            dy = q(conv(dy, flip(q(W[l])), pad=2, mask=acts[l]))
    return loss, dW, dB
