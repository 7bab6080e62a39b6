"""float64 restatement of the learned 3D preconditioner (CNN + per-pixel filter).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, never by the product package.

The reference has no learned component (the learned preconditioner is this
project's own addition), so there is no reference file to cite or golden vector
to pin against: this module restates the network's defining equations so the
GPU kernels (forward, backward data, weight gradients, filter gradient) can be
checked against an independent float64 computation.  Parity here is against
these equations, not against the reference.

Network (all 3x3 convolutions with zero padding, 32 outputs):
  f = features(d) (16 channels: kappa Re d, kappa Im d, 1, x==0, x==W-1,
      y==0, y==H-1, zeros)
  a1 = relu(conv(f, W1) + b1); a2 = relu(conv(a1, W2) + b2);
  a3 = relu(conv(a2, W3) + b3); o = conv(a3, W4) + b4
  F_t = out_scale (o[2t] + i o[2t+1]), t < 13
  y_v = z_v + sum_t F_t(x) z_v(x + o_t)
"""

from __future__ import annotations

import numpy as np

TAPS = ((0, 0), (0, -1), (0, 1), (-1, 0), (1, 0), (-1, -1), (-1, 1), (1, -1), (1, 1), (0, -2), (0, 2), (-2, 0), (2, 0))


def features(d, kappa):
    """(B, H, W) complex diagonals → (B, 16, H, W) float64 features."""
    B, H, W = d.shape
    f = np.zeros((B, 16, H, W))
    f[:, 0] = kappa * d.real
    f[:, 1] = kappa * d.imag
    f[:, 2] = 1.0
    f[:, 3, :, 0] = 1.0
    f[:, 4, :, W - 1] = 1.0
    f[:, 5, 0, :] = 1.0
    f[:, 6, H - 1, :] = 1.0
    return f


def conv3x3(x, w, b=None):
    """Same-padded 3x3 correlation: x (B, C, H, W), w (O, C, 3, 3) → (B, O, H, W)."""
    B, C, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    out = np.zeros((B, w.shape[0], H, W))
    for ty in range(3):
        for tx in range(3):
            out += np.einsum("oc,bchw->bohw", w[:, :, ty, tx], xp[:, :, ty:ty + H, tx:tx + W])
    if b is not None:
        out += b[None, :, None, None]
    return out


def conv3x3_wgrad(x, dy):
    """d/dW of sum(conv3x3(x, W) * dy): (O, C, 3, 3)."""
    B, C, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    g = np.zeros((dy.shape[1], C, 3, 3))
    for ty in range(3):
        for tx in range(3):
            g[:, :, ty, tx] = np.einsum("bohw,bchw->oc", dy, xp[:, :, ty:ty + H, tx:tx + W])
    return g


def conv3x3_dgrad(dy, w):
    """d/dx of sum(conv3x3(x, W) * dy): correlation with the flipped, transposed kernel."""
    return conv3x3(dy, np.flip(w, axis=(2, 3)).transpose(1, 0, 2, 3))


def shift(z, dy, dx):
    """z(x + (dy, dx)) with zeros outside (last two axes)."""
    H, W = z.shape[-2:]
    out = np.zeros_like(z)
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[..., yd, xd] = z[..., ys, xs]
    return out


def filter_from_output(o):
    """(B, 32, H, W) → (B, 13, H, W) complex."""
    return o[:, 0:26:2] + 1j * o[:, 1:26:2]


def filter_apply(F, z, per_image, conj=False):
    """y_v = z_v + sum_t F_t z_v(x + o_t); z (V, H, W), vector v uses F[v // per_image]."""
    Fc = np.conj(F) if conj else F
    y = z.astype(complex).copy()
    for v in range(z.shape[0]):
        Fi = Fc[v // per_image]
        for t, (dy, dx) in enumerate(TAPS):
            y[v] += Fi[t] * shift(z[v], dy, dx)
    return y


def forward(weights, biases, d, kappa, out_scale=1.0):
    """Activations and the filter (out_scale times the last layer) of the four-layer network."""
    f = features(d, kappa)
    a1 = np.maximum(conv3x3(f, weights[0], biases[0]), 0)
    a2 = np.maximum(conv3x3(a1, weights[1], biases[1]), 0)
    a3 = np.maximum(conv3x3(a2, weights[2], biases[2]), 0)
    o = conv3x3(a3, weights[3], biases[3])
    return {"f": f, "a1": a1, "a2": a2, "a3": a3, "o": o, "F": out_scale * filter_from_output(o)}


def loss_and_grads(weights, biases, d, kappa, z, target, scale, per_image, out_scale=1.0):
    """L = sum_v scale_v |y_v - target_v|^2 and its gradients w.r.t. weights and biases."""
    act = forward(weights, biases, d, kappa, out_scale)
    y = filter_apply(act["F"], z, per_image)
    r = y - target
    loss = float(np.sum(scale[:, None, None] * np.abs(r) ** 2))
    e = scale[:, None, None] * r
    B, _, H, W = act["o"].shape
    do = np.zeros((B, 32, H, W))
    for v in range(z.shape[0]):
        img = v // per_image
        for t, (dy, dx) in enumerate(TAPS):
            g = 2 * out_scale * np.conj(shift(z[v], dy, dx)) * e[v]
            do[img, 2 * t] += g.real
            do[img, 2 * t + 1] += g.imag
    gw, gb = [None] * 4, [None] * 4
    gw[3] = conv3x3_wgrad(act["a3"], do)
    gb[3] = do.sum(axis=(0, 2, 3))
    g3 = conv3x3_dgrad(do, weights[3]) * (act["a3"] > 0)
    gw[2] = conv3x3_wgrad(act["a2"], g3)
    gb[2] = g3.sum(axis=(0, 2, 3))
    g2 = conv3x3_dgrad(g3, weights[2]) * (act["a2"] > 0)
    gw[1] = conv3x3_wgrad(act["a1"], g2)
    gb[1] = g2.sum(axis=(0, 2, 3))
    g1 = conv3x3_dgrad(g2, weights[1]) * (act["a1"] > 0)
    gw[0] = conv3x3_wgrad(act["f"], g1)
    gb[0] = g1.sum(axis=(0, 2, 3))
    return loss, gw, gb, act, do
