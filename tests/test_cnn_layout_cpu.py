"""Host-side layout logic of the learned preconditioner, checked on the CPU.

The tcgen05 convolution reads its A operand as runs of 16-byte pixel rows of
the padded-linear activation buffer and its B operand in the [tap][cin/8][32][8]
weight layout.  These tests restate that operand addressing in NumPy on the
buffers the host code builds (``pack_padded``, ``kernel_layout``,
``transposed_layout``) and compare with the float64 oracle's convolution, so a
layout mistake in the host code shows up without a GPU.
"""

import numpy as np
import pytest
import torch

from oracle import cnn_oracle as co
from thick_ptycho_b200.learned import (kernel_layout, pack_padded, padded_linear_geometry, transposed_layout,
                                       unpack_padded, wgrad_to_torch)

TILE, BLOCKS = 512, 4


def emulate_conv(buf, wl, cin, nf, nb, batch):
    """The conv kernel's operand addressing (cnn_tc.cu) on host buffers."""
    wp, s, g0, cs = padded_linear_geometry(nf, nb, batch)
    x = buf.view(torch.bfloat16).float().reshape(cin // 8, cs, 8).numpy().astype(np.float64)
    w = wl.float().numpy().astype(np.float64)  # (9, cin/8, 32, 8)
    R = TILE + 2 * wp + 2
    lb, le = g0 + wp, g0 + batch * s - wp
    out = np.zeros((batch, 32, nb, nf))
    for t in range(-(-(le - lb) // TILE)):
        l0 = lb + t * TILE
        slab = x[:, l0 - wp - 1:l0 - wp - 1 + R]
        for b in range(BLOCKS):
            D = np.zeros((128, 32))
            for tap in range(9):
                ty, tx = divmod(tap, 3)
                base = b * 128 + ty * wp + tx
                for kk in range(cin // 16):
                    A = np.concatenate([slab[2 * kk, base:base + 128], slab[2 * kk + 1, base:base + 128]], axis=1)
                    Bm = np.concatenate([w[tap, 2 * kk], w[tap, 2 * kk + 1]], axis=1)
                    D += A @ Bm.T
            for m in range(128):
                l = l0 + b * 128 + m
                if not lb <= l < le:
                    continue
                rel = l - g0
                p, rem = divmod(rel, s)
                yp, xp = divmod(rem, wp)
                if p < batch and 1 <= yp <= nb and 1 <= xp <= nf:
                    out[p, :, yp - 1, xp - 1] = D[m]
    return out


def bf(x):
    return torch.as_tensor(x).to(torch.bfloat16).double().numpy()


@pytest.mark.parametrize("cin,nf,nb,batch", [(16, 9, 7, 2), (32, 12, 5, 3)])
def test_kernel_operand_layout_matches_convolution(cin, nf, nb, batch):
    rng = np.random.default_rng(cin + nf)
    x = rng.standard_normal((batch, cin, nb, nf))
    w = rng.standard_normal((32, cin, 3, 3))
    got = emulate_conv(pack_padded(torch.from_numpy(x)), kernel_layout(torch.from_numpy(w)), cin, nf, nb, batch)
    ref = co.conv3x3(bf(x), bf(w))
    assert np.abs(got - ref).max() < 1e-9 * max(1.0, np.abs(ref).max())


def test_transposed_layout_is_the_data_gradient():
    rng = np.random.default_rng(5)
    nf, nb, batch = 10, 6, 2
    dy = rng.standard_normal((batch, 32, nb, nf))
    w = rng.standard_normal((32, 32, 3, 3))
    got = emulate_conv(pack_padded(torch.from_numpy(dy)), transposed_layout(torch.from_numpy(w)), 32, nf, nb, batch)
    ref = co.conv3x3_dgrad(bf(dy), bf(w))
    assert np.abs(got - ref).max() < 1e-9 * np.abs(ref).max()


def test_pack_unpack_roundtrip_and_zero_border():
    rng = np.random.default_rng(2)
    x = torch.from_numpy(rng.standard_normal((3, 16, 5, 7)))
    buf = pack_padded(x)
    back = unpack_padded(buf, 16, 3, 7, 5)
    assert torch.equal(back, x.to(torch.bfloat16).float())
    wp, s, g0, cs = padded_linear_geometry(7, 5, 3)
    full = buf.view(torch.bfloat16).reshape(2, cs, 8).float()
    assert float(full.abs().sum()) == pytest.approx(float(back.abs().sum()), rel=1e-6)  # nothing off the interior


def test_wgrad_layout_mapping():
    rng = np.random.default_rng(3)
    g = rng.standard_normal((32, 16, 3, 3))
    flat = torch.from_numpy(g).permute(2, 3, 1, 0).reshape(9, 16, 32).contiguous()  # [tap][c][o]
    assert torch.equal(wgrad_to_torch(flat, 16), torch.from_numpy(g))
