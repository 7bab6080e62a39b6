"""Learned correction of the 3D FFT preconditioner (host side).

The plain preconditioner of the 3D BiCGStab solve (``cn3d.cu``) inverts the
periodic transverse operator ``I − σT K_per`` exactly by 2D FFTs and ignores
the object term ``D_s = σT diag(c_s)`` and the true boundary rows.  The
learned form adds a correction computed from the slice itself: a four-layer
3×3 CNN (``csrc/cnn_tc.cu``; bf16 weights, fp32 accumulation on the tcgen05
tensor cores) maps the object diagonal ``d`` of the slice to a 13-tap complex
filter per pixel, and the preconditioner becomes

    y = z + Σ_t F_t(x) · z(x + o_t),   z = M0⁻¹ v (the plain FFT preconditioner).

The correction is linear in ``z`` (BiCGStab keeps a fixed linear
preconditioner) and the network runs once per slice, shared by every probe
and Krylov iteration.  To first order the exact inverse is
``A⁻¹v ≈ z + M0⁻¹(d ⊙ z)``, a per-pixel filter whose taps are the
preconditioner's Green's function times the neighbouring ``d``; the network
learns this and the boundary corrections from (residual, error) pairs that
the solver itself produces (``CN3D.march(..., train_every=k)``).

The reference has no learned component; this module is the project's own
addition on the 3D path.  Training runs on the GPU with the project's own
forward and backward kernels; the optimiser (Adam) updates the fp32 master
weights with torch elementwise operations.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _native

CHANNELS_IN = 16
WIDTH = 32
TAPS = ((0, 0), (0, -1), (0, 1), (-1, 0), (1, 0), (-1, -1), (-1, 1), (1, -1), (1, 1), (0, -2), (0, 2), (-2, 0), (2, 0))


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def kernel_layout(w: torch.Tensor) -> torch.Tensor:
    """torch weight (32, C, 3, 3) → bf16 [9 taps][C/8][32][8] (the conv kernel's B operand)."""
    o, c = w.shape[0], w.shape[1]
    return w.permute(2, 3, 1, 0).reshape(9, c // 8, 8, o).permute(0, 1, 3, 2).contiguous().to(torch.bfloat16)


def transposed_layout(w: torch.Tensor) -> torch.Tensor:
    """Weights of the backward-data convolution of a 32→32 layer: flipped taps, channels swapped."""
    return kernel_layout(w.flip(2, 3).transpose(0, 1).contiguous())


def wgrad_to_torch(dw: torch.Tensor, cin: int) -> torch.Tensor:
    """fp32 [9][cin][32] (tp_conv3x3_wgrad) → torch layout (32, cin, 3, 3)."""
    return dw.view(3, 3, cin, WIDTH).permute(3, 2, 0, 1).contiguous()


def padded_linear_geometry(nf: int, nb: int, batch: int):
    """(Wp, S, G0, CS) of the padded-linear activation layout (``csrc/cnn_internal.cuh``)."""
    wp = nf + 2
    s = (nb + 2) * wp
    g0 = 8
    g1 = ((512 + wp + 8 + 7) // 8) * 8
    cs = ((g0 + batch * s + g1 + 7) // 8) * 8
    return wp, s, g0, cs


def pack_padded(x: torch.Tensor) -> torch.Tensor:
    """(B, C, nb, nf) real tensor → padded-linear bf16 buffer (as uint8 bytes)."""
    B, C, nb, nf = x.shape
    wp, s, g0, cs = padded_linear_geometry(nf, nb, B)
    buf = torch.zeros((C // 8, cs, 8), dtype=torch.bfloat16, device=x.device)
    img = torch.zeros((B, C, nb + 2, wp), dtype=torch.bfloat16, device=x.device)
    img[:, :, 1:nb + 1, 1:nf + 1] = x.to(torch.bfloat16)
    lin = img.reshape(B, C // 8, 8, s).permute(1, 0, 3, 2).reshape(C // 8, B * s, 8)
    buf[:, g0:g0 + B * s] = lin
    return buf.view(torch.uint8).reshape(-1)


def unpack_padded(buf: torch.Tensor, C: int, batch: int, nf: int, nb: int) -> torch.Tensor:
    """Padded-linear bf16 buffer → (batch, C, nb, nf) float32 (interior pixels)."""
    wp, s, g0, cs = padded_linear_geometry(nf, nb, batch)
    b = buf.view(torch.bfloat16).reshape(C // 8, cs, 8)[:, g0:g0 + batch * s]
    img = b.reshape(C // 8, batch, s, 8).permute(1, 0, 3, 2).reshape(batch, C, nb + 2, wp)
    return img[:, :, 1:nb + 1, 1:nf + 1].float()


class CNNBuffers:
    """Zero-bordered padded-linear activation buffers of one (nf, nb, batch)."""

    def __init__(self, lib, nf, nb, batch, device):
        def act(ch):
            n = int(lib.tp_cnn_act_bytes(nf, nb, batch, ch))
            return torch.zeros(n, dtype=torch.uint8, device=device)

        self.feat = act(CHANNELS_IN)
        self.a = [act(WIDTH) for _ in range(3)]
        self.g = [act(WIDTH) for _ in range(4)]  # dY4, dA3, dA2, dA1


@dataclass
class TrainingPairs:
    """Solver-generated pairs: plain-preconditioned residuals, exact solutions, slice diagonals.

    ``z0`` and ``sol`` are (S, P, N) complex64, ``diag`` is (S, N): for slice k,
    ``(I − P_s) sol[k, p] = r0[k, p]`` and ``z0[k, p] = M0⁻¹ r0[k, p]``; the target
    correction is ``sol − z0``."""

    nf: int
    nb: int
    z0: torch.Tensor
    sol: torch.Tensor
    diag: torch.Tensor
    kind: str = "rhs"

    @property
    def count(self):
        return self.z0.shape[0] * self.z0.shape[1]


@dataclass
class TrainLog:
    losses: List[float] = field(default_factory=list)
    steps: int = 0


class LearnedPreconditioner:
    """Weights, training and the ``tp_cnn_model`` view of the learned correction."""

    def __init__(self, nf: int, nb: int, kappa: float, device=None, seed: int = 0, out_scale: Optional[float] = None):
        if not torch.cuda.is_available():
            raise _native.NativeLibraryError("the learned preconditioner needs a CUDA device (no CPU fallback)")
        self.lib = _native.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.nf, self.nb, self.kappa = int(nf), int(nb), float(kappa)
        # the filter is O(|d|) while the features are O(kappa |d|) = O(1): the
        # network predicts kappa * F, so that optimiser steps act on O(1) outputs
        self.out_scale = float(out_scale) if out_scale is not None else 1.0 / self.kappa
        g = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        for i, cin in enumerate((CHANNELS_IN, WIDTH, WIDTH, WIDTH)):
            std = math.sqrt(2.0 / (9 * cin)) * (1e-2 if i == 3 else 1.0)
            self.w.append((torch.randn((WIDTH, cin, 3, 3), generator=g) * std).to(self.device))
            self.b.append(torch.zeros(WIDTH, device=self.device))
        self._adam = None
        self._sync_kernel_weights()
        self._bufs = {}

    # ----------------------------------------------------------- weights
    def parameters(self):
        return self.w + self.b

    def _sync_kernel_weights(self):
        self.wk = [kernel_layout(w) for w in self.w]
        self.wt = [None] + [transposed_layout(w) for w in self.w[1:]]
        self._model = _native.TpCnnModel()
        for i in range(4):
            self._model.w[i] = self.wk[i].data_ptr()
            self._model.b[i] = self.b[i].data_ptr()
        self._model.kappa = self.kappa
        self._model.out_scale = self.out_scale

    def model(self) -> _native.TpCnnModel:
        """The C ABI view (pointers into this object's tensors; keep it alive)."""
        return self._model

    def state_dict(self):
        return {"nf": self.nf, "nb": self.nb, "kappa": self.kappa, "out_scale": self.out_scale,
                "w": [w.cpu() for w in self.w], "b": [b.cpu() for b in self.b]}

    def load_state_dict(self, sd):
        self.kappa = float(sd["kappa"])
        self.out_scale = float(sd.get("out_scale", 1.0 / self.kappa))
        self.w = [w.to(self.device).float() for w in sd["w"]]
        self.b = [b.to(self.device).float() for b in sd["b"]]
        self._sync_kernel_weights()

    def _buffers(self, batch):
        if batch not in self._bufs:
            self._bufs[batch] = CNNBuffers(self.lib, self.nf, self.nb, batch, self.device)
        return self._bufs[batch]

    # ----------------------------------------------------------- forward
    def filter(self, diag: torch.Tensor, keep=False) -> torch.Tensor:
        """(B, N) complex64 object diagonals → (13, B·N) complex64 filter."""
        B = diag.shape[0]
        N = self.nf * self.nb
        diag = diag.reshape(B, N).contiguous()
        if diag.dtype != torch.complex64:
            raise TypeError("diag must be complex64")
        buf = self._buffers(B)
        st = _stream(self.device)
        L = self.lib
        F = torch.empty((len(TAPS), B * N), dtype=torch.complex64, device=self.device)
        _native.check(L.tp_cnn_features(self.nf, self.nb, B, _ptr(diag), self.kappa, _ptr(buf.feat), st),
                      "tp_cnn_features")
        ins = [buf.feat, buf.a[0], buf.a[1]]
        for i in range(3):
            _native.check(L.tp_conv3x3_bf16(self.nf, self.nb, B, CHANNELS_IN if i == 0 else WIDTH, _native.CONV_RELU,
                                            _ptr(ins[i]), _ptr(self.wk[i]), _ptr(self.b[i]), None, _ptr(buf.a[i]), 1.0,
                                            st), "tp_conv3x3_bf16")
        _native.check(L.tp_conv3x3_bf16(self.nf, self.nb, B, WIDTH, _native.CONV_FILTER, _ptr(buf.a[2]),
                                        _ptr(self.wk[3]), _ptr(self.b[3]), None, _ptr(F), self.out_scale, st),
                      "tp_conv3x3_bf16")
        return F

    def apply(self, F: torch.Tensor, z: torch.Tensor, per_image: int, conj=False) -> torch.Tensor:
        """y_v = z_v + Σ_t F_t z_v(x + o_t); z (V, N) complex64."""
        z = z.contiguous()
        y = torch.empty_like(z)
        _native.check(self.lib.tp_cnn_filter_apply(self.nf, self.nb, z.shape[0], int(per_image), int(conj), _ptr(F),
                                                   _ptr(z), _ptr(y), _stream(self.device)), "tp_cnn_filter_apply")
        return y

    # ----------------------------------------------------------- backward
    def loss_and_grads(self, diag, z, target, scale, per_image):
        """L = Σ_v scale_v |y_v − target_v|² and d L / d (weights, biases), all on the GPU.

        diag (B, N), z and target (B·per_image, N) complex64, scale (B·per_image,) float32."""
        B = diag.shape[0]
        V = z.shape[0]
        if V != B * per_image:
            raise ValueError("z must hold per_image vectors for every diagonal")
        L = self.lib
        st = _stream(self.device)
        F = self.filter(diag)
        y = self.apply(F, z, per_image)
        r = y - target
        e = (r * scale[:, None]).contiguous()
        loss = torch.sum(scale[:, None] * (r.real ** 2 + r.imag ** 2))
        buf = self._buffers(B)
        _native.check(L.tp_cnn_filter_grad(self.nf, self.nb, B, int(per_image), _ptr(z.contiguous()), _ptr(e),
                                           self.out_scale, _ptr(buf.g[0]), st), "tp_cnn_filter_grad")
        gw, gb = [None] * 4, [None] * 4
        acts = [buf.feat, buf.a[0], buf.a[1], buf.a[2]]
        dys = [buf.g[3], buf.g[2], buf.g[1], buf.g[0]]  # gradient at each layer's output
        for i in (3, 2, 1, 0):
            cin = CHANNELS_IN if i == 0 else WIDTH
            dw = torch.zeros((9, cin, WIDTH), dtype=torch.float32, device=self.device)
            db = torch.zeros(WIDTH, dtype=torch.float32, device=self.device)
            _native.check(L.tp_conv3x3_wgrad(self.nf, self.nb, B, cin, _ptr(acts[i]), _ptr(dys[i]), _ptr(dw), _ptr(db),
                                             st), "tp_conv3x3_wgrad")
            gw[i] = wgrad_to_torch(dw, cin)
            gb[i] = db
            if i > 0:
                # gradient at layer i's input = conv(dy_i, W_i^T) masked by ReLU'(a_{i})
                _native.check(L.tp_conv3x3_bf16(self.nf, self.nb, B, WIDTH, _native.CONV_MASK, _ptr(dys[i]),
                                                _ptr(self.wt[i]), None, _ptr(acts[i]), _ptr(dys[i - 1]), 1.0, st),
                              "tp_conv3x3_bf16")
        return loss, gw, gb

    # ----------------------------------------------------------- training
    def train(self, pairs, steps: int = 300, slices_per_batch: int = 4, lr: float = 1e-3,
              seed: int = 0, log_every: int = 0, warmup: int = 20) -> TrainLog:
        """Adam on Σ‖y − sol‖² / Σ‖z0 − sol‖² over batches of `slices_per_batch`
        slices (all their probes), y the corrected preconditioner applied to the
        pair's residual; linear warm-up over `warmup` steps, then cosine decay
        to lr/20.  The loss is 1 for the plain preconditioner (F = 0).
        `pairs` is one :class:`TrainingPairs` or a list of them, visited in
        turn (e.g. right-hand-side pairs and white-noise pairs)."""
        sets = list(pairs) if isinstance(pairs, (list, tuple)) else [pairs]
        norms = []
        for ps in sets:
            # ‖sol − z0‖² per pair: the plain preconditioner's error, the loss unit
            delta = ps.sol - ps.z0
            norms.append((delta.real ** 2 + delta.imag ** 2).sum(-1))  # (S, P)
            del delta
        if self._adam is None:
            self._adam = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.parameters()]
            self._t = 0
        rng = np.random.default_rng(seed)
        log = TrainLog()
        b1, b2, eps = 0.9, 0.999, 1e-8
        for it in range(steps):
            pairs, norm = sets[it % len(sets)], norms[it % len(sets)]
            S, P, N = pairs.z0.shape
            idx = torch.from_numpy(rng.choice(S, size=min(slices_per_batch, S), replace=False)).to(self.device)
            d = pairs.diag.index_select(0, idx)
            z = pairs.z0.index_select(0, idx).reshape(-1, N)
            t = pairs.sol.index_select(0, idx).reshape(-1, N)
            # one scale per batch: loss = Σ‖y − sol‖² / Σ‖z0 − sol‖² (1 for the plain preconditioner)
            tot = norm.index_select(0, idx).sum().clamp_min(1e-30)
            scale = torch.full((z.shape[0],), 1.0, device=self.device) / tot
            scale = scale.float()
            loss, gw, gb = self.loss_and_grads(d, z, t, scale, P)
            grads = gw + gb
            self._t += 1
            if it < warmup:
                lr_t = lr * (it + 1) / warmup
            else:
                frac = (it - warmup) / max(steps - warmup, 1)
                lr_t = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * frac)))
            with torch.no_grad():
                for p, g, (m, v) in zip(self.parameters(), grads, self._adam):
                    m.mul_(b1).add_(g, alpha=1 - b1)
                    v.mul_(b2).addcmul_(g, g, value=1 - b2)
                    mh = m / (1 - b1 ** self._t)
                    vh = v / (1 - b2 ** self._t)
                    p.sub_(lr_t * mh / (vh.sqrt() + eps))
            self._sync_kernel_weights()
            if log_every and (it % log_every == 0 or it == steps - 1):
                log.losses.append(float(loss))
            log.steps += 1
        return log

    def relative_error(self, pairs: TrainingPairs, slices: Optional[List[int]] = None) -> dict:
        """‖y − sol‖ / ‖sol‖ of the learned and of the plain preconditioner on `pairs`."""
        S, P, N = pairs.z0.shape
        ks = range(S) if slices is None else slices
        num_l = num_p = den = 0.0
        for k in ks:
            F = self.filter(pairs.diag[k:k + 1])
            y = self.apply(F, pairs.z0[k], 0)
            num_l += float(torch.sum(torch.abs(y - pairs.sol[k]) ** 2))
            num_p += float(torch.sum(torch.abs(pairs.z0[k] - pairs.sol[k]) ** 2))
            den += float(torch.sum(torch.abs(pairs.sol[k]) ** 2))
        return {"learned": math.sqrt(num_l / den), "plain": math.sqrt(num_p / den)}


def default_kappa(k: float, dz: float, amplitude: float) -> float:
    """Scale that maps the object diagonal of an index perturbation of size
    `amplitude` to features of order one: |d| ≈ (dz/2)·k·|δn|."""
    return 1.0 / max(0.5 * dz * k * amplitude, 1e-30)
