"""Forward + exact-adjoint gradient of the 2D paraxial model on the GPU.

The reference obtains its gradient from one adjoint march per probe plus a
host-side contraction (``reconstruction/pwe_reconstructor.py:100-164``).
Here one batched forward march stores the field, one batched exact-adjoint
march (the transpose of the forward recursion, ``TP_MODE_ADJOINT_EXACT``)
accumulates ``Σ_p λ_s conj(u_s + u_{s−1})`` over probes inside the kernel,
and ``tp_cn2d_grad_to_n`` maps it onto the nodes of n.

Gradients follow torch's complex convention ``∂ℓ/∂Re + i ∂ℓ/∂Im``.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .cn2d import CN2D


def _as_device(x, device, dtype):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype, non_blocking=True)
    return torch.from_numpy(np.ascontiguousarray(x)).to(device=device, dtype=dtype, non_blocking=True)


def amplitude_residual(exit_waves: torch.Tensor, amplitude: torch.Tensor):
    """Loss ``Σ(|F e| − a)²`` and its gradient w.r.t. e (torch convention).

    Equals ``2N(e − P_GS(e))`` with P_GS the reference's modulus projection
    (``base_reconstructor.py:171-207``).  Computed in complex128.
    """
    n = exit_waves.shape[-1]
    U = torch.fft.fft(exit_waves.to(torch.complex128), dim=-1)
    mag = U.abs()
    a = amplitude.to(torch.float64)
    loss = torch.sum((mag - a) ** 2)
    safe = torch.where(mag > 0, mag, torch.ones_like(mag))
    gU = torch.where(mag > 0, 2 * (mag - a) / safe, torch.zeros_like(mag)) * U
    return loss, (n * torch.fft.ifft(gU, dim=-1)).to(torch.complex64)


class PWEGradient2D:
    """Amplitude-loss gradient of a 2D geometry, all probes batched.

    ``geometry`` is a reference ``SimulationSpace2D`` or a
    :class:`~thick_ptycho_b200.geometry.SimulationGeometry`.
    """

    def __init__(self, geometry, bc_type="impedance", device=None):
        self.geometry = geometry
        self.engine = CN2D(
            geometry.block_size, geometry.nz, geometry.k, geometry.dx, geometry.dz, bc_type,
            empty_px=int(getattr(geometry, "empty_space_px", 0) or 0),
            exact_ref_coeff=bool(getattr(geometry, "exact_ref_coeff", False)), device=device,
        )
        self.device = self.engine.device
        self._ff = self.engine.new_factor_buffer()
        self._fa = self.engine.new_factor_buffer()
        self._store = None
        self._grad_c = torch.empty((self.engine.L, self.engine.n), dtype=torch.complex64, device=self.device)

    def _store_for(self, P):
        if self._store is None or self._store.shape[0] != P:
            self._store = self.engine.new_store(P)
        return self._store

    def forward(self, field: torch.Tensor, probes: torch.Tensor, is_delta=False, exit_out=None):
        """Forward march storing the full field; returns (factor set, exit)."""
        P = probes.shape[0]
        fs = self.engine.factor(field, "forward", is_delta, out=self._ff)
        ex = exit_out if exit_out is not None else torch.empty((P, self.engine.n), dtype=torch.complex64, device=self.device)
        self.engine.march(fs, P, probes=probes, u_store=self._store_for(P), exit_out=ex)
        return ex

    def backward(self, field: torch.Tensor, exit_grad: torch.Tensor, is_delta=False) -> torch.Tensor:
        """Exact adjoint from the exit-wave gradient; returns ∂ℓ/∂n (n_obj, nz)."""
        P = exit_grad.shape[0]
        fa = self.engine.factor(field, "adjoint_exact", is_delta, out=self._fa)
        self._grad_c.zero_()
        self.engine.march(fa, P, src_exit=exit_grad.contiguous(), u_fwd=self._store_for(P), grad_c=self._grad_c)
        return self.engine.grad_to_n(self._grad_c, field if self.engine.exact_ref_coeff else None, is_delta)

    def loss_and_grad(self, n, probes, amplitude, grad_out: Optional[torch.Tensor] = None):
        """One forward + adjoint pass: ``(loss, ∂loss/∂n)``.

        ``n``: refractive index (n_obj, nz) as the reference's solvers take it
        (complex128); ``probes``: (P, N); ``amplitude``: measured ``√I`` (P, N).
        Host inputs are copied to the device; if ``grad_out`` is a host tensor
        the gradient is copied back into it.  Returns a float loss.
        """
        field = _as_device(n, self.device, torch.complex128)
        pr = _as_device(probes, self.device, torch.complex64)
        amp = _as_device(amplitude, self.device, torch.float64)
        ex = self.forward(field, pr)
        loss, ge = amplitude_residual(ex, amp)
        g = self.backward(field, ge)
        if grad_out is not None:
            grad_out.copy_(g, non_blocking=True)
        return float(loss.item()), g


class PWEFunction(torch.autograd.Function):
    """``exit = PWE(field)`` with the exact adjoint as its backward.

    ``field`` is n (complex128) or ``n − 1`` (complex64/128 with
    ``is_delta=True``); ``probes`` (P, N) complex64; returns exit waves
    (P, N) complex64.
    """

    @staticmethod
    def forward(ctx, field, probes, grad_engine: PWEGradient2D, is_delta: bool = False):
        ex = grad_engine.forward(field.detach().contiguous(), probes.detach().to(torch.complex64).contiguous(), is_delta)
        ctx.save_for_backward(field)
        ctx.engine = grad_engine
        ctx.is_delta = is_delta
        return ex

    @staticmethod
    def backward(ctx, grad_exit):
        (field,) = ctx.saved_tensors
        g = ctx.engine.backward(field.detach().contiguous(), grad_exit.to(torch.complex64).contiguous(), ctx.is_delta)
        return g.to(field.dtype), None, None, None
