"""The reference's NLCG reconstruction loop on the GPU (2D).

Restates ``ReconstructorPWE.reconstruct`` (``reconstruction/pwe_reconstructor.py:
229-368``) for one projection and angle, with its own step-size and direction
rules, so that a reconstruction follows the reference's trajectory:

* forward model: one batched forward march storing the full field
  (``compute_forward_model``, ``:85-97``);
* exit error at the last slice, with the Gerchberg–Saxton modulus projection
  (``base_reconstructor.py:87-207``) or against known exit waves;
* gradient: one batched reference-adjoint march (mode "adjoint", the
  reference's inexact adjoint) and the contraction with ``grad_A u``
  (``compute_grad_least_squares``, ``:100-164``; ``tp_cn2d_ref_gradient``);
* step sizes ``compute_alphak`` (``:166-219``): the reference solves, per probe,
  a forward march that starts from the probe and adds the source
  ``grad_A u_p`` (times i for the imaginary part); by linearity both solves
  are the stored exit wave plus one batched zero-start march with the source
  (``tp_cn2d_alpha_source``), whose exit is added with weight 1 or i;
* Polak–Ribière / Fletcher–Reeves ``β`` (``compute_betak``, ``:221-228``) and the
  direction update on the device.

Everything that touches a field runs in libtpcuda kernels; the per-iteration
scalars (step sizes, β) are float64 reductions of device vectors.
"""

from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np
import torch

from . import _native, heads
from .cn2d import CN2D, _ptr, _stream
from .heads import fft_plannable


def _projection_error(ex: torch.Tensor, data: torch.Tensor) -> torch.Tensor:
    """``e = exit − ifft(√I · F e/|F e|)`` (the reference's modulus projection; phase 0 where F e = 0)."""
    N = ex.shape[-1]
    if fft_plannable(N):
        _, g = heads.amplitude_residual(ex.contiguous(), torch.sqrt(data).to(torch.float32))
        return g / (2 * N)  # F^H[2(|Fe| − a) Fe/|Fe|] = 2N (e − P(e))
    f = torch.fft.fft(ex.to(torch.complex128), dim=-1)
    mag = f.abs()
    mag = torch.where(mag == 0, torch.ones_like(mag), mag)
    em = torch.fft.ifft(torch.sqrt(data) * (f / mag), dim=-1)
    return (ex.to(torch.complex128) - em).to(torch.complex64)


class ReconstructorPWEGpu:
    """NLCG reconstruction of a 2D refractive index from far-field data.

    ``geometry``: the simulation space (nx, nz, k, dx, dz as the reference's);
    ``data``: (P, N) far-field intensities (``phase_retrieval=True``) or known
    exit waves; ``probes``: (P, N).
    """

    def __init__(self, geometry, data, probes, phase_retrieval=True, bc_type="impedance", device=None):
        if not torch.cuda.is_available():
            raise _native.NativeLibraryError("the GPU reconstructor needs a CUDA device (no CPU fallback)")
        self.device = torch.device(device if device is not None else "cuda")
        self.geometry = geometry
        N = int(geometry.effective_shape[0]) if hasattr(geometry, "effective_shape") else int(geometry.nx)
        if int(getattr(geometry, "empty_space_px", 0)) != 0 or bool(getattr(geometry, "exact_ref_coeff", False)):
            raise NotImplementedError("the GPU NLCG loop needs exact_ref_coeff=False and no empty-space padding")
        self.engine = CN2D(N, geometry.nz, geometry.k, geometry.dx, geometry.dz, bc_type, device=self.device)
        self.N, self.nz, self.L = N, int(geometry.nz), int(geometry.nz) - 1
        self.phase_retrieval = bool(phase_retrieval)
        dt = torch.float64 if phase_retrieval else torch.complex64
        self.data = torch.as_tensor(np.ascontiguousarray(data)).to(self.device, dt).reshape(-1, N)
        self.probes = torch.as_tensor(np.ascontiguousarray(probes)).to(self.device, torch.complex64).reshape(-1, N)
        self.P = self.probes.shape[0]
        e = self.engine
        self._u = e.new_store(self.P)
        self._lam = e.new_store(self.P)
        self._src = torch.empty((self.P, self.L, N), dtype=torch.complex64, device=self.device)
        self._ex = torch.empty((self.P, N), dtype=torch.complex64, device=self.device)
        self._dex = torch.empty((self.P, N), dtype=torch.complex64, device=self.device)
        self._gre = torch.empty(self.L * N, dtype=torch.float32, device=self.device)
        self._gim = torch.empty(self.L * N, dtype=torch.float32, device=self.device)
        self._ff = e.new_factor_buffer()
        self._fa = e.new_factor_buffer()

    # ------------------------------------------------------------ pieces
    def forward_model(self, nk: torch.Tensor):
        e = self.engine
        ff = e.factor(nk, "forward", out=self._ff)
        e.march(ff, self.P, probes=self.probes, u_store=self._u, exit_out=self._ex)
        return ff

    def exit_error(self) -> torch.Tensor:
        if self.phase_retrieval:
            return _projection_error(self._ex, self.data)
        return (self._ex - self.data).contiguous()

    def gradient(self, nk: torch.Tensor, err: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        """The reference's (grad_re, grad_im), z-major (L·N,), float32."""
        e = self.engine
        fa = e.factor(nk, "adjoint", out=self._fa)
        e.march(fa, self.P, src_exit=err.contiguous(), u_store=self._lam)
        rc = e.lib.tp_cn2d_ref_gradient(e.op(), self.P, _ptr(self._u), _ptr(self._lam), _ptr(self._gre),
                                        _ptr(self._gim), _stream(self.device))
        _native.check(rc, "tp_cn2d_ref_gradient")
        return self._gre, self._gim

    def step_sizes(self, ff, g_re, g_im, d_re, d_im) -> Tuple[float, float]:
        """``compute_alphak`` for the real and the imaginary part."""
        e = self.engine
        rc = e.lib.tp_cn2d_alpha_source(e.op(), self.P, _ptr(self._u), _ptr(self._src), _stream(self.device))
        _native.check(rc, "tp_cn2d_alpha_source")
        e.march(ff, self.P, src_probe=self._src, exit_out=self._dex)
        ex, dex = self._ex.to(torch.complex128), self._dex.to(torch.complex128)
        N = self.N
        out = []
        for g, d, w in ((g_re, d_re, 1.0), (g_im, d_im, 1j)):
            d64 = d.to(torch.float64)
            dl = d64[-N:].to(torch.complex128)
            dp = -((ex + w * dex) @ dl)  # (P,)
            den = float(torch.sum(dp.abs() ** 2))
            num = float(torch.dot(d64, g.to(torch.float64)))
            out.append(-(num / den) if den > 0 else 0.0)
        return out[0], out[1]

    @staticmethod
    def beta(g, g_old) -> float:
        g, g_old = g.to(torch.float64), g_old.to(torch.float64)
        nrm = float(torch.dot(g_old, g_old))
        pr = float(torch.dot(g, g - g_old)) / nrm
        fr = float(torch.dot(g, g)) / nrm
        return min(fr, max(pr, 0.0))

    # ------------------------------------------------------------ loop
    def reconstruct(self, max_iters=10, tol=1e-8, n_initial=None, fixed_step_size=None
                    ) -> Tuple[np.ndarray, List[float]]:
        """``reconstruct`` of the reference: returns (n, residuals)."""
        N, L = self.N, self.L
        if n_initial is None:
            n0 = np.ones((N, self.nz), dtype=complex) * complex(getattr(self.geometry, "n_medium", 1.0))
        else:
            n0 = np.array(n_initial, dtype=complex)
        nk = torch.from_numpy(n0).to(self.device)
        residual: List[float] = []
        d_re = d_im = g_re_old = g_im_old = None
        for i in range(max_iters):
            ff = self.forward_model(nk)
            err = self.exit_error()
            residual.append(float(torch.sqrt(torch.mean(err.abs().to(torch.float64) ** 2))))
            if residual[i] < tol:
                break
            g_re, g_im = (x.clone() for x in self.gradient(nk, err))
            if i == 0:
                d_re, g_re_old = -g_re, g_re
                d_im, g_im_old = -g_im, g_im
            if fixed_step_size is not None:
                a_re = a_im = -float(fixed_step_size) / (i + 1)
            else:
                a_re, a_im = self.step_sizes(ff, g_re, g_im, d_re, d_im)
            upd = (a_re * d_re.to(torch.float64)).reshape(L, N).T + 1j * (a_im * d_im.to(torch.float64)).reshape(L, N).T
            nk[:, 1:] += upd
            b_re, b_im = self.beta(g_re, g_re_old), self.beta(g_im, g_im_old)
            d_re, g_re_old = -g_re + b_re * d_re, g_re
            d_im, g_im_old = -g_im + b_im * d_im, g_im
        return nk.cpu().numpy(), residual


def gradient_descent_3d(grad3d, n0, probes, amplitude, iters=20, step=None, max_update=5e-5):
    """Gradient descent on the 3D amplitude loss with :class:`cn3d.PWEGradient3D`:
    ``n ← n − η ∂loss/∂n`` (torch convention ∂/∂Re + i ∂/∂Im).  ``η`` is `step`,
    or chosen at the first iteration so that the largest update is `max_update`.
    Returns (n, losses, Krylov iterations per solve of each iteration)."""
    eng = grad3d.engine
    n = torch.as_tensor(np.ascontiguousarray(n0) if not isinstance(n0, torch.Tensor) else n0)
    n = n.to(eng.device, torch.complex128).reshape(eng.N, eng.nz).clone()
    eta = step
    losses, its = [], []
    eng.read_stats()
    for _ in range(iters):
        loss, g = grad3d.loss_and_grad(n, probes, amplitude)
        st = eng.read_stats()
        losses.append(loss)
        its.append(st["iterations"] / max(st["solves"], 1))
        g = g.reshape(eng.N, eng.nz).to(torch.complex128)
        if eta is None:
            gmax = float(g.abs().max())
            eta = max_update / gmax if gmax > 0 else 0.0
        n -= eta * g
    return n, losses, its
