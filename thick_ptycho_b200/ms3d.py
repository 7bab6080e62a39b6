"""Angular-spectrum multislice on the GPU in 3D.

The reference's multislice solver stops at 2D (``ms_solver.py:28-31``); this
engine runs the same propagator (``ms_solver.py:49-159``) on an (nx, ny)
transverse grid with a two-dimensional transverse wavenumber:
``ψ ← IFFT2(H·FFT2(ψ·T_z))``, ``T_z = exp(ik(n_z − n_med)dz)``,
``H = exp(i(√max(k² − kx² − ky², 0) − k)dz)``.  Slices are the C-order
flattening of (nx, ny), the reference's layout for 3D fields; the index field
is (nx, ny, nz) or (nx·ny, nz).  :class:`MS3DFunction` gives exit waves with
the hand-written adjoint march as its backward.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class MS3D:
    """3D multislice engine for one geometry (nx × ny transverse, nz nodes)."""

    def __init__(self, nx, ny, nz, k, dx, dy, dz, n_medium=1.0, device=None):
        if not torch.cuda.is_available():
            raise _native.NativeLibraryError("MS3D needs a CUDA device (there is no CPU fallback)")
        self.lib = _native.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.nx, self.ny, self.nz, self.L = int(nx), int(ny), int(nz), int(nz) - 1
        self.N = self.nx * self.ny
        o = _native.TpMs3dOp()
        o.n1, o.n2, o.nz = self.nx, self.ny, self.nz
        o.k, o.d1, o.d2, o.dz = float(k), float(dx), float(dy), float(dz)
        nm = complex(n_medium)
        o.n_medium = (ctypes.c_double * 2)(nm.real, nm.imag)
        self._op = o
        self.k, self.dz = float(k), float(dz)
        self._ws = None
        self._ws_P = None

    def workspace(self, P: int) -> torch.Tensor:
        if self._ws is None or self._ws_P != P:
            nbytes = int(self.lib.tp_ms3d_workspace_bytes(self.nx, self.ny, P))
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws_P = P
        return self._ws

    def transmission(self, field: torch.Tensor) -> torch.Tensor:
        """``T_z − 1`` (L, N) complex64 from n (nx, ny, nz) or (N, nz), complex128/64."""
        if field.dim() == 3:
            field = field.reshape(self.N, field.shape[-1])
        if tuple(field.shape) != (self.N, self.nz):
            raise ValueError(f"index field has shape {tuple(field.shape)}, expected {(self.N, self.nz)}")
        field = field.contiguous()
        dt = _native.C128 if field.dtype == torch.complex128 else _native.C64
        T = torch.empty((self.L, self.N), dtype=torch.complex64, device=self.device)
        _native.check(self.lib.tp_ms3d_transmission(ctypes.byref(self._op), _ptr(field), dt, _ptr(T),
                                                    _stream(self.device)), "tp_ms3d_transmission")
        return T

    def march(self, T, probes, u_store=None, exit_out=None):
        """Probes (P, N) or (P, nx, ny) complex64; u_store (P, nz, N); exit_out (P, N)."""
        P = probes.shape[0]
        pr = probes.reshape(P, self.N).contiguous()
        ws = self.workspace(P)
        _native.check(self.lib.tp_ms3d_march(ctypes.byref(self._op), _ptr(T), _ptr(pr), P, _ptr(u_store),
                                             _ptr(exit_out), _ptr(ws), ws.numel(), _stream(self.device)),
                      "tp_ms3d_march")

    def backward(self, T, u_fwd, src_exit, grad_t):
        """Adjoint march: grad_t (L, N) += Σ_p conj(T_z u_z) g_z."""
        P = src_exit.shape[0]
        ws = self.workspace(P)
        _native.check(self.lib.tp_ms3d_backward(ctypes.byref(self._op), _ptr(T), _ptr(u_fwd),
                                                _ptr(src_exit.reshape(P, self.N).contiguous()), P, _ptr(grad_t),
                                                _ptr(ws), ws.numel(), _stream(self.device)), "tp_ms3d_backward")

    def grad_to_n(self, grad_t: torch.Tensor) -> torch.Tensor:
        """(L, N) accumulator → torch-convention ∂loss/∂n of shape (N, nz)."""
        g = torch.zeros((self.N, self.nz), dtype=torch.complex64, device=self.device)
        g[:, :-1] = (np.conj(1j * self.k * self.dz) * grad_t).T
        return g


class MS3DFunction(torch.autograd.Function):
    """``exit = MS3D(n)`` with the adjoint multislice march as backward.

    ``field``: (N, nz) index; ``probes``: (P, N); returns exit waves (P, N).
    """

    @staticmethod
    def forward(ctx, field, probes, engine: MS3D):
        P = probes.shape[0]
        T = engine.transmission(field.detach())
        st = torch.empty((P, engine.nz, engine.N), dtype=torch.complex64, device=engine.device)
        ex = torch.empty((P, engine.N), dtype=torch.complex64, device=engine.device)
        engine.march(T, probes.detach().to(torch.complex64), u_store=st, exit_out=ex)
        ctx.save_for_backward(field)
        ctx.engine, ctx.T, ctx.st = engine, T, st
        return ex

    @staticmethod
    def backward(ctx, grad_exit):
        (field,) = ctx.saved_tensors
        e = ctx.engine
        gt = torch.zeros((e.L, e.N), dtype=torch.complex64, device=e.device)
        e.backward(ctx.T, ctx.st, grad_exit.to(torch.complex64).contiguous(), gt)
        return e.grad_to_n(gt).reshape(field.shape).to(field.dtype), None, None
