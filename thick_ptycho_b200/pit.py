"""Space-time (parallel-in-time) solve of the 2D paraxial march on the GPU.

Drop-in for the reference's ``PWEFullPinTSolver``
(``forward_model/pwe/solvers/full_pint.py:71-275``): the L = nz − 1 steps
form one block-bidiagonal system ``M u = b`` (``_pint_utils.py:27-54``; the
probe enters through ``B u_0`` alone, as in the reference's full-system
solvers) solved by restarted GMRES right-preconditioned with the
α-block-circulant preconditioner of ``_pint_utils.py:57-205``.  Every probe's
Krylov space is built at once in ``tp_pit_solve`` (libtpcuda): the space-time
matvec, Bluestein z-DFTs on the shared-memory FFT, the L shifted tridiagonal
block solves, and fp64 Gram–Schmidt inner products on the GPU; the Givens
rotations and the small least-squares solves on the host.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _native
from .cn2d import CN2D
from .solver import PWEGpuSolver


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class PiT2D:
    """PiT engine for one 2D geometry (N rows, nz nodes)."""

    def __init__(self, engine: CN2D, alpha=1e-2, atol=1e-8, rtol=1e-5, restart=20, max_cycles=1000):
        self.engine = engine
        self.lib = engine.lib
        self.device = engine.device
        self.N, self.nz, self.L = engine.n, engine.nz, engine.L
        self.alpha, self.atol, self.rtol = float(alpha), float(atol), float(rtol)
        self.restart, self.max_cycles = int(restart), int(max_cycles)
        self._ws = None
        self._ws_P = None
        self.iters = None
        self.resid = None

    def workspace(self, P):
        if self._ws is None or self._ws_P != P:
            nbytes = int(self.lib.tp_pit_workspace_bytes(self.N, self.nz, P, self.restart))
            if nbytes == 0:
                raise ValueError(f"PiT does not support N={self.N}, nz={self.nz}, restart={self.restart}")
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws_P = P
        return self._ws

    def solve(self, field: torch.Tensor, probes: Optional[torch.Tensor] = None, rhs: Optional[torch.Tensor] = None,
              u0: Optional[torch.Tensor] = None, num_probes: Optional[int] = None, mode="forward") -> torch.Tensor:
        """The field at steps 1..L, (P, L, N) complex64; ``u0`` is the initial
        guess (a warm start, e.g. an earlier solution).  ``mode`` "adjoint"
        solves the reference's adjoint system (conjugate-transposed blocks,
        z-flipped conjugate object term, the forward preconditioner)."""
        if mode not in ("forward", "adjoint"):
            raise ValueError(f"PiT mode must be 'forward' or 'adjoint' (got {mode!r})")
        field = self.engine._check_field(field)
        P = int(num_probes if num_probes is not None else (probes.shape[0] if probes is not None else rhs.shape[0]))
        for name, t, shp in (("probes", probes, (P, self.N)), ("rhs", rhs, (P, self.L, self.N)),
                             ("u0", u0, (P, self.L, self.N))):
            if t is not None and (t.dtype != torch.complex64 or tuple(t.shape) != shp or not t.is_contiguous()):
                raise ValueError(f"{name} must be contiguous complex64 of shape {shp}")
        u = u0.clone() if u0 is not None else torch.zeros((P, self.L, self.N), dtype=torch.complex64,
                                                          device=self.device)
        iters = (ctypes.c_int32 * P)()
        resid = (ctypes.c_double * P)()
        a = _native.TpPitArgs()
        a.num_probes, a.restart, a.max_cycles = P, self.restart, self.max_cycles
        a.mode = _native.MODES[mode]
        a.alpha, a.rtol, a.atol = self.alpha, self.rtol, self.atol
        a.probes, a.rhs, a.u = _ptr(probes), _ptr(rhs), _ptr(u)
        a.iters = ctypes.cast(iters, ctypes.POINTER(ctypes.c_int32))
        a.resid = ctypes.cast(resid, ctypes.POINTER(ctypes.c_double))
        ws = self.workspace(P)
        dtype = _native.C128 if field.dtype == torch.complex128 else _native.C64
        o = self.engine.op()
        rc = self.lib.tp_pit_solve(ctypes.byref(o), _ptr(field), dtype, ctypes.byref(a), _ptr(ws), ws.numel(),
                                   _stream(self.device))
        _native.check(rc, "tp_pit_solve")
        self.iters = list(iters)
        self.resid = list(resid)
        return u


class PWEGpuPiTSolver(PWEGpuSolver):
    """Drop-in for ``PWEFullPinTSolver`` (2D; modes "forward" and "adjoint") on one B200.

    Same constructor arguments (``alpha``, ``atol``) and ``solve`` /
    ``_solve_single_probe`` results; ``gmres_iterations`` holds the Arnoldi
    steps of the last solve per probe.  ``rtol`` (default 1e-6) is the
    relative residual at which GMRES stops: the reference stops at 1e-5 in
    complex128 (``full_pint.py:250``), whose solution then sits ~1e-6 from the
    exact one; stopping ten times tighter keeps this complex64 solve within
    1e-5 of both.  Like the reference's per-mode
    ``u0_cache``, the last solution of a mode warm-starts that mode's next
    solve for the same ``n`` object (per probe here: the probes are solved together; the
    reference keeps the preconditioned unknown, this keeps u itself).
    """

    def __init__(self, simulation_space, ptycho_probes, bc_type="impedance", results_dir="", use_logging=False,
                 verbose=False, log=None, alpha=1e-2, atol=1e-8, test_bcs=None, device=None, restart=20, rtol=1e-6):
        super().__init__(simulation_space, ptycho_probes, bc_type=bc_type, results_dir=results_dir,
                         use_logging=use_logging, verbose=verbose, log=log, test_bcs=test_bcs, device=device)
        if self.dimension != 2:
            raise NotImplementedError("the GPU PiT solver covers 2D simulation spaces")
        if test_bcs is not None:
            raise NotImplementedError("the GPU PiT solver does not take exact test boundary data")
        self.alpha, self.atol = float(alpha), float(atol)
        self.pit = PiT2D(self.engine, alpha=alpha, atol=atol, rtol=rtol, restart=restart)
        self._warm = {}  # mode -> (n object, u)
        self.gmres_iterations = None

    def _rhs_rows(self, rhs_block) -> np.ndarray:
        """``rhs_block`` as (L, N) slice-major: an (N, L) array, or the flat
        space-time vector in the reference's column-major (N, L) order."""
        rb = np.asarray(rhs_block)
        if rb.ndim == 1:
            rb = rb.reshape(self.block_size, self.nz - 1, order="F")
        return np.ascontiguousarray(rb.reshape(self.block_size, self.nz - 1).T)

    def _pit(self, n, probes_dev, rhs=None, mode="forward"):
        if n is None:
            n = self.simulation_space.refractive_index_empty
        field = self._field_device(n)
        P = probes_dev.shape[0] if probes_dev is not None else rhs.shape[0]
        u0 = None
        warm = self._warm.get(mode)
        if warm is not None and warm[0] is n and tuple(warm[1].shape)[0] == P:
            u0 = warm[1]
        u = self.pit.solve(field, probes=probes_dev, rhs=rhs, u0=u0, num_probes=P, mode=mode)
        self._warm[mode] = (n, u)
        self.gmres_iterations = self.pit.iters
        return u

    @staticmethod
    def _check_mode(mode):
        if mode not in ("forward", "adjoint"):
            raise NotImplementedError(f"the PiT solver supports modes 'forward' and 'adjoint' (got {mode!r})")

    def solve(self, n=None, mode="forward", rhs_block=None, probes=None, **kwargs) -> np.ndarray:
        """All probes, shape (proj, angle, probes, N, nz) complex128 (``full_pint.py:179-275``);
        in mode "adjoint" the reference's adjoint system (``full_pint.py:140-166``)."""
        self._check_mode(mode)
        if self.num_projections != 1:
            raise NotImplementedError("the GPU PiT solver covers one projection")
        count = self.num_angles * self.num_probes
        pr = self._probes_device(self.probes if probes is None else probes, count)
        rhs = None
        pr_in = pr
        if rhs_block is not None:
            rows = self._rhs_rows(rhs_block)
            rhs = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(rows, (count, self.nz - 1, self.block_size)))
                                   .astype(np.complex64)).to(self.device)
            pr_in = None
        u = self._pit(n, pr_in, rhs, mode)
        full = torch.cat([pr[:, None, :], u], dim=1).permute(0, 2, 1)
        out = np.zeros((self.num_projections, self.num_angles, self.num_probes, *self.effective_shape), dtype=complex)
        out[0] = full.cpu().numpy().astype(np.complex128).reshape(self.num_angles, self.num_probes,
                                                                   *self.effective_shape)
        return out

    def _solve_single_probe(self, scan_idx=0, proj_idx=0, probe=None, n=None, mode="forward", rhs_block=None):
        """One probe, shape (N, nz) (``full_pint.py:179-275``): with ``rhs_block``
        it replaces b (the reference's behaviour), else b = [B u_0, 0, …] (the
        forward B in both modes, as the reference's ``probe_contribution``)."""
        self._check_mode(mode)
        pr = self._probes_device(probe if probe is not None else np.zeros(self.block_size), 1)
        rhs = None
        if rhs_block is not None:
            rhs = torch.from_numpy(self._rhs_rows(rhs_block)[None].astype(np.complex64)).to(self.device)
        u = self._pit(n, None if rhs is not None else pr, rhs, mode)
        full = torch.cat([pr[:, None, :], u], dim=1)[0].T
        return full.cpu().numpy().astype(np.complex128)
