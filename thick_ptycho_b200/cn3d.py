"""Batched 3D Crank–Nicolson propagation on the GPU (host side).

:class:`CN3D` holds the 5-point operator of one 3D geometry (restated from the
reference's ``operator_matrices.py:75-126`` / ``boundary_conditions.py:96-130``
in :func:`operators.operator_2d_diagonals`) and calls ``tp_cn3d_march``:
every slice is solved by FFT-preconditioned BiCGStab in delta form, all probes
at once.  Vectors follow the reference's flattening of (nx, ny) arrays.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _native
from .operators import BCCoefficients, normalize_bc, operator_2d_diagonals


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _c2(z: complex):
    return (ctypes.c_double * 2)(z.real, z.imag)


class CN3D:
    """One 3D geometry: nx × ny transverse (N = nx·ny), nz nodes."""

    def __init__(self, nx, ny, nz, k, dx, dy, dz, bc_type="impedance", exact_ref_coeff=False, device=None,
                 check=False):
        """``check=True`` runs the geometry on the complex128 check build
        (``libtpcuda_c128.so``): operator, vectors, stores and sources
        complex128, the FFT-preconditioned (not the learned) march only."""
        if not torch.cuda.is_available():
            raise _native.NativeLibraryError("CN3D needs a CUDA device (there is no CPU fallback)")
        self.check = bool(check)
        self.lib = _native.load_check() if self.check else _native.load()
        self.cdtype = torch.complex128 if self.check else torch.complex64
        self.device = torch.device(device if device is not None else "cuda")
        self.nx, self.ny, self.nz, self.L = int(nx), int(ny), int(nz), int(nz) - 1
        self.N = self.nx * self.ny
        self.k, self.dz = float(k), float(dz)
        self.bc_type = normalize_bc(bc_type)
        self.exact_ref_coeff = bool(exact_ref_coeff)
        co = BCCoefficients.make(self.k, dx, dz, self.bc_type, dy=dy, dimension=3)
        diags = operator_2d_diagonals(self.nx, self.ny, co, self.bc_type)
        npc = np.complex128 if self.check else np.complex64
        self._diags = [torch.from_numpy(d.astype(npc)).to(self.device) for d in diags]
        self.co = co
        self._ws = None
        self._ws_P = None
        self._lws = None
        self._lws_P = None
        self.stats = torch.zeros(5, dtype=torch.int32, device=self.device)
        self.fallbacks = 0
        # 0: each march runs as one CUDA graph with device-side step and
        # iteration loops; 1: step by step (host loop)
        self.launch = 0
        # kernel choice (tp_cn3d_march_args.kernels; the same arithmetic):
        # 0 = automatic; bit 0 = Stockham transforms always, bit 1 = the
        # stencil kernels with per-thread loads instead of tensor-memory copies,
        # bit 2 = the learned filter by register shuffles instead of bulk-staged rows
        self.kernels = 0

    def op(self, is_delta=False) -> _native.TpCn3dOp:
        o = _native.TpCn3dOp()
        o.nf, o.nb, o.nz = self.nx, self.ny, self.nz
        o.exact_ref_coeff, o.field_is_delta = int(self.exact_ref_coeff), int(is_delta)
        o.k, o.dz = self.k, self.dz
        o.mu_x, o.mu_y = _c2(self.co.mu_x), _c2(self.co.mu_y)
        o.kc, o.kw, o.ke, o.ks, o.kn = (ctypes.c_void_p(d.data_ptr()) for d in self._diags)
        return o

    def workspace(self, P):
        if self._ws is None or self._ws_P != P:
            nbytes = int(self.lib.tp_cn3d_workspace_bytes(self.N, P))
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws_P = P
        return self._ws

    def learned_workspace(self, P):
        if self._lws is None or self._lws_P != P:
            nbytes = int(self.lib.tp_cn3d_learned_ws_bytes(self.nx, self.ny, self.nz, P))
            self._lws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._lws_P = P
        return self._lws

    def new_store(self, P):
        return torch.empty((P, self.nz, self.N), dtype=self.cdtype, device=self.device)

    def march(self, field: torch.Tensor, num_probes: int, mode="forward", probes=None, src_shared=None, src_exit=None,
              u_store=None, exit_out=None, u_fwd=None, grad_c=None, tol=1e-6, max_iter=20, precond=True,
              host_check=True, is_delta=False, model=None, train=None, train_every=0, fallback=True,
              reuse_filters=False):
        """One batched march; tensors complex64 (complex128 in the check build;
        field complex128/complex64 (N, nz)).

        ``precond``: True/"fft" (periodic FFT preconditioner), False/"none", or
        "learned" (FFT preconditioner with the per-pixel correction of
        ``model``, a :class:`learned.LearnedPreconditioner`).  With "learned"
        and ``fallback``, a march in which any solve missed its tolerance
        (judged by the true residual) is re-run with the plain FFT
        preconditioner; ``self.fallbacks`` counts such re-runs.  ``train`` is a
        :class:`learned.TrainingPairs` whose buffers receive the pair of every
        ``train_every``-th step (see :func:`generate_pairs`)."""
        if precond == "learned":
            if model is None:
                raise ValueError('precond="learned" needs a model')
            if fallback:
                before = int(self.stats[2].item())
                self._march(field, num_probes, mode, probes, src_shared, src_exit, u_store, exit_out, u_fwd, grad_c, tol,
                            max_iter, 2, host_check, is_delta, model, train, train_every, reuse_filters)
                if int(self.stats[2].item()) > before:
                    self.fallbacks += 1
                    if grad_c is not None:
                        raise RuntimeError("learned adjoint solve missed its tolerance; re-run with precond=True "
                                           "(the gradient accumulator already holds a partial sum)")
                    self._march(field, num_probes, mode, probes, src_shared, src_exit, u_store, exit_out, u_fwd,
                                grad_c, tol, max_iter, 1, host_check, is_delta, None, train, train_every)
                return
            code = 2
        elif precond in (True, "fft", 1):
            code = 1
        elif precond in (False, "none", 0, None):
            code = 0
        else:
            raise ValueError(f"unknown preconditioner {precond!r}")
        self._march(field, num_probes, mode, probes, src_shared, src_exit, u_store, exit_out, u_fwd, grad_c, tol,
                    max_iter, code, host_check, is_delta, model, train, train_every, reuse_filters)

    def _march(self, field, num_probes, mode, probes, src_shared, src_exit, u_store, exit_out, u_fwd, grad_c, tol,
               max_iter, precond, host_check, is_delta, model, train, train_every, reuse_filters=False):
        P = int(num_probes)
        field = field.reshape(self.N, self.nz).contiguous()
        mode_i = _native.MODES[mode] if isinstance(mode, str) else int(mode)
        for name, t, shp in (("probes", probes, (P, self.N)), ("src_shared", src_shared, (self.L, self.N)),
                             ("src_exit", src_exit, (P, self.N)), ("u_store", u_store, (P, self.nz, self.N)),
                             ("exit_out", exit_out, (P, self.N)), ("grad_c", grad_c, (self.L, self.N))):
            if t is not None and (t.dtype != self.cdtype or not t.is_contiguous() or tuple(t.shape) != shp):
                raise ValueError(f"{name} must be a contiguous {self.cdtype} tensor of shape {shp}")
        a = _native.TpCn3dMarchArgs()
        a.num_probes, a.mode, a.max_iter, a.precond, a.host_check = P, mode_i, int(max_iter), int(precond), int(host_check)
        a.tol = float(tol)
        a.launch = int(self.launch)
        a.kernels = int(self.kernels)
        a.probes, a.src_shared, a.src_exit = _ptr(probes), _ptr(src_shared), _ptr(src_exit)
        a.u_store, a.exit_out, a.u_fwd, a.grad_c = _ptr(u_store), _ptr(exit_out), _ptr(u_fwd), _ptr(grad_c)
        a.stats = ctypes.c_void_p(self.stats.data_ptr())
        if precond == 2:
            reused = reuse_filters and self._lws is not None and self._lws_P == P
            lws = self.learned_workspace(P)
            a.learned_reuse = 1 if reused else 0
            mdl = model.model()
            a.model = ctypes.cast(ctypes.pointer(mdl), ctypes.c_void_p)
            a.learned_ws, a.learned_ws_bytes = _ptr(lws), lws.numel()
        if train is not None and train_every > 0:
            S = self.L // int(train_every)
            if tuple(train.z0.shape) != (S, P, self.N) or tuple(train.sol.shape) != (S, P, self.N) or \
                    tuple(train.diag.shape) != (S, self.N):
                raise ValueError(f"training buffers must be ({S}, {P}, {self.N}) and ({S}, {self.N})")
            a.train_z0, a.train_sol, a.train_diag = _ptr(train.z0), _ptr(train.sol), _ptr(train.diag)
            a.train_every = int(train_every)
            a.train_kind = 1 if train.kind == "noise" else 0
        ws = self.workspace(P)
        dt = _native.C128 if field.dtype == torch.complex128 else _native.C64
        o = self.op(is_delta)
        rc = self.lib.tp_cn3d_march(ctypes.byref(o), _ptr(field), dt, ctypes.byref(a), _ptr(ws), ws.numel(),
                                    ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))
        _native.check(rc, "tp_cn3d_march", self.lib)

    def device_status(self):
        """Raise if a bounded device-side wait of this library gave up (the
        tensor-memory stencil kernels' stage waits, the bulk-staged learned
        filter's row waits); synchronises the stream."""
        code = ctypes.c_int32()
        rc = self.lib.tp_device_status(ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream),
                                       ctypes.byref(code))
        _native.check(rc, "tp_device_status", self.lib)

    def read_stats(self, reset=True):
        """(total iterations, solves, failed solves, max iterations per solve,
        whether the last march ran as one CUDA graph)."""
        s = self.stats.cpu().tolist()
        if reset:
            self.stats.zero_()
        return {"iterations": s[0], "solves": s[1], "failed": s[2], "max_iterations": s[3], "graph": bool(s[4])}

    def grad_to_n(self, grad_c: torch.Tensor, field=None, is_delta=False) -> torch.Tensor:
        """Σ_p λ conj(u_s + u_{s−1}) (L, N) → torch-convention ∂/∂n (N, nz)."""
        acc = torch.zeros((self.N, self.nz), dtype=torch.complex128, device=self.device)
        g = grad_c.to(torch.complex128).T
        acc[:, :-1] += g
        acc[:, 1:] += g
        d = (self.dz / 4) * (self.k / 1j)
        if self.exact_ref_coeff:
            f = field.reshape(self.N, self.nz).to(torch.complex128)
            nn = f + 1 if is_delta else f
            return (np.conj(d) * torch.conj(nn) * acc).to(self.cdtype)
        return (np.conj(d) * acc).to(self.cdtype)


class PWEGradient3D:
    """Amplitude-loss gradient of a 3D geometry, all probes batched
    (far field ``|FFT2(exit)|`` of each probe's nx × ny exit wave; forward +
    exact adjoint by :class:`CN3D`; ``precond="learned"`` with a
    :class:`learned.LearnedPreconditioner` uses the learned correction in both)."""

    def __init__(self, geometry, bc_type="impedance", device=None, tol=1e-6, max_iter=20, precond=True, model=None):
        self.geometry = geometry
        self.engine = CN3D(geometry.effective_shape[0], geometry.effective_shape[1], geometry.nz, geometry.k,
                           geometry.dx, getattr(geometry, "dy", geometry.dx), geometry.dz, bc_type,
                           exact_ref_coeff=bool(getattr(geometry, "exact_ref_coeff", False)), device=device)
        self.device = self.engine.device
        self.kw = dict(tol=tol, max_iter=max_iter, precond=precond, model=model)
        self._store = None

    def forward(self, field, probes):
        e = self.engine
        P = probes.shape[0]
        if self._store is None or self._store.shape[0] != P:
            self._store = e.new_store(P)
        ex = torch.empty((P, e.N), dtype=torch.complex64, device=self.device)
        e.march(field, P, "forward", probes=probes.reshape(P, e.N).contiguous(), u_store=self._store, exit_out=ex,
                **self.kw)
        self._filters_of = field  # the learned filters now in the engine's workspace
        return ex

    def backward(self, field, exit_grad):
        e = self.engine
        P = exit_grad.shape[0]
        gc = torch.zeros((e.L, e.N), dtype=torch.complex64, device=self.device)
        e.march(field, P, "adjoint_exact", src_exit=exit_grad.reshape(P, e.N).contiguous(), u_fwd=self._store,
                grad_c=gc, reuse_filters=getattr(self, "_filters_of", None) is field, **self.kw)
        self.grad_c = gc
        return e.grad_to_n(gc, field)

    def loss_and_grad(self, n, probes, amplitude):
        e = self.engine
        field = torch.as_tensor(np.ascontiguousarray(n) if not isinstance(n, torch.Tensor) else n).to(
            self.device, torch.complex128)
        pr = torch.as_tensor(np.ascontiguousarray(probes) if not isinstance(probes, torch.Tensor) else probes).to(
            self.device, torch.complex64).reshape(-1, e.N)
        amp = torch.as_tensor(np.ascontiguousarray(amplitude) if not isinstance(amplitude, torch.Tensor) else amplitude).to(
            self.device, torch.float64).reshape(-1, e.nx, e.ny)
        from . import heads

        ex = self.forward(field, pr).reshape(-1, e.nx, e.ny).contiguous()
        if heads.fft_plannable(e.nx) and heads.fft_plannable(e.ny):
            U = heads.fft2_last(ex)
        else:
            U = torch.fft.fft2(ex)
        mag = U.abs().to(torch.float64)
        loss = torch.sum((mag - amp) ** 2)
        safe = torch.where(mag > 0, mag, torch.ones_like(mag))
        gU = (torch.where(mag > 0, 2 * (mag - amp) / safe, torch.zeros_like(mag)).to(torch.float32) * U).contiguous()
        if heads.fft_plannable(e.nx) and heads.fft_plannable(e.ny):
            ge = (e.N * heads.fft2_last(gU, inverse=True)).reshape(-1, e.N).contiguous()
        else:
            ge = (e.N * torch.fft.ifft2(gU)).reshape(-1, e.N).contiguous()
        g = self.backward(field, ge)
        return float(loss.item()), g.reshape(e.nx, e.ny, e.nz)


def generate_pairs(engine: CN3D, field, probes, every=1, tol=1e-6, max_iter=20, mode="forward", kind="rhs"):
    """Training pairs from a plain FFT-preconditioned march over `field`:
    every `every`-th step gives, per probe, z0 = M0⁻¹ v and x with
    (I − P_s) x = v, and the slice's object diagonal (see
    :class:`learned.TrainingPairs`).  kind "rhs": v is the step's right-hand
    side and x its converged update; kind "noise": x is white noise and
    v = (I − P_s) x, which exposes the correction to every spatial frequency
    (the Krylov search directions are rougher than the right-hand sides)."""
    from .learned import TrainingPairs

    if kind not in ("rhs", "noise"):
        raise ValueError(f"unknown pair kind {kind!r}")
    P = probes.shape[0]
    S = engine.L // int(every)
    N = engine.N
    dev = engine.device
    pairs = TrainingPairs(engine.nx, engine.ny, torch.empty((S, P, N), dtype=torch.complex64, device=dev),
                          torch.empty((S, P, N), dtype=torch.complex64, device=dev),
                          torch.empty((S, N), dtype=torch.complex64, device=dev), kind)
    engine.march(field, P, mode, probes=probes, tol=tol, max_iter=max_iter, precond=True, train=pairs,
                 train_every=every)
    return pairs
