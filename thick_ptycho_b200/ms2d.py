"""Angular-spectrum multislice on the GPU (2D), drop-in for the reference's
``MSForwardModelSolver`` (``forward_model/multislice/ms_solver.py:8-159``).

The index field enters through a transmission table (``T_z − 1`` with
``T_z = exp(ik(n_z − n_med)dz)``) built once per ``n`` in fp64; every probe is then marched through
all slices inside one CTA (field in shared memory, FFTs by libtpcuda's
mixed-radix shared-memory FFT).  :class:`MSFunction` gives the exit waves
with the hand-written adjoint march as its backward.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _native, heads


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class MS2D:
    """Multislice engine for one geometry (n transverse points, nz nodes)."""

    def __init__(self, n, nz, k, dx, dz, n_medium=1.0, device=None):
        if not torch.cuda.is_available():
            raise _native.NativeLibraryError("MS2D needs a CUDA device (there is no CPU fallback)")
        self.lib = _native.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.n, self.nz, self.L = int(n), int(nz), int(nz) - 1
        o = _native.TpMs2dOp()
        o.n, o.nz, o.k, o.dx, o.dz = self.n, self.nz, float(k), float(dx), float(dz)
        nm = complex(n_medium)
        o.n_medium = (ctypes.c_double * 2)(nm.real, nm.imag)
        self._op = o
        self.k, self.dz = float(k), float(dz)

    def transmission(self, field: torch.Tensor) -> torch.Tensor:
        if tuple(field.shape) != (self.n, self.nz):
            raise ValueError(f"index field has shape {tuple(field.shape)}, expected {(self.n, self.nz)}")
        field = field.contiguous()
        dt = _native.C128 if field.dtype == torch.complex128 else _native.C64
        T = torch.empty((self.L, self.n), dtype=torch.complex64, device=self.device)
        _native.check(self.lib.tp_ms2d_transmission(ctypes.byref(self._op), _ptr(field), dt, _ptr(T), _stream(self.device)),
                      "tp_ms2d_transmission")
        return T

    def march(self, T, probes, u_store=None, exit_out=None):
        P = probes.shape[0]
        _native.check(self.lib.tp_ms2d_march(ctypes.byref(self._op), _ptr(T), _ptr(probes.contiguous()), P, _ptr(u_store),
                                             _ptr(exit_out), _stream(self.device)), "tp_ms2d_march")

    def backward(self, T, u_fwd, src_exit, grad_t):
        P = src_exit.shape[0]
        _native.check(self.lib.tp_ms2d_backward(ctypes.byref(self._op), _ptr(T), _ptr(u_fwd), _ptr(src_exit.contiguous()),
                                                P, _ptr(grad_t), _stream(self.device)), "tp_ms2d_backward")

    def grad_to_n(self, grad_t: torch.Tensor) -> torch.Tensor:
        """(L, n) accumulator → torch-convention ∂loss/∂n of shape (n, nz)."""
        g = torch.zeros((self.n, self.nz), dtype=torch.complex64, device=self.device)
        g[:, :-1] = (np.conj(1j * self.k * self.dz) * grad_t).T
        return g


class MSFunction(torch.autograd.Function):
    """``exit = MS(n)`` with the adjoint multislice march as backward."""

    @staticmethod
    def forward(ctx, field, probes, engine: MS2D):
        P = probes.shape[0]
        T = engine.transmission(field.detach())
        st = torch.empty((P, engine.nz, engine.n), dtype=torch.complex64, device=engine.device)
        ex = torch.empty((P, engine.n), dtype=torch.complex64, device=engine.device)
        engine.march(T, probes.detach().to(torch.complex64), u_store=st, exit_out=ex)
        ctx.save_for_backward(field)
        ctx.engine, ctx.T, ctx.st = engine, T, st
        return ex

    @staticmethod
    def backward(ctx, grad_exit):
        (field,) = ctx.saved_tensors
        e = ctx.engine
        gt = torch.zeros((e.L, e.n), dtype=torch.complex64, device=e.device)
        e.backward(ctx.T, ctx.st, grad_exit.to(torch.complex64).contiguous(), gt)
        return e.grad_to_n(gt).to(field.dtype), None, None


class MSGpuSolver:
    """Drop-in for ``MSForwardModelSolver`` running on one B200.

    2D as the reference; a 3D simulation space (which the reference rejects,
    ``ms_solver.py:28-31``) runs the 3D propagator of :mod:`.ms3d`, with
    fields of shape (proj, angle, probes, nx, ny, nz).
    """

    def __init__(self, simulation_space, ptycho_probes, results_dir="", use_logging=False, verbose=False, log=None,
                 device=None):
        ss = simulation_space
        self.dimension = int(getattr(ss, "dimension", 2))
        self.simulation_space = ss
        self.probes = ptycho_probes
        self.verbose = verbose
        self.effective_shape = tuple(ss.effective_shape)
        self.block_size = ss.block_size
        self.nz = ss.nz
        self.nx_eff = getattr(ss, "effective_nx", ss.nx)
        self.num_probes = ss.num_probes
        self.num_projections = ss.num_projections
        self.probe_angles = ss.probe_angles
        self.num_angles = len(self.probe_angles)
        self.n_medium = complex(getattr(ss, "n_medium", 1.0))
        self.solver_type = self.__class__.__name__
        if self.dimension == 3:
            from .ms3d import MS3D

            ny_eff = getattr(ss, "effective_ny", self.nx_eff)
            self.engine = MS3D(self.nx_eff, ny_eff, self.nz, ss.k, ss.dx, getattr(ss, "dy", ss.dx), ss.dz,
                               self.n_medium, device=device)
            self.block = self.nx_eff * ny_eff
        else:
            self.engine = MS2D(self.nx_eff, self.nz, ss.k, ss.dx, ss.dz, self.n_medium, device=device)
            self.block = self.nx_eff
        self.device = self.engine.device

    def reset_cache(self):
        """Nothing is cached across calls (the transmission is rebuilt per ``n``)."""

    def _field(self, n):
        if n is None:
            n = self.simulation_space.refractive_index_empty
        if isinstance(n, torch.Tensor):
            f = n.to(self.device)
        else:
            f = torch.from_numpy(np.ascontiguousarray(n, dtype=np.complex128)).to(self.device)
        return f.reshape(self.block, self.nz)

    def solve(self, n=None, mode="forward", rhs_block=None, probes=None, **kwargs) -> np.ndarray:
        """All probes, shape (proj, angle, probes, nx, nz) complex128 (``base/base_solver.py:84-154``)."""
        assert mode in {"forward", "adjoint", "reverse"}, f"Invalid mode: {mode!r}"
        if mode != "forward":
            raise AssertionError(f"Invalid mode: {mode}")  # the reference's MS accepts forward only here
        probes = self.probes if probes is None else probes
        count = self.num_angles * self.num_probes
        T = self.engine.transmission(self._field(n))
        pr = torch.from_numpy(np.ascontiguousarray(probes).reshape(count, self.block).astype(np.complex64)).to(self.device)
        st = torch.empty((count, self.nz, self.block), dtype=torch.complex64, device=self.device)
        self.engine.march(T, pr, u_store=st)
        u = st.permute(0, 2, 1).cpu().numpy().astype(np.complex128)
        out = np.zeros((self.num_projections, self.num_angles, self.num_probes, *self.effective_shape), dtype=complex)
        out[0] = u.reshape(self.num_angles, self.num_probes, *self.effective_shape)
        return out

    def _solve_single_probe(self, scan_idx=0, proj_idx=0, n=None, mode="forward", probe=None, **kwargs):
        assert mode in {"forward", "backward"}, f"Invalid mode: {mode}"
        if probe is None:
            probe = np.zeros(self.block, dtype=complex)
        T = self.engine.transmission(self._field(n))
        pr = torch.from_numpy(np.asarray(probe, dtype=np.complex64).reshape(1, -1)).to(self.device)
        st = torch.empty((1, self.nz, self.block), dtype=torch.complex64, device=self.device)
        self.engine.march(T, pr, u_store=st)
        return st[0].T.cpu().numpy().astype(np.complex128).reshape(*self.effective_shape)

    def get_exit_waves(self, u=None) -> np.ndarray:
        return u[..., -1].reshape((self.simulation_space.total_scans, self.simulation_space.block_size))

    def get_farfield_intensities(self, u=None, exit_waves=None, poisson_noise=True) -> np.ndarray:
        """``|FFT(exit)|²`` computed on the GPU (``base/base_solver.py:213-249``); in 3D,
        as the reference's base solver, ``fft2`` over the last two axes of the
        (total_scans, block_size) exit-wave array."""
        exit_waves = self.get_exit_waves(u=u) if exit_waves is None else exit_waves
        ex = torch.from_numpy(np.ascontiguousarray(exit_waves).astype(np.complex64)).to(self.device)
        if self.dimension == 3:
            ex = ex.reshape(self.simulation_space.total_scans, self.simulation_space.block_size)
            if heads.fft_plannable(ex.shape[0]) and heads.fft_plannable(ex.shape[1]):
                inten = (heads.fft2_last(ex).abs() ** 2).cpu().numpy().astype(np.float64)
            else:
                inten = (torch.fft.fft2(ex.to(torch.complex128), dim=(-2, -1)).abs() ** 2).cpu().numpy()
        else:
            inten = heads.farfield_intensity(ex).cpu().numpy().astype(np.float64)
        if poisson_noise:
            inten = np.random.poisson(inten)
        return inten.reshape((self.simulation_space.total_scans, self.simulation_space.block_size))


class ReconstructorMSGpu:
    """Multislice 3PIE reconstruction (``reconstruction/ms_reconstructor.py:40-190``) on the GPU.

    Same arguments and results as the reference's ``ReconstructorMS``:
    ``reconstruct(max_iters, alpha_obj)`` returns the estimate (nx, nz)
    complex128 and the per-epoch rms exit-wave error.  The update is
    sequential over probes, as the reference's, and runs in one kernel
    (``tp_ms2d_3pie``).  ``data``: (P, N) far-field intensities with
    ``phase_retrieval`` (else known exit waves); ``probes``: (P, N).
    """

    def __init__(self, n, nz, k, dx, dz, data, probes, phase_retrieval=True, n_medium=1.0, device=None):
        self.engine = MS2D(n, nz, k, dx, dz, n_medium=n_medium, device=device)
        e = self.engine
        self.n_medium = complex(n_medium)
        self.phase_retrieval = bool(phase_retrieval)
        dt = torch.float32 if phase_retrieval else torch.complex64
        self.data = torch.as_tensor(np.ascontiguousarray(data)).to(e.device, dt).reshape(-1, e.n).contiguous()
        self.probes = torch.as_tensor(np.ascontiguousarray(probes)).to(e.device, torch.complex64).reshape(-1, e.n)
        self.probes = self.probes.contiguous()
        self.ws = torch.empty(int(e.lib.tp_ms2d_3pie_workspace_bytes(e.n, e.nz)), dtype=torch.uint8, device=e.device)

    def reconstruct(self, max_iters=10, alpha_obj=1.0, refractive_index=None):
        e = self.engine
        if refractive_index is None:
            n0 = self.n_medium * np.ones((e.n, e.nz), dtype=complex)
        else:
            n0 = np.array(refractive_index, dtype=complex)
        n_est = torch.from_numpy(n0).to(e.device).contiguous()
        loss = torch.zeros(max(int(max_iters), 1), dtype=torch.float64, device=e.device)
        rc = e.lib.tp_ms2d_3pie(ctypes.byref(e._op), _ptr(self.probes), self.probes.shape[0], _ptr(self.data),
                                int(self.phase_retrieval), int(max_iters), float(alpha_obj), _ptr(n_est), _ptr(loss),
                                _ptr(self.ws), self.ws.numel(), _stream(e.device))
        _native.check(rc, "tp_ms2d_3pie")
        return n_est.cpu().numpy(), loss[: int(max_iters)].cpu().numpy().tolist()
