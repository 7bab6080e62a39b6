"""Drop-in GPU replacement for the reference ``PWEIterativeLUSolver``.

:class:`PWEGpuSolver` keeps the reference solver's constructor, methods,
array shapes and error behaviour (``forward_model/pwe/solvers/
iterative_lu.py:36-197``, ``pwe/solvers/base_solver.py:29-209``,
``base/base_solver.py:14-249``) and runs the arithmetic in libtpcuda:

* ``_construct_solve_cache`` → one ``tp_cn2d_factor`` call (all slices) in
  place of ``nz − 1`` SuperLU factorisations (``iterative_lu.py:103-133``);
* ``solve`` → one batched ``tp_cn2d_march`` over every (angle, probe) in place
  of the serial probe loop (``base/base_solver.py:124-143``);
* ``_solve_single_probe`` → the same march for one probe with an optional
  ``rhs_block`` (the reconstructor's adjoint and step-size solves).

3D simulation spaces (2D transverse, ``iterative_lu.py`` on the 5-point
operators of ``operator_matrices.py:75-126``) run through ``tp_cn3d_march``:
no factorisation is cached (each slice is an FFT-preconditioned BiCGStab
solve to ``tol``), so the mode cache holds only the device copy of n.

Inputs and outputs are NumPy arrays as in the reference (complex128 out); the
arithmetic is complex64 with fp64 factorisation.  The ``*_device`` methods
take and return torch CUDA tensors for callers that keep data on the GPU.
"""

from __future__ import annotations

import time
from typing import Optional, Tuple

import numpy as np
import scipy.sparse as sp
import torch

from . import _native
from .cn2d import CN2D
from .cn3d import CN3D
from .operators import normalize_bc

_MODES = ("forward", "adjoint", "reverse", "adjoint_exact")


class _ModeCache:
    __slots__ = ("n_ref", "factors")

    def __init__(self):
        self.n_ref = None
        self.factors = None


class PWEGpuSolver:
    """Slice-by-slice Crank–Nicolson PWE solver on one B200 (2D and 3D problems)."""

    def __init__(
        self,
        simulation_space,
        ptycho_probes,
        bc_type="impedance",
        results_dir="",
        use_logging=False,
        verbose=False,
        log=None,
        test_bcs=None,
        device=None,
        tol=1e-6,
        max_iter=20,
    ):
        ss = simulation_space
        self.simulation_space = ss
        self.verbose = verbose
        self.results_dir = results_dir
        self._log = log or (print if verbose else (lambda *a, **k: None))
        self.solve_reduced_domain = bool(getattr(ss, "solve_reduced_domain", False))
        if self.solve_reduced_domain:
            raise NotImplementedError("PWEGpuSolver solves the full domain (solve_reduced_domain=False)")
        self.effective_shape = tuple(ss.effective_shape)
        self.block_size = int(ss.block_size)
        self.nz = int(ss.nz)
        self.probes = ptycho_probes
        self.num_probes = int(ss.num_probes)
        self.num_projections = int(ss.num_projections)
        assert self.num_projections <= 2, "Only supports up to 2 projections."
        self.probe_angles = ss.probe_angles
        self.num_angles = len(self.probe_angles)
        self.solver_type = self.__class__.__name__
        self.test_bcs = test_bcs
        self.bc_type = normalize_bc(bc_type)
        self.dimension = int(ss.dimension)
        empty_px = int(getattr(ss, "empty_space_px", 0) or 0)
        if self.dimension == 2:
            self.engine = CN2D(
                self.block_size,
                self.nz,
                ss.k,
                ss.dx,
                ss.dz,
                bc_type=self.bc_type,
                empty_px=empty_px,
                exact_ref_coeff=bool(getattr(ss, "exact_ref_coeff", False)),
                device=device,
            )
        elif self.dimension == 3:
            if empty_px > 0:
                # the reference pads only axis 0 of a 3D coefficient array (base_simulation_space.py:363-376)
                raise NotImplementedError("3D simulation spaces with empty_space_px > 0 are not supported")
            self.engine = CN3D(self.effective_shape[0], self.effective_shape[1], self.nz, ss.k, ss.dx,
                               getattr(ss, "dy", ss.dx), ss.dz, bc_type=self.bc_type,
                               exact_ref_coeff=bool(getattr(ss, "exact_ref_coeff", False)), device=device)
            self.krylov = dict(tol=tol, max_iter=max_iter)
        else:
            raise ValueError(f"dimension must be 2 or 3, not {ss.dimension}")
        self.device = self.engine.device
        self.create_projection_cache()

    # ------------------------------------------------------------------ cache
    def create_projection_cache(self):
        self.projection_cache = [{m: _ModeCache() for m in _MODES} for _ in range(self.num_projections)]

    def reset_cache(self):
        """Drop every factor set (``base_solver.py:326-329``)."""
        self.create_projection_cache()

    def get_projected_obj(self, n, mode="forward", proj_idx=0):
        """Rotate n for the second projection (``base/base_solver.py:67-78``)."""
        if self.simulation_space.num_projections == 1 or proj_idx == 0:
            return n
        if proj_idx == 1:
            return np.rot90(n, k=1)
        raise ValueError(f"Invalid projection index: {proj_idx}")

    def _field_device(self, n) -> torch.Tensor:
        if isinstance(n, torch.Tensor):
            t = n.to(self.device)
            return t if t.dtype in (torch.complex128, torch.complex64) else t.to(torch.complex128)
        return torch.from_numpy(np.ascontiguousarray(n, dtype=np.complex128)).to(self.device)

    def _construct_solve_cache(self, n=None, mode="forward", scan_idx=0, proj_idx=0):
        """Factorise all slices for ``mode`` (``iterative_lu.py:66-101``)."""
        if n is None:
            n = self.simulation_space.refractive_index_empty
        field = self._field_device(self.get_projected_obj(n, proj_idx=proj_idx))
        cache = self.projection_cache[proj_idx][mode]
        cache.factors = self.engine.factor(field, mode) if self.dimension == 2 else field
        cache.n_ref = n

    def _get_or_construct_cache(self, n, mode, proj_idx=0, scan_idx=0):
        """Factorise if missing or if a different ``n`` object is passed.

        Like the reference (``base_solver.py:89-119``) an ``n`` mutated in
        place is not detected: call ``prepare_solver_caches`` or
        ``reset_cache`` after changing it.
        """
        assert mode in self.projection_cache[proj_idx], f"Invalid mode: {mode!r}"
        cache = self.projection_cache[proj_idx][mode]
        if cache.factors is None or cache.n_ref is not n:
            self._construct_solve_cache(n=n, mode=mode, proj_idx=proj_idx, scan_idx=scan_idx)

    def prepare_solver_caches(self, n, modes: Tuple[str, ...] = ("forward", "adjoint")):
        """(Re)build the factor sets of every projection and mode (``base_solver.py:318-324``)."""
        for proj_idx in range(self.num_projections):
            for mode in modes:
                self._construct_solve_cache(n=n, proj_idx=proj_idx, mode=mode)

    # ---------------------------------------------------------------- sources
    def _test_bc_source(self) -> Optional[torch.Tensor]:
        if self.test_bcs is None:
            return None
        rows = [np.asarray(self.test_bcs.test_exact_impedance_rhs_step(j)).ravel() for j in range(1, self.nz)]
        return torch.from_numpy(np.stack(rows).astype(np.complex64)).to(self.device)

    def _step_source(self, rhs_block, mode) -> torch.Tensor:
        """``rhs_block`` (block_size·(nz−1)) as the (L, N) source of each march step
        (the adjoint reads column −j at step j, ``iterative_lu.py:172-176``)."""
        rb = np.asarray(rhs_block).reshape(self.block_size, self.nz - 1)
        if mode in ("adjoint", "adjoint_exact"):
            rb = rb[:, ::-1]
        return torch.from_numpy(np.ascontiguousarray(rb.T).astype(np.complex64)).to(self.device)

    def _march3d(self, field, count, mode, probes, src_shared, store, exit_w):
        self.engine.march(field, count, mode, probes=probes, src_shared=src_shared, u_store=store, exit_out=exit_w,
                          **self.krylov)

    def _unstore(self, store) -> torch.Tensor:
        """Device store → (P, *effective_shape) complex64."""
        if self.dimension == 2:
            return self.engine.unchunk(store)
        P = store.shape[0]
        return store.permute(0, 2, 1).reshape(P, *self.effective_shape)

    def _probes_device(self, probes, count) -> torch.Tensor:
        if isinstance(probes, torch.Tensor):
            t = probes.to(self.device, torch.complex64)
        else:
            t = torch.from_numpy(np.ascontiguousarray(probes).astype(np.complex64)).to(self.device)
        return t.reshape(count, self.block_size).contiguous()

    # ------------------------------------------------------------------ solve
    def solve_device(self, n=None, mode="forward", rhs_block=None, probes=None, proj_idx=0, full_field=True):
        """Batched march of every (angle, probe) for one projection.

        Returns ``(u_store, exit)``: the full field (2D: chunked (A·P, nz,
        Npad); 3D: (A·P, nz, N)) or None, and the last-step field (A·P, N),
        complex64 on the device.
        """
        if mode not in _MODES:
            raise AssertionError(f"Invalid mode: {mode!r}")
        if n is None:
            n = self.simulation_space.refractive_index_empty
        if probes is None:
            probes = self.probes
        count = self.num_angles * self.num_probes
        self._get_or_construct_cache(n, mode, proj_idx=proj_idx)
        fs = self.projection_cache[proj_idx][mode].factors
        src_shared = self._test_bc_source()
        if src_shared is None and rhs_block is not None:
            src_shared = self._step_source(rhs_block, mode)
        pr = self._probes_device(probes, count)
        store = self.engine.new_store(count) if full_field else None
        exit_w = torch.empty((count, self.block_size), dtype=torch.complex64, device=self.device)
        if self.dimension == 3:
            self._march3d(fs, count, mode, pr, src_shared, store, exit_w)
        else:
            self.engine.march(fs, count, probes=pr, src_shared=src_shared, u_store=store, exit_out=exit_w)
        return store, exit_w

    def solve(self, n=None, mode="forward", rhs_block=None, probes=None, **kwargs) -> np.ndarray:
        """Every projection, angle and probe (``base/base_solver.py:84-154``).

        Returns complex128 of shape (num_projections, num_angles, num_probes,
        *effective_shape).
        """
        assert mode in {"forward", "adjoint", "reverse", "adjoint_exact"}, f"Invalid mode: {mode!r}"
        t0 = time.time()
        out = np.zeros((self.num_projections, self.num_angles, self.num_probes, *self.effective_shape), dtype=complex)
        for proj_idx in range(self.num_projections):
            store, _ = self.solve_device(n=n, mode=mode, rhs_block=rhs_block, probes=probes, proj_idx=proj_idx)
            u = self._unstore(store).cpu().numpy().astype(np.complex128)
            out[proj_idx] = u.reshape(self.num_angles, self.num_probes, *self.effective_shape)
        if self.verbose:
            self._log(f"[{self.solver_type}] solved {self.num_projections * self.num_angles * self.num_probes} "
                      f"probes in {time.time() - t0:.3f}s")
        return out

    def _solve_single_probe(self, scan_idx=0, proj_idx=0, probe=None, n=None, mode="forward", rhs_block=None):
        """One probe's field, shape (block_size, nz) (``pwe/solvers/base_solver.py:134-179``)."""
        self._get_or_construct_cache(n=n, mode=mode, proj_idx=proj_idx, scan_idx=scan_idx)
        return self._solve_single_probe_impl(scan_idx, proj_idx, probe, mode, rhs_block)

    def _solve_single_probe_impl(self, scan_idx=0, proj_idx=0, probe=None, mode="forward", rhs_block=None):
        """March one probe (``iterative_lu.py:138-197``)."""
        fs = self.projection_cache[proj_idx][mode].factors
        pr = None if probe is None else self._probes_device(probe, 1)
        src_shared = self._test_bc_source()
        src_probe = None
        store = self.engine.new_store(1)
        if self.dimension == 3:
            if src_shared is None and rhs_block is not None:
                src_shared = self._step_source(rhs_block, mode)
            self._march3d(fs, 1, mode, pr, src_shared, store, None)
        else:
            if src_shared is None and rhs_block is not None:
                rb = np.asarray(rhs_block).reshape(self.block_size, self.nz - 1)
                src_probe = torch.from_numpy(np.ascontiguousarray(rb.T).astype(np.complex64)).to(self.device)[None]
            self.engine.march(fs, 1, probes=pr, src_shared=src_shared, src_probe=src_probe, u_store=store)
        return self._unstore(store)[0].reshape(self.block_size, self.nz).cpu().numpy().astype(np.complex128)

    # --------------------------------------------------------------- outputs
    def get_gradient(self, n):
        """``diag(G) + subdiag(G)`` with G the grad-form object contribution
        (``pwe/solvers/base_solver.py:193-209``, ``forward_model.py:128-153``)."""
        ss = self.simulation_space
        k, dz = ss.k, ss.dz
        n = np.asarray(n)
        coef = (k / 1j) * (n if getattr(ss, "exact_ref_coeff", False) else np.ones_like(n))
        e = int(getattr(ss, "empty_space_px", 0) or 0)
        if e > 0:
            coef = np.pad(coef, ((e, e), (0, 0)))
        G = (dz / 2) * (coef[..., :-1] + coef[..., 1:]) / 2
        return sp.diags(G.T.flatten()) + sp.diags([G[..., 1:].T.flatten()], offsets=[-self.block_size])

    def get_exit_waves(self, u=None) -> np.ndarray:
        """``u[..., −1]`` as (total_scans, block_size) (``base/base_solver.py:194-211``)."""
        return u[..., -1].reshape((self.simulation_space.total_scans, self.block_size))

    def get_farfield_intensities(self, u=None, exit_waves=None, poisson_noise=True,
                                 generator: Optional[torch.Generator] = None) -> np.ndarray:
        """``|FFT(exit)|²`` with optional Poisson noise (``base/base_solver.py:213-249``), on the GPU.

        2D: FFT of each exit wave (libtpcuda's FFT head when the length is
        2^a 3^b 5^c ≤ 4096, else cuFFT through torch).  3D: as the reference,
        ``fft2`` over the last two axes of the (total_scans, block_size)
        exit-wave array.  Poisson noise is drawn on the device from
        `generator` (the reference draws from numpy's unseeded global RNG);
        noisy intensities are returned as int64 like ``numpy.random.poisson``.
        """
        from . import heads

        exit_waves = self.get_exit_waves(u=u) if exit_waves is None else exit_waves
        ex = torch.as_tensor(np.ascontiguousarray(exit_waves)).to(self.device, torch.complex64)
        ex = ex.reshape(self.simulation_space.total_scans, self.block_size).contiguous()
        if self.dimension == 2 and heads.fft_plannable(self.block_size):
            inten = heads.farfield_intensity(ex).to(torch.float64)
        elif self.dimension == 2:
            inten = torch.fft.fft(ex.to(torch.complex128), dim=-1).abs() ** 2
        else:
            inten = torch.fft.fft2(ex.to(torch.complex128), dim=(-2, -1)).abs() ** 2
        if poisson_noise:
            inten = torch.poisson(inten, generator=generator).to(torch.int64)
        return inten.cpu().numpy().reshape((self.simulation_space.total_scans, self.block_size))

    def save_simulated_data(self, path, n=None, poisson_noise=True, generator: Optional[torch.Generator] = None):
        """Forward-simulate and write ``{intensity, exit_waves}`` in the
        reference's ``simulated_data.npz`` format (``generate_data.py:185-197``,
        read back by ``reconstruct_sample.py:62-67``)."""
        u = self.solve(n=n)
        exit_waves = self.get_exit_waves(u)
        data = self.get_farfield_intensities(exit_waves=exit_waves, poisson_noise=poisson_noise, generator=generator)
        np.savez_compressed(path, intensity=data, exit_waves=exit_waves)
        return data, exit_waves

    def device_status(self):
        """Raise if a device-side bounded wait of an earlier launch timed out."""
        self.engine.device_status()
