"""Batched 2D Crank–Nicolson propagation on the GPU (host side).

:class:`CN2D` owns the device workspaces of one geometry and calls the C ABI
of libtpcuda.so (``include/tpcuda.h``) on the current torch CUDA stream.
Tensors are complex64 on the device except the refractive index, which may
be complex128 (``n``) or complex64 holding ``n − 1`` (``is_delta=True``).
With ``check=True`` the geometry runs on the complex128 check build
(``libtpcuda_c128.so``): the same algorithms with complex128 state, factor
sets and fields, and every complex tensor complex128.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _native
from .operators import BCCoefficients, normalize_bc, operator_1d


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _c2(z: complex):
    return (ctypes.c_double * 2)(z.real, z.imag)


@dataclass
class FactorSet:
    mode: int
    buf: torch.Tensor  # uint8 workspace


class CN2D:
    """One 2D geometry: N transverse rows, nz nodes (L = nz − 1 steps)."""

    def __init__(self, n, nz, k, dx, dz, bc_type="impedance", empty_px=0, exact_ref_coeff=False, device=None,
                 check=False):
        if not torch.cuda.is_available():
            raise _native.NativeLibraryError("CN2D needs a CUDA device (there is no CPU fallback)")
        self.check = bool(check)
        self.lib = _native.load_check() if self.check else _native.load()
        # complex type of fields, sources, exit waves and gradients
        self.cdtype = torch.complex128 if self.check else torch.complex64
        self.device = torch.device(device if device is not None else "cuda")
        self.n, self.nz, self.L = int(n), int(nz), int(nz) - 1
        self.k, self.dx, self.dz = float(k), float(dx), float(dz)
        self.bc_type = normalize_bc(bc_type)
        self.empty_px = int(empty_px)
        self.n_obj = self.n - 2 * self.empty_px
        self.exact_ref_coeff = bool(exact_ref_coeff)
        co = BCCoefficients.make(self.k, self.dx, self.dz, self.bc_type)
        self.kop = operator_1d(self.n, co, self.bc_type, self.dz)
        c, m, npad = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        rc = self.lib.tp_cn2d_layout(self.n, ctypes.byref(c), ctypes.byref(m), ctypes.byref(npad))
        _native.check(rc, "tp_cn2d_layout", self.lib)
        self.chunks, self.rows_per_chunk, self.npad = c.value, m.value, npad.value
        self.factor_bytes = int(self.lib.tp_cn2d_factor_bytes(self.n, self.nz))

    # ------------------------------------------------------------------ op
    def op(self, is_delta=False) -> _native.TpCn2dOp:
        o = _native.TpCn2dOp()
        o.n, o.nz, o.n_obj, o.empty_px = self.n, self.nz, self.n_obj, self.empty_px
        o.exact_ref_coeff = int(self.exact_ref_coeff)
        o.field_is_delta = int(is_delta)
        o.k, o.dz = self.k, self.dz
        o.k_off, o.k_diag = _c2(self.kop.k_off), _c2(self.kop.k_diag)
        o.k_d0, o.k_dn = _c2(self.kop.k_d0), _c2(self.kop.k_dn)
        o.k_01, o.k_nm = _c2(self.kop.k_01), _c2(self.kop.k_nm)
        return o

    def _check_field(self, field: torch.Tensor):
        if field.device != self.device and not (field.is_cuda and self.device.type == "cuda"):
            raise ValueError("refractive index must be on the solver's device")
        if tuple(field.shape) != (self.n_obj, self.nz):
            raise ValueError(f"refractive index has shape {tuple(field.shape)}, expected {(self.n_obj, self.nz)}")
        if field.dtype not in (torch.complex128, torch.complex64):
            raise TypeError("refractive index must be complex128 or complex64")
        return field.contiguous()

    # ------------------------------------------------------------- factor
    def new_factor_buffer(self) -> torch.Tensor:
        return torch.empty(self.factor_bytes, dtype=torch.uint8, device=self.device)

    def factor(self, field: torch.Tensor, mode="forward", is_delta=False, out: Optional[torch.Tensor] = None) -> FactorSet:
        """Per-slice factor set of ``mode`` for the index field ``field``."""
        field = self._check_field(field)
        mode_i = _native.MODES[mode] if isinstance(mode, str) else int(mode)
        buf = out if out is not None else self.new_factor_buffer()
        dtype = _native.C128 if field.dtype == torch.complex128 else _native.C64
        o = self.op(is_delta)
        rc = self.lib.tp_cn2d_factor(ctypes.byref(o), _ptr(field), dtype, mode_i, _ptr(buf), buf.numel(),
                                     _stream(self.device))
        _native.check(rc, "tp_cn2d_factor", self.lib)
        return FactorSet(mode_i, buf)

    def factor_range(self, field: torch.Tensor, mode, slice_begin: int, slice_end: int, out: torch.Tensor,
                     is_delta=False) -> FactorSet:
        """Factorise slices ``slice_begin..slice_end`` (1-based, inclusive) of ``mode``
        into ``out``; slice s reads index columns s−1 and s.  The range that
        starts at slice 1 resets the PCR coupling bound the later ranges raise."""
        field = self._check_field(field)
        mode_i = _native.MODES[mode] if isinstance(mode, str) else int(mode)
        dtype = _native.C128 if field.dtype == torch.complex128 else _native.C64
        o = self.op(is_delta)
        rc = self.lib.tp_cn2d_factor_range(ctypes.byref(o), _ptr(field), dtype, mode_i, _ptr(out), out.numel(),
                                           int(slice_begin), int(slice_end), _stream(self.device))
        _native.check(rc, "tp_cn2d_factor_range", self.lib)
        return FactorSet(mode_i, out)

    # -------------------------------------------------------------- march
    def march(
        self,
        fs: FactorSet,
        num_probes: int,
        probes: Optional[torch.Tensor] = None,
        src_shared: Optional[torch.Tensor] = None,
        src_probe: Optional[torch.Tensor] = None,
        src_exit: Optional[torch.Tensor] = None,
        u_store: Optional[torch.Tensor] = None,
        exit_out: Optional[torch.Tensor] = None,
        u_fwd: Optional[torch.Tensor] = None,
        grad_c: Optional[torch.Tensor] = None,
        t_begin: int = 0,
        t_end: int = 0,
        state_in: Optional[torch.Tensor] = None,
        state_out: Optional[torch.Tensor] = None,
        store_every: int = 0,
        store_base: int = 0,
        ufwd_base: int = 0,
        store_sums: bool = False,
    ):
        """One batched march; every tensor is complex64 (complex128 in the
        check build), contiguous, on device.

        ``u_store`` is (P, S, Npad) with S slices per probe: the state after
        step t goes to index ``t − store_base`` (or ``t / store_every`` when
        ``store_every > 1``, only for multiples).  ``u_fwd`` is (≥P, S', Npad)
        with forward slice s at index ``s − ufwd_base``.  ``t_begin..t_end``
        restricts the steps; ``state_in``/``state_out`` (P, Npad) carry the
        state across partial marches.  ``store_sums`` (team path, N in
        {512, 1024, 2048}): a forward march stores ``(u_t + u_{t−1})/2`` (the
        exact-adjoint gradient contracts with the pair sum; the half sum is
        the Cayley step's solve result, stored at no extra cost) instead of
        ``u_t``, and an exact-adjoint march reads ``u_fwd`` as those.
        """
        P = int(num_probes)
        shapes = {
            "probes": (probes, (P, self.n)),
            "src_shared": (src_shared, (self.L, self.n)),
            "src_probe": (src_probe, (P, self.L, self.n)),
            "src_exit": (src_exit, (P, self.n)),
            "u_store": (u_store, None),
            "exit_out": (exit_out, (P, self.n)),
            "u_fwd": (u_fwd, None),
            "grad_c": (grad_c, (self.L, self.npad)),
            "state_in": (state_in, (P, self.npad)),
            "state_out": (state_out, (P, self.npad)),
        }
        for name, (t, shp) in shapes.items():
            if t is None:
                continue
            if t.dtype != self.cdtype or not t.is_contiguous() or not t.is_cuda:
                raise TypeError(f"{name} must be a contiguous {self.cdtype} CUDA tensor")
            if shp is not None and tuple(t.shape) != shp:
                raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {shp}")
        if u_fwd is not None and (u_fwd.dim() != 3 or u_fwd.shape[2] != self.npad or u_fwd.shape[0] < P):
            raise ValueError("u_fwd must be a chunked forward field (P, slices, Npad)")
        if u_store is not None and (u_store.dim() != 3 or u_store.shape[0] != P or u_store.shape[2] != self.npad):
            raise ValueError("u_store must be a chunked field (P, slices, Npad)")
        a = _native.TpCn2dMarchArgs()
        a.num_probes, a.mode = P, fs.mode
        a.probes, a.src_shared, a.src_probe, a.src_exit = _ptr(probes), _ptr(src_shared), _ptr(src_probe), _ptr(src_exit)
        a.u_store, a.exit_out, a.u_fwd, a.grad_c = _ptr(u_store), _ptr(exit_out), _ptr(u_fwd), _ptr(grad_c)
        a.t_begin, a.t_end = int(t_begin), int(t_end)
        a.state_in, a.state_out = _ptr(state_in), _ptr(state_out)
        a.store_slices = 0 if u_store is None else int(u_store.shape[1])
        a.store_every, a.store_base = int(store_every), int(store_base)
        a.ufwd_slices = 0 if u_fwd is None else int(u_fwd.shape[1])
        a.ufwd_base = int(ufwd_base)
        a.store_sums = 1 if store_sums else 0
        o = self.op()
        rc = self.lib.tp_cn2d_march(ctypes.byref(o), _ptr(fs.buf), ctypes.byref(a), _stream(self.device))
        _native.check(rc, "tp_cn2d_march", self.lib)

    # ------------------------------------------------------------ helpers
    def new_store(self, num_probes: int, slices: Optional[int] = None) -> torch.Tensor:
        s = self.nz if slices is None else int(slices)
        return torch.empty((num_probes, s, self.npad), dtype=self.cdtype, device=self.device)

    def unchunk(self, u_store: torch.Tensor) -> torch.Tensor:
        """Chunked (P, nz, Npad) → reference layout (P, N, nz)."""
        P = u_store.shape[0]
        out = torch.empty((P, self.n, self.nz), dtype=self.cdtype, device=self.device)
        o = self.op()
        rc = self.lib.tp_cn2d_unchunk(ctypes.byref(o), P, _ptr(u_store), _ptr(out), _stream(self.device))
        _native.check(rc, "tp_cn2d_unchunk", self.lib)
        return out

    def chunk_index(self) -> torch.Tensor:
        """Offsets of matrix rows 0..N−1 within one chunked slice (Npad)."""
        if getattr(self, "_chunk_idx", None) is None:
            g = torch.arange(self.n)
            i, k = g % self.rows_per_chunk, g // self.rows_per_chunk
            if self.chunks == 128:
                off = ((i // 2) * self.chunks + k) * 2 + (i % 2)
            else:
                off = i * self.chunks + k
            self._chunk_idx = off.to(self.device)
        return self._chunk_idx

    def unchunk_rows(self, x: torch.Tensor) -> torch.Tensor:
        """(..., Npad) chunked → (..., N) natural row order."""
        return x.index_select(-1, self.chunk_index())

    def new_grad_buffer(self) -> torch.Tensor:
        return torch.zeros((self.L, self.npad), dtype=self.cdtype, device=self.device)

    def grad_to_n(self, grad_c: torch.Tensor, field: Optional[torch.Tensor] = None, is_delta=False) -> torch.Tensor:
        """Σ_p λ conj(u_s + u_{s−1}) (L, Npad chunked) → torch-convention gradient on n (n_obj, nz)."""
        out = torch.empty((self.n_obj, self.nz), dtype=self.cdtype, device=self.device)
        dtype = _native.C128
        if field is not None:
            field = self._check_field(field)
            dtype = _native.C128 if field.dtype == torch.complex128 else _native.C64
        o = self.op(is_delta)
        rc = self.lib.tp_cn2d_grad_to_n(ctypes.byref(o), _ptr(grad_c), _ptr(field), dtype, _ptr(out), _stream(self.device))
        _native.check(rc, "tp_cn2d_grad_to_n", self.lib)
        return out

    def grad_to_n_range(self, grad_c: torch.Tensor, out: torch.Tensor, node_begin: int, node_end: int,
                        field: Optional[torch.Tensor] = None, is_delta=False) -> torch.Tensor:
        """:meth:`grad_to_n` for node columns ``node_begin..node_end`` of ``out`` only."""
        dtype = _native.C128
        if field is not None:
            field = self._check_field(field)
            dtype = _native.C128 if field.dtype == torch.complex128 else _native.C64
        o = self.op(is_delta)
        rc = self.lib.tp_cn2d_grad_to_n_range(ctypes.byref(o), _ptr(grad_c), _ptr(field), dtype, _ptr(out),
                                              int(node_begin), int(node_end), _stream(self.device))
        _native.check(rc, "tp_cn2d_grad_to_n_range", self.lib)
        return out

    def device_status(self):
        code = ctypes.c_int32()
        rc = self.lib.tp_device_status(_stream(self.device), ctypes.byref(code))
        _native.check(rc, "tp_device_status", self.lib)
