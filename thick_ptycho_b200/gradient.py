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

import ctypes
import math
from typing import Optional, Union

import numpy as np
import torch

from . import _native, heads
from .cn2d import CN2D


def _as_device(x, device, dtype):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype, non_blocking=True)
    return torch.from_numpy(np.ascontiguousarray(x)).to(device=device, dtype=dtype, non_blocking=True)


def amplitude_residual(exit_waves: torch.Tensor, amplitude: torch.Tensor):
    """Loss ``Σ(|F e| − a)²`` and its gradient w.r.t. e (torch convention).

    Equals ``2N(e − P_GS(e))`` with P_GS the reference's modulus projection
    (``base_reconstructor.py:171-207``); one fused libtpcuda kernel
    (FFT, residual, inverse FFT) per row group.
    """
    return heads.amplitude_residual(exit_waves.contiguous(), amplitude)


class PWEGradient2D:
    """Amplitude-loss gradient of a 2D geometry, all probes batched.

    ``geometry`` is a reference ``SimulationSpace2D`` or a
    :class:`~thick_ptycho_b200.geometry.SimulationGeometry`.

    ``checkpoint``: ``"sqrt"`` keeps the field every ⌈√L⌉ slices during the
    forward march and recomputes each segment before its adjoint sweep
    (memory ∝ √L per probe, one extra forward march); ``None`` keeps every
    slice (memory ∝ L, fastest); an int sets the checkpoint spacing.
    """

    def __init__(self, geometry, bc_type="impedance", device=None, checkpoint: Union[str, int, None] = None):
        self.geometry = geometry
        self.engine = CN2D(
            geometry.block_size, geometry.nz, geometry.k, geometry.dx, geometry.dz, bc_type,
            empty_px=int(getattr(geometry, "empty_space_px", 0) or 0),
            exact_ref_coeff=bool(getattr(geometry, "exact_ref_coeff", False)), device=device,
        )
        self.device = self.engine.device
        L = self.engine.L
        if checkpoint == "sqrt":
            self.ckpt = max(1, math.ceil(math.sqrt(L)))
        elif checkpoint is None or checkpoint == 0:
            self.ckpt = 0
        else:
            self.ckpt = int(checkpoint)
        if self.ckpt >= L:
            self.ckpt = 0
        # team path: the kept field holds the half pair sums (u_s + u_{s-1})/2, so the
        # exact-adjoint march reads one slice per step and runs in Cayley form
        self.sums = self.engine.chunks == 128
        self._ff = self.engine.new_factor_buffer()
        self._fa = self.engine.new_factor_buffer()
        self._copy_stream = None
        self._factor_stream = None
        self._n_dev = None
        self._bufs = {}
        self._grad_c = self.engine.new_grad_buffer()

    def _buf(self, name, P, slices):
        b = self._bufs.get(name)
        if b is None or b.shape[0] != P or b.shape[1] != slices:
            b = self.engine.new_store(P, slices)
            self._bufs[name] = b
        return b

    def field_bytes(self, P) -> int:
        """Device bytes of the stored forward field for P probes."""
        e = self.engine
        if not self.ckpt:
            return P * e.nz * e.npad * 8
        return P * (e.L // self.ckpt + 1 + self.ckpt + 1 + 2) * e.npad * 8

    def forward(self, field: torch.Tensor, probes: torch.Tensor, is_delta=False, exit_out=None, probes_ready=None):
        """Forward march keeping the field (every slice, or the checkpoints).

        ``probes_ready``: a CUDA event the march waits for (the probes may
        still be in flight on another stream while the slices factorise)."""
        P = probes.shape[0]
        e = self.engine
        fs = e.factor(field, "forward", is_delta, out=self._ff)
        if probes_ready is not None:
            torch.cuda.current_stream(self.device).wait_event(probes_ready)
        ex = exit_out if exit_out is not None else torch.empty((P, e.n), dtype=torch.complex64, device=self.device)
        if not self.ckpt:
            e.march(fs, P, probes=probes, u_store=self._buf("full", P, e.nz), exit_out=ex, store_sums=self.sums)
        else:
            ck = self._buf("ckpt", P, e.L // self.ckpt + 1)
            e.march(fs, P, probes=probes, u_store=ck, store_every=self.ckpt, exit_out=ex)
        self._fs_fwd = fs
        return ex

    def _n_device(self) -> torch.Tensor:
        """Device buffer for a host index field (complex128, (n_obj, nz))."""
        e = self.engine
        if self._n_dev is None:
            self._n_dev = torch.empty((e.n_obj, e.nz), dtype=torch.complex128, device=self.device)
        return self._n_dev

    # Range boundaries as fractions of the slices: a short first range, so
    # that little of the index field (and, for the adjoint, which runs the
    # ranges backwards, little of the gradient) is exposed outside the
    # overlap, then ranges doubling in length, so that each range's index
    # columns arrive and its slices are factorised while the one before it
    # marches.
    _RANGE_FRACTIONS = (0.0, 1.0 / 32.0, 1.0 / 16.0, 1.0 / 8.0, 1.0 / 4.0, 1.0 / 2.0, 1.0)

    def _slice_ranges(self):
        """Consecutive slice ranges covering 1..L (1-based, inclusive)."""
        L = self.engine.L
        b = sorted({round(f * L) for f in self._RANGE_FRACTIONS})
        return [(b[k] + 1, b[k + 1]) for k in range(len(b) - 1) if b[k + 1] > b[k]]

    def _forward_ranges(self, fs, probes, probes_ready, ranges, prepare):
        """Forward march range by range, each after its slices were factorised
        into ``fs``: the first range's already on this stream; ``prepare(k)``
        enqueues what range k > 0 needs and returns the event its march waits
        for, so that the host enqueues each range right after the one before.
        The state passes from range to range; the stored field and the exit
        wave are those of one march over all slices."""
        e = self.engine
        P = probes.shape[0]
        main = torch.cuda.current_stream(self.device)
        ex = torch.empty((P, e.n), dtype=torch.complex64, device=self.device)
        store = self._buf("full", P, e.nz)
        state = [self._buf("range_state0", P, 1)[:, 0], self._buf("range_state1", P, 1)[:, 0]]
        last = len(ranges) - 1
        for k, (s0, s1) in enumerate(ranges):
            main.wait_event(probes_ready if k == 0 else prepare(k))
            e.march(fs, P, probes=probes if k == 0 else None, u_store=store, exit_out=ex, t_begin=s0, t_end=s1,
                    state_in=None if k == 0 else state[(k - 1) % 2], state_out=None if k == last else state[k % 2],
                    store_sums=self.sums)
        self._fs_fwd = fs
        return ex

    def _backward_ranges(self, field, exit_grad, grad_out, side, fa):
        """:meth:`backward` (full field kept, exact-adjoint factor set ``fa``
        ready on this stream) with the adjoint run range by range from the last
        slice down: once slices s0..L are done, index nodes s0..nz-1 are final
        (node t reads slices t and t+1), so they are mapped and copied into the
        host tensor `grad_out` on the side stream while the adjoint goes on with
        the earlier slices.  Returns the device gradient."""
        e = self.engine
        P = exit_grad.shape[0]
        main = torch.cuda.current_stream(self.device)
        self._grad_c.zero_()
        src = exit_grad.contiguous()
        gn = torch.empty((e.n_obj, e.nz), dtype=torch.complex64, device=self.device)
        state = [self._buf("range_state0", P, 1)[:, 0], self._buf("range_state1", P, 1)[:, 0]]
        ranges = self._slice_ranges()[::-1]  # last slices first
        hi = e.nz - 1  # highest node not yet mapped
        for k, (s0, s1) in enumerate(ranges):
            # slices s1 .. s0 are steps L+1-s1 .. L+1-s0 of the adjoint march
            e.march(fa, P, src_exit=src if k == 0 else None, u_fwd=self._buf("full", P, e.nz), grad_c=self._grad_c,
                    t_begin=e.L + 1 - s1, t_end=e.L + 1 - s0,
                    state_in=None if k == 0 else state[(k - 1) % 2],
                    state_out=None if k == len(ranges) - 1 else state[k % 2], store_sums=self.sums)
            lo = 0 if k == len(ranges) - 1 else s0
            e.grad_to_n_range(self._grad_c, gn, lo, hi, field if e.exact_ref_coeff else None)
            side.wait_stream(main)
            with torch.cuda.stream(side):
                rc = e.lib.tp_copy_columns(ctypes.c_void_p(grad_out.data_ptr()), ctypes.c_void_p(gn.data_ptr()),
                                           e.n_obj, e.nz * 8, lo * 8, (hi - lo + 1) * 8,
                                           ctypes.c_void_p(side.cuda_stream))
                _native.check(rc, "tp_copy_columns")
            hi = lo - 1
        gn.record_stream(side)
        return gn

    def backward(self, field: torch.Tensor, exit_grad: torch.Tensor, is_delta=False, fa=None) -> torch.Tensor:
        """Exact adjoint from the exit-wave gradient; returns ∂ℓ/∂n (n_obj, nz).

        Must follow :meth:`forward` with the same field (it reuses the kept
        field and, when checkpointing, the forward factor set).  ``fa``: the
        field's exact-adjoint factor set when already computed.
        """
        P = exit_grad.shape[0]
        e = self.engine
        if fa is None:
            fa = e.factor(field, "adjoint_exact", is_delta, out=self._fa)
        self._grad_c.zero_()
        src = exit_grad.contiguous()
        if not self.ckpt:
            e.march(fa, P, src_exit=src, u_fwd=self._buf("full", P, e.nz), grad_c=self._grad_c,
                    store_sums=self.sums)
        else:
            S, L = self.ckpt, e.L
            ck = self._bufs["ckpt"]
            seg = self._buf("segment", P, S + 1)
            state = [self._buf("state0", P, 1)[:, 0], self._buf("state1", P, 1)[:, 0]]
            start = self._buf("start", P, 1)[:, 0]
            nseg = -(-L // S)
            first = True
            for k in reversed(range(nseg)):
                a, b = k * S, min(k * S + S, L)
                start.copy_(ck[:, a // S])
                # recompute u_a .. u_b of this segment (indices 0 .. b - a)
                e.march(self._fs_fwd, P, t_begin=a + 1, t_end=b, state_in=start, u_store=seg, store_base=a,
                        store_sums=self.sums)
                # adjoint steps for slices b .. a+1 (step t = L + 1 - s)
                e.march(fa, P, t_begin=L + 1 - b, t_end=L - a, src_exit=src if first else None,
                        state_in=None if first else state[0], state_out=state[1], u_fwd=seg, ufwd_base=a,
                        grad_c=self._grad_c, store_sums=self.sums)
                state.reverse()
                first = False
        return e.grad_to_n(self._grad_c, field if e.exact_ref_coeff else None, is_delta)

    def step_gradient(self) -> torch.Tensor:
        """Σ_p λ_s conj(u_s + u_{s−1}) of the last backward pass, (L, N) natural rows."""
        return self.engine.unchunk_rows(self._grad_c)

    def loss_and_grad(self, n, probes, amplitude, grad_out: Optional[torch.Tensor] = None):
        """One forward + adjoint pass: ``(loss, ∂loss/∂n)``.

        ``n``: refractive index (n_obj, nz) as the reference's solvers take it
        (complex128); ``probes``: (P, N); ``amplitude``: measured ``√I`` (P, N).
        Host inputs are copied to the device; if ``grad_out`` is a host tensor
        the gradient is copied back into it.  Returns a float loss.
        """
        main = torch.cuda.current_stream(self.device)
        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream(self.device)
        side = self._copy_stream
        side.wait_stream(main)
        e = self.engine
        streamed = (isinstance(n, torch.Tensor) and not n.is_cuda and n.dtype == torch.complex128
                    and n.is_contiguous() and tuple(n.shape) == (e.n_obj, e.nz) and not self.ckpt and e.L >= 64)
        if streamed:
            # A host index field goes up in column blocks on the side stream
            # (slice s needs index columns s-1 and s).  The first block's
            # slices are factorised on this stream as soon as it lands (while
            # the probes follow it up); every later block's slices, and then
            # the exact-adjoint factor set, on the factor stream, beside the
            # marches (which leave SMs free); each range marches once its
            # slices are factorised, and the amplitudes go up last.
            field = self._n_device()
            ranges = self._slice_ranges()
            if self._factor_stream is None:
                self._factor_stream = torch.cuda.Stream(self.device)
            fstream = self._factor_stream
            fstream.wait_stream(main)

            def columns(c0, c1):
                rc = e.lib.tp_copy_columns(ctypes.c_void_p(field.data_ptr()), ctypes.c_void_p(n.data_ptr()),
                                           e.n_obj, e.nz * 16, c0 * 16, (c1 - c0 + 1) * 16,
                                           ctypes.c_void_p(side.cuda_stream))
                _native.check(rc, "tp_copy_columns")
                return side.record_event()

            with torch.cuda.stream(side):
                arrived = columns(0, ranges[0][1])
            main.wait_event(arrived)
            fs = e.factor_range(field, "forward", ranges[0][0], ranges[0][1], out=self._ff)
            first_done = main.record_event()  # the first range also resets the PCR coupling bound
            with torch.cuda.stream(side):
                pr = _as_device(probes, self.device, torch.complex64)
                pr_ready = side.record_event()
            fstream.wait_event(first_done)

            def prepare(k):
                s0, s1 = ranges[k]
                with torch.cuda.stream(side):
                    arrived = columns(s0, s1)
                with torch.cuda.stream(fstream):
                    fstream.wait_event(arrived)
                    e.factor_range(field, "forward", s0, s1, out=self._ff)
                    return fstream.record_event()
        else:
            field = _as_device(n, self.device, torch.complex128)
            # Host probes and amplitudes travel on a side stream after n, so that
            # their copies overlap the factorisation and the forward march (n is
            # needed first; the probes at the march, the amplitudes at the residual).
            with torch.cuda.stream(side):
                pr = _as_device(probes, self.device, torch.complex64)
                pr_ready = side.record_event()
                amp = _as_device(amplitude, self.device, torch.float64)
                amp_ready = side.record_event()
        pr.record_stream(main)
        if streamed:
            ex = self._forward_ranges(fs, pr, pr_ready, ranges, prepare)
            with torch.cuda.stream(side):
                amp = _as_device(amplitude, self.device, torch.float64)
                amp_ready = side.record_event()
            with torch.cuda.stream(fstream):  # all index columns have arrived
                fa = e.factor(field, "adjoint_exact", out=self._fa)
                fa_ready = fstream.record_event()
        else:
            ex = self.forward(field, pr, probes_ready=pr_ready)
        amp.record_stream(main)
        main.wait_event(amp_ready)
        loss, ge = amplitude_residual(ex, amp)
        host_out = (grad_out is not None and not grad_out.is_cuda and grad_out.dtype == torch.complex64
                    and grad_out.is_contiguous() and tuple(grad_out.shape) == (e.n_obj, e.nz))
        if streamed:
            main.wait_event(fa_ready)
        if streamed and host_out:
            g = self._backward_ranges(field, ge, grad_out, side, fa)
            main.wait_stream(side)
        else:
            g = self.backward(field, ge, fa=fa if streamed else None)
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
