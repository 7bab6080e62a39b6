"""FFT heads on the GPU: batched FFTs, far-field intensities and the
amplitude-loss residual, on libtpcuda's shared-memory mixed-radix FFT.

Replace ``numpy.fft`` in the far field (``forward_model/base/base_solver.py:
234-242``) and the phase-retrieval projection
(``reconstruction/base_reconstructor.py:171-207``).  Rows of length
n = 2^a 3^b 5^c ≤ 4096, complex64.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native


def fft_plannable(n: int) -> bool:
    """True when libtpcuda's shared-memory FFT handles length n (2^a 3^b 5^c ≤ 4096)."""
    n = int(n)
    if n < 1 or n > 4096:
        return False
    for f in (2, 3, 5):
        while n % f == 0:
            n //= f
    return n == 1


def _stream(t: torch.Tensor):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _check(t: torch.Tensor, name, dtype=torch.complex64):
    if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
        raise TypeError(f"{name} must be a contiguous {dtype} CUDA tensor")


def fft1d(x: torch.Tensor, inverse: bool = False, out: torch.Tensor = None) -> torch.Tensor:
    """FFT along the last axis (numpy conventions)."""
    _check(x, "x")
    n = x.shape[-1]
    out = torch.empty_like(x) if out is None else out
    rc = _native.load().tp_fft1d(n, x.numel() // n, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 int(inverse), _stream(x))
    _native.check(rc, "tp_fft1d")
    return out


def fft2_last(x: torch.Tensor, inverse: bool = False) -> torch.Tensor:
    """2D FFT over the last two axes (numpy conventions) with the 1D FFT head:
    a pass along the last axis, a transpose, a pass along the other axis and a
    transpose back.  Both lengths must be 2^a 3^b 5^c ≤ 4096."""
    _check(x, "x")
    n0, n1 = x.shape[-2], x.shape[-1]
    if not (fft_plannable(n0) and fft_plannable(n1)):
        raise ValueError(f"fft2_last needs 2^a 3^b 5^c <= 4096 lengths, got {n0} x {n1}")
    y = fft1d(x, inverse)
    yt = y.transpose(-1, -2).contiguous()
    z = fft1d(yt, inverse)
    return z.transpose(-1, -2).contiguous()


def farfield_intensity(exit_waves: torch.Tensor) -> torch.Tensor:
    """``|FFT(exit)|²`` along the last axis, float32."""
    _check(exit_waves, "exit_waves")
    n = exit_waves.shape[-1]
    out = torch.empty(exit_waves.shape, dtype=torch.float32, device=exit_waves.device)
    rc = _native.load().tp_farfield_intensity(n, exit_waves.numel() // n, ctypes.c_void_p(exit_waves.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()), _stream(exit_waves))
    _native.check(rc, "tp_farfield_intensity")
    return out


def amplitude_residual(exit_waves: torch.Tensor, amplitude: torch.Tensor, grad_out: torch.Tensor = None,
                       loss_out: torch.Tensor = None):
    """Loss ``Σ(|F e| − a)²`` (float64 device scalar) and ``∂loss/∂e`` (torch convention)."""
    _check(exit_waves, "exit_waves")
    amp = amplitude if amplitude.dtype == torch.float32 else amplitude.to(torch.float32)
    _check(amp.contiguous(), "amplitude", torch.float32)
    amp = amp.contiguous()
    n = exit_waves.shape[-1]
    grad = torch.empty_like(exit_waves) if grad_out is None else grad_out
    loss = torch.zeros((), dtype=torch.float64, device=exit_waves.device) if loss_out is None else loss_out.zero_()
    rc = _native.load().tp_amplitude_residual(n, exit_waves.numel() // n, ctypes.c_void_p(exit_waves.data_ptr()),
                                              ctypes.c_void_p(amp.data_ptr()), ctypes.c_void_p(grad.data_ptr()),
                                              ctypes.c_void_p(loss.data_ptr()), _stream(exit_waves))
    _native.check(rc, "tp_amplitude_residual")
    return loss, grad
