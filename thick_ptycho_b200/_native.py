"""ctypes binding of libtpcuda.so (declared in include/tpcuda.h).

The library is built in-tree by :mod:`thick_ptycho_b200.build_native`.  There
is no fallback: if it is missing or fails to load, every GPU entry point
raises :class:`NativeLibraryError`.
"""

from __future__ import annotations

import ctypes
import os
import threading

from .build_native import LIB, LIB_C128

_lock = threading.Lock()
_lib = None
_lib_c128 = None

TP_OK = 0
TP_ERR_TIMEOUT = 4

MODE_FORWARD = 0
MODE_ADJOINT = 1
MODE_REVERSE = 2
MODE_ADJOINT_EXACT = 3
MODES = {"forward": MODE_FORWARD, "adjoint": MODE_ADJOINT, "reverse": MODE_REVERSE, "adjoint_exact": MODE_ADJOINT_EXACT}

C128 = 0
C64 = 1


class NativeLibraryError(RuntimeError):
    """libtpcuda.so is missing, failed to load, or a call returned an error."""


class TpCn2dOp(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("n_obj", ctypes.c_int32),
        ("empty_px", ctypes.c_int32),
        ("exact_ref_coeff", ctypes.c_int32),
        ("field_is_delta", ctypes.c_int32),
        ("k", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("k_off", ctypes.c_double * 2),
        ("k_diag", ctypes.c_double * 2),
        ("k_d0", ctypes.c_double * 2),
        ("k_dn", ctypes.c_double * 2),
        ("k_01", ctypes.c_double * 2),
        ("k_nm", ctypes.c_double * 2),
    ]


class TpCn2dMarchArgs(ctypes.Structure):
    _fields_ = [
        ("num_probes", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("probes", ctypes.c_void_p),
        ("src_shared", ctypes.c_void_p),
        ("src_probe", ctypes.c_void_p),
        ("src_exit", ctypes.c_void_p),
        ("u_store", ctypes.c_void_p),
        ("exit_out", ctypes.c_void_p),
        ("u_fwd", ctypes.c_void_p),
        ("grad_c", ctypes.c_void_p),
        ("t_begin", ctypes.c_int32),
        ("t_end", ctypes.c_int32),
        ("state_in", ctypes.c_void_p),
        ("state_out", ctypes.c_void_p),
        ("store_slices", ctypes.c_int32),
        ("store_every", ctypes.c_int32),
        ("store_base", ctypes.c_int32),
        ("ufwd_slices", ctypes.c_int32),
        ("ufwd_base", ctypes.c_int32),
        ("store_sums", ctypes.c_int32),
    ]


class TpMs2dOp(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("k", ctypes.c_double),
        ("dx", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("n_medium", ctypes.c_double * 2),
    ]


class TpPitArgs(ctypes.Structure):
    _fields_ = [
        ("num_probes", ctypes.c_int32),
        ("restart", ctypes.c_int32),
        ("max_cycles", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("alpha", ctypes.c_double),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("probes", ctypes.c_void_p),
        ("rhs", ctypes.c_void_p),
        ("u", ctypes.c_void_p),
        ("iters", ctypes.POINTER(ctypes.c_int32)),
        ("resid", ctypes.POINTER(ctypes.c_double)),
    ]


class TpMs3dOp(ctypes.Structure):
    _fields_ = [
        ("n1", ctypes.c_int32),
        ("n2", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("k", ctypes.c_double),
        ("d1", ctypes.c_double),
        ("d2", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("n_medium", ctypes.c_double * 2),
    ]


class TpCn3dOp(ctypes.Structure):
    _fields_ = [
        ("nf", ctypes.c_int32), ("nb", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("exact_ref_coeff", ctypes.c_int32), ("field_is_delta", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("k", ctypes.c_double), ("dz", ctypes.c_double),
        ("mu_x", ctypes.c_double * 2), ("mu_y", ctypes.c_double * 2),
        ("kc", ctypes.c_void_p), ("kw", ctypes.c_void_p), ("ke", ctypes.c_void_p), ("ks", ctypes.c_void_p),
        ("kn", ctypes.c_void_p),
    ]


class TpCn3dMarchArgs(ctypes.Structure):
    _fields_ = [
        ("num_probes", ctypes.c_int32), ("mode", ctypes.c_int32), ("max_iter", ctypes.c_int32),
        ("precond", ctypes.c_int32), ("host_check", ctypes.c_int32), ("launch", ctypes.c_int32),
        ("tol", ctypes.c_double),
        ("probes", ctypes.c_void_p), ("src_shared", ctypes.c_void_p), ("src_exit", ctypes.c_void_p),
        ("u_store", ctypes.c_void_p), ("exit_out", ctypes.c_void_p), ("u_fwd", ctypes.c_void_p),
        ("grad_c", ctypes.c_void_p), ("stats", ctypes.c_void_p),
        ("model", ctypes.c_void_p), ("learned_ws", ctypes.c_void_p), ("learned_ws_bytes", ctypes.c_size_t),
        ("train_z0", ctypes.c_void_p), ("train_sol", ctypes.c_void_p), ("train_diag", ctypes.c_void_p),
        ("train_every", ctypes.c_int32), ("train_kind", ctypes.c_int32),
        ("learned_reuse", ctypes.c_int32), ("kernels", ctypes.c_int32),
    ]


class TpCnnModel(ctypes.Structure):
    _fields_ = [
        ("w", ctypes.c_void_p * 4),
        ("b", ctypes.c_void_p * 4),
        ("kappa", ctypes.c_float),
        ("out_scale", ctypes.c_float),
    ]


CONV_RELU = 0
CONV_MASK = 1
CONV_FILTER = 2

# (name, restype, argtypes) of every exported symbol of include/tpcuda.h
SIGNATURES = [
    ("tp_cn2d_layout", ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_int32)]),
    ("tp_cn2d_factor_bytes", ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    ("tp_cn2d_factor", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    ("tp_cn2d_factor_range", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_void_p]),
    ("tp_copy_columns", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p]),
    ("tp_cn2d_march", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.POINTER(TpCn2dMarchArgs),
                                     ctypes.c_void_p]),
    ("tp_cn2d_grad_to_n", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    ("tp_cn2d_grad_to_n_range", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                               ctypes.c_void_p]),
    ("tp_cn2d_unchunk", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]),
    ("tp_cn2d_march_noalloc", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.c_int32,
                                             ctypes.POINTER(TpCn2dMarchArgs), ctypes.c_void_p]),
    ("tp_cn2d_ref_gradient", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("tp_cn2d_alpha_source", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    ("tp_fft1d", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                ctypes.c_void_p]),
    ("tp_farfield_intensity", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    ("tp_amplitude_residual", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("tp_ms2d_transmission", ctypes.c_int, [ctypes.POINTER(TpMs2dOp), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    ("tp_ms2d_march", ctypes.c_int, [ctypes.POINTER(TpMs2dOp), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("tp_ms2d_backward", ctypes.c_int, [ctypes.POINTER(TpMs2dOp), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ("tp_ms2d_3pie_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    ("tp_ms2d_3pie", ctypes.c_int, [ctypes.POINTER(TpMs2dOp), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                    ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    ("tp_ms3d_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32] * 3),
    ("tp_pit_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32] * 4),
    ("tp_pit_solve", ctypes.c_int, [ctypes.POINTER(TpCn2dOp), ctypes.c_void_p, ctypes.c_int32,
                                    ctypes.POINTER(TpPitArgs), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    ("tp_ms3d_transmission", ctypes.c_int, [ctypes.POINTER(TpMs3dOp), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    ("tp_ms3d_march", ctypes.c_int, [ctypes.POINTER(TpMs3dOp), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.c_void_p]),
    ("tp_ms3d_backward", ctypes.c_int, [ctypes.POINTER(TpMs3dOp), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.c_void_p]),
    ("tp_cn3d_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    ("tp_cn3d_learned_ws_bytes", ctypes.c_size_t, [ctypes.c_int32] * 4),
    ("tp_cn3d_march", ctypes.c_int, [ctypes.POINTER(TpCn3dOp), ctypes.c_void_p, ctypes.c_int32,
                                     ctypes.POINTER(TpCn3dMarchArgs), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    ("tp_cnn_act_bytes", ctypes.c_size_t, [ctypes.c_int32] * 4),
    ("tp_cnn_features", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_float,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    ("tp_conv3x3_bf16", ctypes.c_int, [ctypes.c_int32] * 5 + [ctypes.c_void_p] * 5 + [ctypes.c_float, ctypes.c_void_p]),
    ("tp_conv3x3_wgrad", ctypes.c_int, [ctypes.c_int32] * 4 + [ctypes.c_void_p] * 5),
    ("tp_cnn_filter_apply", ctypes.c_int, [ctypes.c_int32] * 5 + [ctypes.c_void_p] * 4),
    ("tp_cnn_filter_grad", ctypes.c_int, [ctypes.c_int32] * 4 + [ctypes.c_void_p] * 2 + [ctypes.c_float] +
     [ctypes.c_void_p] * 2),
    ("tp_cnn_forward_ws_bytes", ctypes.c_size_t, [ctypes.c_int32] * 3),
    ("tp_cnn_forward", ctypes.c_int, [ctypes.c_int32] * 3 + [ctypes.POINTER(TpCnnModel), ctypes.c_void_p,
                                                             ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                                             ctypes.c_void_p]),
    ("tp_device_status", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ("tp_last_error_string", ctypes.c_char_p, []),
    ("tp_version", ctypes.c_int, []),
]


def lib_path() -> str:
    return os.environ.get("TPCUDA_LIB", LIB)


def load() -> ctypes.CDLL:
    """Load libtpcuda.so once; raise NativeLibraryError if it is unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = lib_path()
        if not os.path.exists(path):
            raise NativeLibraryError(
                f"{path} not found: build it with `python -m thick_ptycho_b200.build_native` "
                "(there is no CPU fallback)"
            )
        try:
            lib = ctypes.CDLL(path)
        except OSError as e:  # pragma: no cover - depends on the machine
            raise NativeLibraryError(f"failed to load {path}: {e}") from e
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def load_check() -> ctypes.CDLL:
    """Load libtpcuda_c128.so, the complex128 check build of the 2D and 3D
    Crank–Nicolson entry points (tp_cn2d_*, tp_cn3d_*: every complex buffer
    complex128)."""
    global _lib_c128
    if _lib_c128 is not None:
        return _lib_c128
    with _lock:
        if _lib_c128 is not None:
            return _lib_c128
        if not os.path.exists(LIB_C128):
            raise NativeLibraryError(f"{LIB_C128} not found: build it with `python -m thick_ptycho_b200.build_native`")
        try:
            lib = ctypes.CDLL(LIB_C128)
        except OSError as e:  # pragma: no cover - depends on the machine
            raise NativeLibraryError(f"failed to load {LIB_C128}: {e}") from e
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name, None)
            if fn is not None:
                fn.restype = res
                fn.argtypes = args
        _lib_c128 = lib
        return lib


def check(rc: int, what: str, lib=None):
    if rc != TP_OK:
        msg = (lib or load()).tp_last_error_string().decode(errors="replace")
        raise NativeLibraryError(f"{what} failed (status {rc}): {msg}")
