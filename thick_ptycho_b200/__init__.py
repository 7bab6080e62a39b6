"""thick_ptycho_b200: the thick_ptycho paraxial (PWE) hot path on NVIDIA B200.

Public entry points:

* :class:`PWEGpuSolver` -- drop-in for the reference ``PWEIterativeLUSolver``
  (same constructor, ``solve``, ``_solve_single_probe``,
  ``prepare_solver_caches``, ``reset_cache``, ``get_gradient``,
  ``get_exit_waves``, ``get_farfield_intensities``).
* :class:`PWEGpuPiTSolver` -- drop-in for ``PWEFullPinTSolver`` (the
  α-circulant preconditioned space-time GMRES, 2D forward mode).
* :class:`MSGpuSolver` -- drop-in for ``MSForwardModelSolver`` (2D, and 3D
  spaces, which the reference rejects).
* :class:`CN2D` -- batched 2D Crank–Nicolson propagation on device tensors.
* :class:`SimulationGeometry` -- the geometry attributes the solvers read.

The kernels live in ``libtpcuda.so`` (C ABI in ``include/tpcuda.h``), built by
``python -m thick_ptycho_b200.build_native``.  There is no CPU fallback.
"""

from .geometry import SimulationGeometry, scan_centres_1d, order_scan_2d  # noqa: F401
from .operators import BCCoefficients, normalize_bc, operator_1d  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # GPU-facing classes import torch lazily.
    if name == "PWEGpuSolver":
        from .solver import PWEGpuSolver

        return PWEGpuSolver
    if name == "PWEGpuPiTSolver":
        from .pit import PWEGpuPiTSolver

        return PWEGpuPiTSolver
    if name == "MSGpuSolver":
        from .ms2d import MSGpuSolver

        return MSGpuSolver
    if name == "CN2D":
        from .cn2d import CN2D

        return CN2D
    raise AttributeError(name)
