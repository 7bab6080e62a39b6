"""Host-side assembly of the compact step operators.

The reference builds sparse ``A_step = I − K`` and ``B_step = I + K``
(``operator_matrices.py:36-126``) with boundary-row edits
(``boundary_conditions.py:9-130``).  For the GPU kernels only K's interior
values and its edited boundary entries are needed; this module computes them
with the same formulas.
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import Enum

import numpy as np

BC_TYPES = ("dirichlet", "neumann", "impedance", "impedance2")


def normalize_bc(bc_type) -> str:
    """Accept a ``BoundaryType``-like Enum or a string; return the string.

    The reference compares ``bc_type`` against strings, so its Enum default
    silently degrades to Neumann in 2D and raises in 3D; this drop-in takes
    the Enum's value instead.
    """
    if isinstance(bc_type, Enum):
        bc_type = bc_type.value
    bc_type = str(bc_type).lower()
    if bc_type not in BC_TYPES:
        raise ValueError(f"Invalid boundary condition type {bc_type!r}; expected one of {BC_TYPES}")
    return bc_type


@dataclass(frozen=True)
class BCCoefficients:
    """μ, β and γ of ``boundary_conditions.py:9-55``."""

    mu_x: complex
    mu_y: complex
    beta_x: complex
    beta_y: complex
    gamma: complex

    @classmethod
    def make(cls, k, dx, dz, bc_type, dy=None, dimension=2):
        a = 1j / (2 * k)
        mu_x = a * (0.5 * dz / dx**2)
        mu_y = a * (0.5 * dz / dy**2) if dimension == 3 else 0.0
        beta_x = beta_y = gamma = 0.0
        if bc_type in ("impedance", "impedance2"):
            beta_x = mu_x * 2j * k * dx
            beta_y = mu_y * 2j * k * dy if dimension == 3 else 0.0
        if bc_type == "impedance2":
            gamma = -1 / (2j * k)
        return cls(complex(mu_x), complex(mu_y), complex(beta_x), complex(beta_y), complex(gamma))


@dataclass(frozen=True)
class Operator1D:
    """K = tridiag(k_off, k_diag, k_off) with edited corner entries.

    ``k_d0 = K[0,0]``, ``k_dn = K[N−1,N−1]``, ``k_01 = K[0,1]``,
    ``k_nm = K[N−1,N−2]``; every other entry equals the interior value.
    """

    n: int
    k_off: complex
    k_diag: complex
    k_d0: complex
    k_dn: complex
    k_01: complex
    k_nm: complex

    def dense(self) -> np.ndarray:
        """Dense K (for tests)."""
        K = np.zeros((self.n, self.n), dtype=complex)
        i = np.arange(self.n)
        K[i, i] = self.k_diag
        K[i[1:], i[:-1]] = self.k_off
        K[i[:-1], i[1:]] = self.k_off
        K[0, 0], K[-1, -1], K[0, 1], K[-1, -2] = self.k_d0, self.k_dn, self.k_01, self.k_nm
        return K


def operator_1d(n, co: BCCoefficients, bc_type: str, dz: float) -> Operator1D:
    """K of ``operator_matrices.py:36-72`` for an n-row transverse axis.

    The interior diagonal is ``−2(μx + μy)`` (μy is 0 in 2D); Dirichlet zeroes
    the two boundary rows; otherwise the Neumann edit doubles the two
    boundary couplings and the impedance variants shift the corners.
    """
    mu = co.mu_x
    diag = -2 * (co.mu_x + co.mu_y)
    if bc_type == "dirichlet":
        return Operator1D(n, mu, diag, 0j, 0j, 0j, 0j)
    d0 = dn = diag
    c01 = cnm = 2 * mu
    if bc_type == "impedance":
        d0 += co.beta_x
        dn += co.beta_x
    elif bc_type == "impedance2":
        g = co.gamma / dz**2
        d0 += co.beta_x + g
        dn += co.beta_x + g
        c01 += -g
        cnm += -g
    return Operator1D(n, complex(mu), complex(diag), complex(d0), complex(dn), complex(c01), complex(cnm))
