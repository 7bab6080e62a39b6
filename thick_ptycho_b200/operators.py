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


def operator_2d_diagonals(nx, ny, co: BCCoefficients, bc_type: str):
    """The 5 diagonals of the 3D (2D-transverse) scaled Laplacian K, K = I − A.

    Restates ``operator_matrices.py:75-126`` and ``boundary_conditions.py:
    96-130`` row by row.  The operator acts on vectors of length nx·ny with
    index ``i = b·nx + f`` (``f`` the fast index of ``kron(I_y, A_x)``); the
    1D part carries the x-edge rules (Dirichlet zero rows, Neumann doubled
    couplings, impedance ``+β_x``) and the block part the y-edge rules
    (Dirichlet identity blocks, doubled block couplings, impedance ``+β_y``).
    Returns ``(center, west, east, south, north)`` complex128 arrays of
    length nx·ny: ``(K x)_i = c_i x_i + w_i x_{i−1} + e_i x_{i+1} + s_i x_{i−nx}
    + n_i x_{i+nx}`` (coefficients are zero where the neighbour is absent).
    """
    if bc_type not in ("dirichlet", "neumann", "impedance"):
        raise ValueError(f"3D operators support dirichlet, neumann and impedance, not {bc_type!r}")
    mux, muy = co.mu_x, co.mu_y
    f = np.tile(np.arange(nx), ny)
    b = np.repeat(np.arange(ny), nx)
    N = nx * ny
    center = np.full(N, -2 * (mux + muy), dtype=complex)
    west = np.where(f > 0, mux, 0).astype(complex)
    east = np.where(f < nx - 1, mux, 0).astype(complex)
    south = np.where(b > 0, muy, 0).astype(complex)
    north = np.where(b < ny - 1, muy, 0).astype(complex)
    fe0, fe1 = f == 0, f == nx - 1
    be0, be1 = b == 0, b == ny - 1
    if bc_type == "dirichlet":
        # 1D Dirichlet rows of A_x: K rows f = 0, nx-1 lose the x part and the diagonal
        center[fe0 | fe1] = 0
        east[fe0] = 0
        west[fe1] = 0
        # 2D Dirichlet: first/last blocks become identity rows of A (K rows zero)
        for arr in (center, west, east, south, north):
            arr[be0 | be1] = 0
        return center, west, east, south, north
    east[fe0] *= 2
    west[fe1] *= 2
    if bc_type == "impedance":
        center[fe0 | fe1] += co.beta_x
    north[be0] *= 2
    south[be1] *= 2
    if bc_type == "impedance":
        center[be0 | be1] += co.beta_y
    return center, west, east, south, north


def transpose_diagonals(nx, center, west, east, south, north):
    """Diagonals of Kᵀ (the neighbour coefficients move to the neighbour's row)."""
    N = len(center)
    w2, e2, s2, n2 = (np.zeros(N, complex) for _ in range(4))
    w2[1:] = east[:-1]
    e2[:-1] = west[1:]
    s2[nx:] = north[:-nx]
    n2[:-nx] = south[nx:]
    return center.copy(), w2, e2, s2, n2
