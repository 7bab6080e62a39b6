"""Host-side 3D operator diagonals against the oracle's sparse matrices."""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import pwe_oracle as po
from thick_ptycho_b200.operators import BCCoefficients, operator_2d_diagonals, transpose_diagonals


def _sparse(nx, diags):
    c, w, e, s, n = diags
    N = len(c)
    return sp.diags([c, w[1:], e[:-1], s[nx:], n[:-nx]], [0, -1, 1, -nx, nx], shape=(N, N)).toarray()


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet"])
@pytest.mark.parametrize("nx", [5, 8])
def test_diagonals_match_oracle(bc, nx):
    k, dx, dz = 4 * np.pi, 0.9, 1.1
    co = BCCoefficients.make(k, dx, dz, bc, dy=dx, dimension=3)
    d = operator_2d_diagonals(nx, nx, co, bc)
    A, B = po.step_matrices_2d(nx, nx, po.bc_coefficients(k, dx, dz, dy=dx, bc_type=bc, dimension=3), bc, dz)
    K = np.eye(nx * nx) - A.toarray()
    assert np.allclose(_sparse(nx, d), K, rtol=0, atol=1e-15)
    assert np.allclose(np.eye(nx * nx) + _sparse(nx, d), B.toarray(), rtol=0, atol=1e-15)
    assert np.allclose(_sparse(nx, transpose_diagonals(nx, *d)), K.T, rtol=0, atol=1e-15)
