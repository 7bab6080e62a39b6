"""complex128 restatement of the reference's paraxial (PWE) and multislice paths.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU legs, never by the product package.

Every function cites the reference file:line it restates (paths are relative
to the reference project root).  Parity of this restatement with the
unmodified reference is pinned by the golden fixtures in ``tests/golden``.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

BC_TYPES = ("dirichlet", "neumann", "impedance", "impedance2")


# ---------------------------------------------------------------------------
# Boundary-condition coefficients and step matrices
# ---------------------------------------------------------------------------
def bc_coefficients(k, dx, dz, dy=None, bc_type="impedance", dimension=2):
    """μ, β and γ coefficients.

    Restates ``thick_ptycho/forward_model/pwe/operators/finite_differences/
    boundary_conditions.py:9-55``: ``a = i/(2k)``, ``μ_x = a·dz/(2dx²)``,
    ``μ_y`` likewise in 3D (0 in 2D), ``β = μ·2ik·dx`` for the impedance
    variants and ``γ = −1/(2ik)`` for impedance2.
    """
    a = 1j / (2 * k)
    mu_x = a * (0.5 * dz / dx**2)
    mu_y = a * (0.5 * dz / dy**2) if dimension == 3 else 0.0
    out = {"mu_x": mu_x, "mu_y": mu_y, "beta_x": 0.0, "beta_y": 0.0, "gamma": 0.0}
    if bc_type in ("impedance", "impedance2"):
        out["beta_x"] = mu_x * 2j * k * dx
        out["beta_y"] = mu_y * 2j * k * dy if dimension == 3 else 0.0
    if bc_type == "impedance2":
        out["gamma"] = -1 / (2j * k)
    return out


def laplacian_1d(nx, mu_x, mu_y=0.0):
    """Scaled 1D second difference ``K = tridiag(μx, −2(μx+μy), μx)``.

    Restates ``operator_matrices.py:36-45``.
    """
    e = np.ones(nx, dtype=complex)
    return sp.diags(
        [mu_x * e[1:], -2 * (mu_x + mu_y) * e, mu_x * e[1:]],
        offsets=[-1, 0, 1],
        shape=(nx, nx),
        dtype=complex,
    ).tolil()


def apply_bc_1d(K, bc_type, co, dz):
    """Boundary-row edits of K.

    Restates ``operator_matrices.py:59-72`` and ``boundary_conditions.py:
    57-94``: Dirichlet zeroes rows 0 and N−1; otherwise the Neumann edit
    doubles ``K[0,1]`` and ``K[N−1,N−2]``, then impedance adds β to the two
    corner diagonals and impedance2 adds ``β + γ/dz²`` there and ``−γ/dz²`` to
    the doubled couplings.
    """
    K = K.tolil()
    if bc_type == "dirichlet":
        K[0, 1] = 0
        K[-1, -2] = 0
        K[0, 0] = 0
        K[-1, -1] = 0
        return K.tocsr()
    K[0, 1] *= 2
    K[-1, -2] *= 2
    if bc_type == "impedance":
        K[0, 0] += co["beta_x"]
        K[-1, -1] += co["beta_x"]
    elif bc_type == "impedance2":
        g = co["gamma"] / dz**2
        K[0, 0] += co["beta_x"] + g
        K[0, 1] += -g
        K[-1, -1] += co["beta_x"] + g
        K[-1, -2] += -g
    return K.tocsr()


def step_matrices_1d(nx, co, bc_type, dz):
    """``A = I − K``, ``B = I + K`` for 2D problems (1D transverse).

    Restates ``operator_matrices.py:47-57``.
    """
    K = apply_bc_1d(laplacian_1d(nx, co["mu_x"], co["mu_y"]), bc_type, co, dz)
    eye = sp.eye(nx, dtype=complex)
    return (eye - K).tocsr(), (eye + K).tocsr()


def step_matrices_2d(nx, ny, co, bc_type, dz):
    """5-point step matrices for 3D problems (2D transverse).

    Restates ``operator_matrices.py:75-126`` and ``boundary_conditions.py:
    96-130``: ``A = kron(I_y, A_x) + kron(offdiag_y, −μ_y I_x)`` (``+μ_y`` for
    B), then the y-edge rules (Dirichlet identity blocks, Neumann doubled
    couplings, impedance ``∓β_y I`` on the first and last blocks).
    """
    if bc_type not in ("dirichlet", "neumann", "impedance"):
        raise ValueError(f"3D step matrices do not support bc_type={bc_type!r}")
    Ax, Bx = step_matrices_1d(nx, co, bc_type, dz)
    Ix = sp.eye(nx, dtype=complex)
    Iy = sp.eye(ny, dtype=complex)
    off = sp.diags([1.0, 1.0], [-1, 1], shape=(ny, ny), dtype=complex)
    Axy = (sp.kron(Iy, Ax) + sp.kron(off, -co["mu_y"] * Ix)).tolil()
    Bxy = (sp.kron(Iy, Bx) + sp.kron(off, co["mu_y"] * Ix)).tolil()
    if bc_type == "dirichlet":
        Axy[:nx, :nx] = Ix
        Axy[-nx:, -nx:] = Ix
        Bxy[:nx, :nx] = Ix
        Bxy[-nx:, -nx:] = Ix
        Axy[:nx, nx : 2 * nx] *= 0
        Axy[-nx:, -2 * nx : -nx] *= 0
        Bxy[:nx, nx : 2 * nx] *= 0
        Bxy[-nx:, -2 * nx : -nx] *= 0
        return Axy.tocsr(), Bxy.tocsr()
    Axy[:nx, nx : 2 * nx] *= 2
    Axy[-nx:, -2 * nx : -nx] *= 2
    Bxy[:nx, nx : 2 * nx] *= 2
    Bxy[-nx:, -2 * nx : -nx] *= 2
    if bc_type == "impedance":
        Axy[:nx, :nx] -= co["beta_y"] * Ix
        Axy[-nx:, -nx:] -= co["beta_y"] * Ix
        Bxy[:nx, :nx] += co["beta_y"] * Ix
        Bxy[-nx:, -nx:] += co["beta_y"] * Ix
    return Axy.tocsr(), Bxy.tocsr()


def probe_bc_rhs_1d(nx, co, bc_type, probe=None):
    """Step RHS ``b`` (zero unless a probe is set for Dirichlet/impedance).

    Restates ``operator_matrices.py:152-166``.
    """
    ubc = np.zeros(nx, dtype=complex)
    if probe is None:
        return ubc
    if bc_type == "dirichlet":
        ubc[1] += 2 * co["mu_x"] * probe[0]
        ubc[-2] += 2 * co["mu_x"] * probe[-1]
    elif bc_type == "impedance":
        ubc[0] -= 2 * co["beta_x"] * probe[0]
        ubc[-1] -= 2 * co["beta_x"] * probe[-1]
    return ubc


# ---------------------------------------------------------------------------
# Object contribution C_j
# ---------------------------------------------------------------------------
def object_contribution(n, k, dz, grad=False, exact_ref_coeff=False, empty_space_px=0):
    """Per-step object coefficients ``C[..., j]`` (j = 0..Nz−2).

    Restates ``simulation/simulation_space/base_simulation_space.py:315-383``:
    ``coef = (k/i)(n−1)`` (or ``(k/2i)(n²−1)`` when ``exact_ref_coeff``; with
    ``grad`` the derivative forms ``k/i`` or ``(k/i)n``), optional zero padding
    of the first transverse axis, then ``(dz/2)·½(coef_j + coef_{j+1})``.
    """
    n = np.asarray(n)
    if grad:
        coef = (k / 1j) * (n if exact_ref_coeff else np.ones_like(n))
    else:
        coef = (k / 1j) * (n - 1) if not exact_ref_coeff else (k / 2j) * (n**2 - 1)
    if empty_space_px > 0:
        pad = [(empty_space_px, empty_space_px)] + [(0, 0)] * (coef.ndim - 1)
        coef = np.pad(coef, pad, mode="constant", constant_values=0.0)
    return (dz / 2) * (coef[..., :-1] + coef[..., 1:]) / 2


# ---------------------------------------------------------------------------
# Slice-by-slice LU march (the reference's IterativeLU path)
# ---------------------------------------------------------------------------
def build_lu_factors(A, B, C2d, mode="forward"):
    """Per-slice ``splu(A − C_j)`` and ``B + C_j`` for a mode.

    Restates ``forward_model/pwe/solvers/iterative_lu.py:90-133``: reverse
    swaps A and B (and negates b, done by the caller) and uses ``−C[:, −j]``;
    adjoint uses ``C[:, −j]`` and conjugate-transposes both matrices; forward
    uses ``C[:, j−1]``.
    """
    if mode == "reverse":
        A, B = B, A
    L = C2d.shape[1]
    lus, Bs = [], []
    for j in range(1, L + 1):
        if mode == "reverse":
            C = -sp.diags(C2d[:, -j])
        elif mode == "adjoint":
            C = sp.diags(C2d[:, -j])
        else:
            C = sp.diags(C2d[:, j - 1])
        Aw = A - C
        Bw = B + C
        if mode == "adjoint":
            Aw, Bw = Aw.conj().T, Bw.conj().T
        lus.append(spla.splu(Aw.tocsc()))
        Bs.append(Bw.tocsr())
    return lus, Bs


def march_with_lu(lus, Bs, b, probe, mode="forward", rhs_block=None, test_rhs=None):
    """One probe's z-march with prebuilt factors.

    Restates ``iterative_lu.py:138-197``: ``u[:,0] = probe``; per step
    ``u_j = LU_j⁻¹(B_j u_{j−1} + b)`` with ``b = rhs_block[:, −j]`` (adjoint)
    or ``rhs_block[:, j−1]``, overridden by the exact test boundary data when
    given; the adjoint result is flipped along z.
    """
    N = Bs[0].shape[0]
    L = len(lus)
    if mode == "reverse":
        b = -np.asarray(b)
    u = np.zeros((N, L + 1), dtype=complex)
    if probe is not None:
        u[:, 0] = np.asarray(probe).ravel()
    for j in range(1, L + 1):
        bj = b
        if rhs_block is not None:
            bj = rhs_block[:, -j] if mode == "adjoint" else rhs_block[:, j - 1]
        if test_rhs is not None:
            bj = test_rhs[j - 1]
        u[:, j] = lus[j - 1].solve(Bs[j - 1] @ u[:, j - 1] + bj)
    if mode == "adjoint":
        u = np.flip(u, axis=1)
    return u


def march(A, B, C2d, probe, mode="forward", b=None, rhs_block=None, test_rhs=None):
    """Convenience wrapper: factorise then march one probe."""
    lus, Bs = build_lu_factors(A, B, C2d, mode)
    if b is None:
        b = np.zeros(A.shape[0], dtype=complex)
    return march_with_lu(lus, Bs, b, probe, mode, rhs_block, test_rhs)


class NodePerturbation:
    """Exit waves of a probe stack when one index node is perturbed, for
    central finite differences at full depth.

    The forward march of ``march_with_lu`` (``iterative_lu.py:185-193``) is run
    once with every slice's factor and state kept.  Node t of n enters only the
    object terms C[:, t−1] and C[:, t] (``base_simulation_space.py:375-381``:
    C_j averages nodes j and j+1), i.e. slices t and t+1, so a perturbed exit
    refactorises those two slices and re-marches from the stored state u_{t−1};
    the arithmetic of every slice is that of the full march.
    """

    def __init__(self, A, B, n, k, dz, probes, exact_ref_coeff=False):
        self.A, self.B, self.k, self.dz = A, B, k, dz
        self.exact = exact_ref_coeff
        self.n = np.array(n, dtype=complex)
        self.C = object_contribution(self.n, k, dz, exact_ref_coeff=exact_ref_coeff)
        self.lus, self.Bs = build_lu_factors(A, B, self.C)
        L = self.C.shape[1]
        u = np.asarray(probes, dtype=complex).T.copy()  # (N, P)
        self.states = [u]
        for j in range(1, L + 1):
            u = self.lus[j - 1].solve(self.Bs[j - 1] @ u)
            self.states.append(u)

    def exits(self, x=None, t=None, delta=0.0):
        """(P, N) exit waves, with n[x, t] += delta when x is given."""
        L = self.C.shape[1]
        if x is None:
            return self.states[-1].T.copy()
        cols = {}
        for j in (t - 1, t):  # C columns that read node t
            if 0 <= j < L:
                seg = self.n[x, j:j + 2].copy()
                seg[t - j] += delta
                c = object_contribution(seg[None, :], self.k, self.dz, exact_ref_coeff=self.exact)[0, 0]
                cols[j] = c
        j0 = min(cols)  # first changed column: slice j0 + 1 (1-based)
        u = self.states[j0]
        for j in range(j0, L):
            if j in cols:
                Cj = self.C[:, j].copy()
                Cj[x] = cols[j]
                D = sp.diags(Cj)
                lu = spla.splu((self.A - D).tocsc())
                u = lu.solve((self.B + D) @ u)
            else:
                u = self.lus[j].solve(self.Bs[j] @ u)
        return u.T.copy()


def march_streamed(A, B, C2d, probes, keep=None):
    """Forward march of several probes, one slice factorised at a time.

    The same arithmetic as ``build_lu_factors(…, "forward")`` followed by
    ``march_with_lu`` (``iterative_lu.py:116-122,185-193``: ``u_j =
    splu(A − C_j)⁻¹ (B + C_j) u_{j−1}``, b = 0), but only the current slice's
    factor is held, so the 3D operators of large grids (one SuperLU of a
    65 536-unknown 5-point matrix is ~100 MB) fit in memory.  ``probes`` is
    (K, N).  Returns the exit waves (K, N) and, for the node indices in
    ``keep``, ``{t: u_t (K, N)}``.
    """
    probes = np.asarray(probes, dtype=complex)
    L = C2d.shape[1]
    u = probes.T.copy()
    kept = {}
    keep = set(keep or ())
    if 0 in keep:
        kept[0] = u.T.copy()
    for j in range(1, L + 1):
        C = sp.diags(C2d[:, j - 1])
        lu = spla.splu((A - C).tocsc())
        u = lu.solve((B + C) @ u)
        if j in keep:
            kept[j] = u.T.copy()
    return u.T.copy(), kept


# ---------------------------------------------------------------------------
# Space-time (parallel-in-time) solve: the reference's PWEFullPinTSolver
# ---------------------------------------------------------------------------
def pit_matvec(A, B, C2d, v):
    """Space-time operator ``M v``: slice j gets ``(A − C_j) v_j − (B + C_j) v_{j−1}``
    (vectors slice-major, ``v[j·N + i]``).  Restates ``_pint_utils.py:27-54``
    (forward mode), which pairs the subdiagonal of row j with ``C[:, j]``."""
    N, L = C2d.shape
    V = np.reshape(v, (N, L), order="F")
    U = (A @ V) - C2d * V
    U[:, 1:] -= B @ V[:, :-1] + C2d[:, 1:] * V[:, :-1]
    return np.reshape(U, (N * L,), order="F")


class PiTPreconditionerOracle:
    """α-block-circulant preconditioner of ``_pint_utils.py:57-205``.

    ``ω_j = α^{1/L} e^{2πij/L}``, ``γ_j = α^{j/L}`` (``setup``, :150-163);
    blocks ``splu(A − ω_j B)`` of the free-space A, B (``factorize_blocks``,
    :175-205; the solver never calls ``update``, so C does not enter); apply
    (forward, :91-104): scale by γ, ``ifft`` along z (ortho), block solves,
    ``fft`` along z (ortho), divide by γ.
    """

    def __init__(self, A, B, L, alpha):
        from scipy.fft import fft, ifft

        self._fft, self._ifft = fft, ifft
        self.N, self.L = A.shape[0], L
        self.omegas = np.exp(2j * np.pi * np.arange(L) / L) * alpha ** (1.0 / L)
        self.gamma = (alpha ** (np.arange(L) / L)).astype(np.complex128)
        A, B = A.tocsr(), B.tocsr()
        self.lus = [spla.splu((A - w * B).astype(np.complex128).tocsc()) for w in self.omegas]

    def apply(self, v):
        X = np.asarray(v, dtype=np.complex128).reshape(self.L, self.N)
        X = self.gamma[:, None] * X
        Xh = self._ifft(X, axis=0, norm="ortho")
        for j in range(self.L):
            Xh[j, :] = self.lus[j].solve(Xh[j, :])
        Y = self._fft(Xh, axis=0, norm="ortho")
        return (Y / self.gamma[:, None]).ravel()


def pit_rhs(B, probe, L, b_step=None):
    """Stacked right-hand side ``[B u_0 + b, 0, …, 0]`` of the full-system
    solvers (``forward_model.py:155-192``): the probe enters through B alone,
    without ``C_0 u_0`` (the reference's full-system form)."""
    N = B.shape[0]
    b0 = B @ np.asarray(probe, dtype=complex).ravel()
    if b_step is not None:
        b0 = b0 + b_step
    return np.concatenate([b0, np.zeros(N * (L - 1), dtype=complex)])


def full_system_solve(A, B, C2d, b):
    """Direct solve of the space-time system ``M u = b`` (slice-major b and u):
    ``M = kron(I, A) − kron(S, B) − diag(C) − subdiag(C)`` with S the
    subdiagonal shift, factorised once — ``PWEFullLUSolver``
    (``full_lu.py:72-172`` with ``forward_model.py:108-153,194-209``)."""
    N, L = C2d.shape
    S = sp.diags([np.ones(L - 1)], [-1], shape=(L, L), format="csr", dtype=complex)
    M = sp.kron(sp.eye(L, format="csr"), A) - sp.kron(S, B)
    cf = C2d.T.ravel()
    M = M - sp.diags(cf) - sp.diags([cf[N:]], [-N], shape=M.shape)
    return spla.spsolve(M.tocsc(), b)


def pit_solve(A, B, C2d, probes, alpha=1e-2, atol=1e-8, rtol=1e-5, restart=20, warm_start=True):
    """``PWEFullPinTSolver.solve`` for a probe stack: right-preconditioned GMRES
    on ``M R y = b``, ``u = R y`` (``full_pint.py:179-275``; scipy's ``gmres``
    with the reference's ``atol`` and its default ``rtol`` and ``restart``).
    With ``warm_start`` each probe starts from the previous probe's ``y``, as
    the reference's per-mode ``u0_cache`` does within one ``solve``.
    Returns ``u`` (P, N, L+1) with the probe as column 0, and the GMRES
    iteration counts."""
    N, L = C2d.shape
    R = PiTPreconditionerOracle(A, B, L, alpha)
    M = spla.LinearOperator((N * L, N * L), dtype=np.complex128,
                            matvec=lambda y: pit_matvec(A, B, C2d, R.apply(y)))
    out = np.zeros((len(probes), N, L + 1), dtype=complex)
    its = []
    y0 = None
    for p, probe in enumerate(probes):
        b = pit_rhs(B, probe, L)
        count = [0]

        def cb(_r):
            count[0] += 1

        y, info = spla.gmres(M, b, atol=atol, rtol=rtol, restart=restart, x0=y0, callback=cb,
                             callback_type="pr_norm")
        u = R.apply(y).reshape(L, N).T
        out[p, :, 0] = np.asarray(probe).ravel()
        out[p, :, 1:] = u
        its.append(count[0])
        if warm_start:
            y0 = y
    return out, its


def pit_solve_adjoint(A, B, C2d, probe=None, rhs=None, alpha=1e-2, atol=1e-8, rtol=1e-5, restart=20):
    """``PWEFullPinTSolver`` in mode "adjoint" for one probe (``full_pint.py:
    140-166`` with ``_pintobj_matvec_exact`` in its forward form,
    ``_pint_utils.py:27-54``): the system keeps the forward block structure —
    diagonal ``Aᴴ − C'_j``, subdiagonal ``−(Bᴴ + C'_j)`` of row j — with
    ``C' = conj(C)`` flipped along z, right-preconditioned by the *forward*
    α-circulant preconditioner of A, B (the solver builds one, in mode
    "forward").  The right-hand side is ``rhs`` (the flat column-major (N, L)
    vector, used as given) or ``[B u_0, 0, …]`` with the forward B.  Returns
    ``u`` (N, L+1) with the probe (or zeros) as column 0 — no flip along z —
    and the GMRES iteration count."""
    N, L = C2d.shape
    Ah, Bh = A.conj().T.tocsr(), B.conj().T.tocsr()
    Cf = np.flip(np.conj(C2d), axis=1)
    R = PiTPreconditionerOracle(A, B, L, alpha)
    M = spla.LinearOperator((N * L, N * L), dtype=np.complex128,
                            matvec=lambda y: pit_matvec(Ah, Bh, Cf, R.apply(y)))
    p0 = np.zeros(N, dtype=complex) if probe is None else np.asarray(probe, dtype=complex).ravel()
    b = np.asarray(rhs, dtype=complex).ravel() if rhs is not None else pit_rhs(B, p0, L)
    count = [0]

    def cb(_r):
        count[0] += 1

    y, info = spla.gmres(M, b, atol=atol, rtol=rtol, restart=restart, callback=cb, callback_type="pr_norm")
    u = np.zeros((N, L + 1), dtype=complex)
    u[:, 0] = p0
    u[:, 1:] = R.apply(y).reshape(L, N).T
    return u, count[0]


# ---------------------------------------------------------------------------
# Exact discrete adjoint and gradient (no reference counterpart; the
# reference's adjoint differs, see ``reference_grad_least_squares``)
# ---------------------------------------------------------------------------
def exact_adjoint(A, B, C2d, src):
    """λ_j solving ``(A − C_j)ᴴ λ_j = src_j + (B + C_{j+1})ᴴ λ_{j+1}``.

    ``src`` has shape (N, L); column j−1 is the source of slice j.  This is
    the exact adjoint of the forward march of ``march`` (mode "forward").
    Returns λ with shape (N, L), column j−1 holding slice j.
    """
    N, L = C2d.shape
    lam = np.zeros((N, L), dtype=complex)
    nxt = np.zeros(N, dtype=complex)
    for j in range(L, 0, -1):
        rhs = src[:, j - 1].copy()
        if j < L:
            Rn = (B + sp.diags(C2d[:, j])).conj().T
            rhs = rhs + Rn @ nxt
        Mj = (A - sp.diags(C2d[:, j - 1])).conj().T.tocsc()
        lam[:, j - 1] = spla.spsolve(Mj, rhs)
        nxt = lam[:, j - 1]
    return lam


def exact_adjoint_many(A, B, C2d, srcs):
    """``exact_adjoint`` for several sources sharing one factorisation per slice.

    ``srcs`` has shape (K, N, L); returns λ of the same shape.
    """
    K, N, L = srcs.shape
    lam = np.zeros_like(srcs, dtype=complex)
    nxt = np.zeros((N, K), dtype=complex)
    for j in range(L, 0, -1):
        rhs = srcs[:, :, j - 1].T.copy()
        if j < L:
            Rn = (B + sp.diags(C2d[:, j])).conj().T
            rhs = rhs + Rn @ nxt
        lu = spla.splu((A - sp.diags(C2d[:, j - 1])).conj().T.tocsc())
        nxt = lu.solve(rhs)
        lam[:, :, j - 1] = nxt.T
    return lam


def grad_c_from_adjoint(u, lam):
    """Torch-convention gradient w.r.t. each step coefficient c_j.

    ``u`` is (N, Nz), ``lam`` is (N, L).  ``∂ℓ/∂Re c + i∂ℓ/∂Im c =
    λ_j · conj(u_j + u_{j−1})``.
    """
    return lam * np.conj(u[:, 1:] + u[:, :-1])


def chain_grad_to_n(grad_c, k, dz, n=None, exact_ref_coeff=False, empty_space_px=0):
    """Map gradients w.r.t. c_j onto the z nodes of n (torch convention).

    ``c_j = (dz/4)(coef(n_{j−1}) + coef(n_j))`` so node t receives
    ``conj((dz/4)·coef'(n_t))·(g_t + g_{t+1})`` with out-of-range terms zero.
    """
    if empty_space_px > 0:
        grad_c = grad_c[empty_space_px:-empty_space_px]
    N, L = grad_c.shape
    acc = np.zeros((N, L + 1), dtype=complex)
    acc[:, :-1] += grad_c
    acc[:, 1:] += grad_c
    if exact_ref_coeff:
        dcoef = (k / 1j) * np.asarray(n)
    else:
        dcoef = (k / 1j) * np.ones((N, L + 1))
    return np.conj((dz / 4) * dcoef) * acc


# ---------------------------------------------------------------------------
# Exit waves, far field, phase-retrieval projection, amplitude loss
# ---------------------------------------------------------------------------
def farfield_intensity(exit_waves, dimension=2):
    """``|FFT(exit)|²`` without noise.

    Restates ``forward_model/base/base_solver.py:213-249``: 2D, the FFT of each
    exit wave; 3D, ``fft2`` over the last two axes of the (total_scans,
    block_size) exit-wave array — the reference transforms across the scan
    index and the flattened pixels, and this restates it as it is.
    """
    if dimension == 2:
        return np.abs(np.fft.fft(exit_waves, axis=-1)) ** 2
    return np.abs(np.fft.fft2(exit_waves, axes=(-2, -1))) ** 2


def phase_retrieval_projection(exit_waves, data):
    """Gerchberg–Saxton modulus projection.

    Restates ``reconstruction/base_reconstructor.py:171-207``.
    """
    f = np.fft.fft(exit_waves, axis=-1)
    mag = np.abs(f)
    mag[mag == 0] = 1.0
    return np.fft.ifft(np.sqrt(data) * (f / mag), axis=-1)


def amplitude_loss_and_grad(exit_waves, amplitude):
    """``ℓ = Σ(|F e| − a)²`` and its torch-convention gradient w.r.t. e."""
    N = exit_waves.shape[-1]
    U = np.fft.fft(exit_waves, axis=-1)
    mag = np.abs(U)
    loss = float(np.sum((mag - amplitude) ** 2))
    safe = np.where(mag > 0, mag, 1.0)
    gU = 2 * (mag - amplitude) * U / safe
    gU = np.where(mag > 0, gU, 0)
    return loss, N * np.fft.ifft(gU, axis=-1)


# ---------------------------------------------------------------------------
# Reference-compatible least-squares gradient (reproduces its B1/B2/B3)
# ---------------------------------------------------------------------------
def reference_grad_least_squares(A, B, C2d, u_all, exit_err, k, dz):
    """The reference's ``compute_grad_least_squares`` for one projection.

    Restates ``reconstruction/pwe_reconstructor.py:100-164`` (no reduced
    domain): per probe an adjoint march (mode "adjoint", source = exit error
    at the last slice), ``g = grad_A @ u`` with ``grad_A = −(diag(G) +
    subdiag(G))`` and ``G = (dz/2)(k/i)`` (``forward_model.py:128-153``),
    then ``grad_re −= Re(conj(g)λ)``, ``grad_im −= Re(conj(ig)λ)``.
    ``u_all`` is (P, N, Nz), ``exit_err`` (P, N); returns two (L·N,) arrays
    laid out z-major like the reference.
    """
    P, N, Nz = u_all.shape
    L = Nz - 1
    lus, Bs = build_lu_factors(A, B, C2d, "adjoint")
    G = (dz / 2) * (k / 1j)
    gre = np.zeros(L * N)
    gim = np.zeros(L * N)
    zero_b = np.zeros(N, dtype=complex)
    for p in range(P):
        rhs_block = np.zeros((N, L), dtype=complex)
        rhs_block[:, -1] = exit_err[p]
        bp = march_with_lu(lus, Bs, zero_b, None, "adjoint", rhs_block)
        bp = bp[:, :-1].T.ravel()
        uk = u_all[p][:, 1:].T  # (L, N)
        g = -G * uk.copy()
        g[1:] += -G * uk[:-1]
        g = g.ravel()
        gre -= (g.conj() * bp).real
        gim -= ((1j * g).conj() * bp).real
    return gre, gim


def reference_alphak(A, B, C2d, u_all, probes, grad_E, d, k, dz, imaginary=False):
    """The reference's ``compute_alphak`` (``pwe_reconstructor.py:166-219``).

    Per probe: the source ``grad_A @ u`` (times i for the imaginary part),
    a forward solve that starts from the probe itself, and
    ``δp = −δu_L · d_L`` (plain dot product over the last slice); the step is
    ``−vdot(d, grad_E) / Σ_p |δp|²``.
    """
    P, N, Nz = u_all.shape
    L = Nz - 1
    G = (dz / 2) * (k / 1j)
    lus, Bs = build_lu_factors(A, B, C2d, "forward")
    den = 0.0
    for p in range(P):
        uk = u_all[p][:, 1:].T  # (L, N): vector-form blocks
        g = -G * uk.copy()
        g[1:] += -G * uk[:-1]
        if imaginary:
            g = 1j * g
        du = march_with_lu(lus, Bs, np.zeros(N, dtype=complex), probes[p], "forward", g.T)
        dp = -(du[:, -1] @ d[-N:])
        den += abs(dp) ** 2
    num = np.vdot(d, grad_E)
    return -(num / den) if den > 0 else 0.0


def reference_betak(g, g_old):
    """``compute_betak`` (``pwe_reconstructor.py:221-228``): min(FR, max(PR, 0))."""
    nrm = np.vdot(g_old, g_old)
    pr = np.vdot(g, g - g_old) / nrm
    fr = np.vdot(g, g) / nrm
    return min(fr, max(pr, 0))


def reference_nlcg(A, B, n0, probes, data, k, dz, iters, phase_retrieval=True):
    """``ReconstructorPWE.reconstruct`` (``pwe_reconstructor.py:229-368``) for one
    projection and angle, computed step sizes, no regularisation, constant
    gradient operator (``exact_ref_coeff`` off).  Returns (n, residuals)."""
    nk = np.array(n0, dtype=complex)
    N, Nz = nk.shape
    L = Nz - 1
    P = probes.shape[0]
    residual = []
    d_re = d_im = g_re_old = g_im_old = None
    for i in range(iters):
        C = object_contribution(nk, k, dz)
        lus, Bs = build_lu_factors(A, B, C, "forward")
        u = np.stack([march_with_lu(lus, Bs, np.zeros(N, dtype=complex), probes[p], "forward") for p in range(P)])
        ex = u[:, :, -1]
        err = ex - (phase_retrieval_projection(ex, data) if phase_retrieval else data)
        residual.append(float(np.sqrt(np.mean(np.abs(err) ** 2))))
        g_re, g_im = reference_grad_least_squares(A, B, C, u, err, k, dz)
        if i == 0:
            d_re, g_re_old = -g_re, g_re
            d_im, g_im_old = -g_im, g_im
        a_re = reference_alphak(A, B, C, u, probes, g_re, d_re, k, dz)
        a_im = reference_alphak(A, B, C, u, probes, g_im, d_im, k, dz, imaginary=True)
        nk[:, 1:] += (a_re * d_re).reshape(L, N).T + 1j * (a_im * d_im).reshape(L, N).T
        b_re = reference_betak(g_re, g_re_old)
        b_im = reference_betak(g_im, g_im_old)
        d_re, g_re_old = -g_re + b_re * d_re, g_re
        d_im, g_im_old = -g_im + b_im * d_im, g_im
    return nk, residual


# ---------------------------------------------------------------------------
# Multislice (angular spectrum), 2D
# ---------------------------------------------------------------------------
def ms_kernel(nx_eff, dx, k, dz, remove_global_phase=True):
    """Angular-spectrum kernel ``H = exp(i k_z dz)·exp(−ik dz)``.

    Restates ``forward_model/multislice/ms_solver.py:49-72``.
    """
    kx = 2 * np.pi * np.fft.fftfreq(nx_eff, d=dx)
    kz = np.sqrt(np.clip(k**2 - kx**2, 0.0, None))
    H = np.exp(1j * kz * dz)
    if remove_global_phase:
        H = H * np.exp(-1j * k * dz)
    return H.astype(np.complex128)


def ms_forward(n, probe, k, dx, dz, n_medium=1.0):
    """Multislice march of one probe, shape (N, Nz).

    Restates ``ms_solver.py:74-78,86-88,90-159``: transmit by
    ``exp(ik(n_z − n_med)dz)`` then propagate with H (global phase removed).
    """
    N, Nz = n.shape
    H = ms_kernel(N, dx, k, dz)
    u = np.empty((N, Nz), dtype=complex)
    psi = np.asarray(probe, dtype=complex).copy()
    u[:, 0] = psi
    for z in range(Nz - 1):
        psi = psi * np.exp(1j * k * (n[:, z] - n_medium) * dz)
        psi = np.fft.ifft(np.fft.fft(psi) * H)
        u[:, z + 1] = psi
    return u


def ms_kernel_3d(n1, n2, d1, d2, k, dz):
    """3D angular-spectrum kernel: ``ms_kernel`` with kx² replaced by
    k1² + k2² over the (n1, n2) grid (``ms_solver.py:49-72`` made 2D in the
    transverse plane; the reference itself has no 3D multislice)."""
    k1 = 2 * np.pi * np.fft.fftfreq(n1, d=d1)[:, None]
    k2 = 2 * np.pi * np.fft.fftfreq(n2, d=d2)[None, :]
    kz = np.sqrt(np.clip(k**2 - k1**2 - k2**2, 0.0, None))
    return np.exp(1j * kz * dz) * np.exp(-1j * k * dz)


def ms_forward_3d(n, probe, k, d1, d2, dz, n_medium=1.0):
    """3D multislice march of one probe: n (n1, n2, Nz), probe (n1, n2) →
    u (n1, n2, Nz).  Same steps as :func:`ms_forward` with ``fft2``."""
    n1, n2, Nz = n.shape
    H = ms_kernel_3d(n1, n2, d1, d2, k, dz)
    u = np.empty((n1, n2, Nz), dtype=complex)
    psi = np.asarray(probe, dtype=complex).copy()
    u[:, :, 0] = psi
    for z in range(Nz - 1):
        psi = psi * np.exp(1j * k * (n[:, :, z] - n_medium) * dz)
        psi = np.fft.ifft2(np.fft.fft2(psi) * H)
        u[:, :, z + 1] = psi
    return u


def ms_3pie(probes, data, k, dx, dz, nz, iters, alpha_obj=1.0, n_medium=1.0, phase_retrieval=True):
    """Multislice 3PIE reconstruction (``reconstruction/ms_reconstructor.py:40-190``).

    Epochs over the probes in scan order; per probe: multislice forward from
    the current estimate, modulus constraint on the exit wave
    (``phase = F ψ / (|F ψ| + 1e-12)``), then from the detector plane back to
    the entrance, for every slice z (last to first): ``ψ ← F⁻¹(conj(H) F ψ)``,
    ``ψ ← ψ · conj(T_z)``, ``δψ = ψ − u_z`` and
    ``n_z += (α/(it+1)) conj(u_z) δψ / (max|u_z|² + 1e-12) / (i k dz)``
    (the estimate changes in place, probe after probe).  Returns (n, loss
    per epoch) with loss = rms of (corrected − modelled) exit waves.
    """
    P, N = probes.shape
    n_est = n_medium * np.ones((N, nz), dtype=complex)
    H = ms_kernel(N, dx, k, dz)
    loss = []
    for it in range(iters):
        err = np.zeros((P, N), dtype=complex)
        for p in range(P):
            u = ms_forward(n_est, probes[p], k, dx, dz, n_medium)
            ex = u[:, -1]
            if phase_retrieval:
                f = np.fft.fft(ex)
                corr = np.fft.ifft(np.sqrt(data[p]) * (f / (np.abs(f) + 1e-12)))
            else:
                corr = data[p]
            err[p] = corr - ex
            psi = corr
            step = alpha_obj / (it + 1)
            for z in reversed(range(nz)):
                psi = np.fft.ifft(np.fft.fft(psi) * np.conj(H))
                psi = psi * np.conj(np.exp(1j * k * (n_est[:, z] - n_medium) * dz))
                dpsi = psi - u[:, z]
                scale = np.max(np.abs(u[:, z]) ** 2) + 1e-12
                n_est[:, z] = n_est[:, z] + step * (np.conj(u[:, z]) * dpsi / scale) / (1j * k * dz)
        loss.append(float(np.sqrt(np.mean(np.abs(err) ** 2))))
    return n_est, loss


# ---------------------------------------------------------------------------
# Exact impedance test boundary data (the reference's known-answer tests)
# ---------------------------------------------------------------------------
def exact_impedance_test_rhs(x, z, k, beta_x, y=None, beta_y=0.0):
    """Per-step test boundary data, shape (L, N).

    Restates ``boundary_condition_test.py:49-114``: the analytic Neumann mode
    sum evaluated on the boundary, ``−2β·u_exact`` on the edge rows, averaged
    between z_{j−1} and z_j.
    """
    a = 1j / (2 * k)

    def u_nm(n, m, xx, yy, zz):
        return np.exp(-a * ((n**2 + m**2) * np.pi**2) * zz) * np.cos(n * np.pi * xx) * np.cos(m * np.pi * yy)

    def bnd(zz):
        if y is None:
            ue = lambda xx: u_nm(1, 0, xx, 0, zz) + 0.5 * u_nm(2, 0, xx, 0, zz) + 0.2 * u_nm(5, 0, xx, 0, zz)  # noqa: E731
            ubc = np.zeros(len(x), dtype=complex)
            ubc[0] -= 2 * beta_x * ue(x[0])
            ubc[-1] -= 2 * beta_x * ue(x[-1])
            return ubc
        ue = lambda xx, yy: u_nm(1, 1, xx, yy, zz) + 0.5 * u_nm(2, 2, xx, yy, zz) + 0.2 * u_nm(5, 5, xx, yy, zz)  # noqa: E731
        ubc = np.zeros((len(x), len(y)), dtype=complex)
        ubc[0, :] -= 2 * beta_x * ue(x[0], y)
        ubc[-1, :] -= 2 * beta_x * ue(x[-1], y)
        ubc[:, 0] -= 2 * beta_y * ue(x, y[0])
        ubc[:, -1] -= 2 * beta_y * ue(x, y[-1])
        return ubc.ravel()

    return np.stack([0.5 * (bnd(z[j - 1]) + bnd(z[j])) for j in range(1, len(z))])
