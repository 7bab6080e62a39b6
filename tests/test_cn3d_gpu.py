"""Batched 3D (5-point, BiCGStab) march against the reference's golden
vectors and the complex128 oracle (sparse LU per slice).

Tolerances: fields ≤ 1e-5 relative L2 against complex128 (BiCGStab at its
default stopping residual, complex64 vectors, FP64 dot products); exact-adjoint
gradients ≤ 1e-5 relative L2 against the oracle's discrete adjoint.
"""

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200 import SimulationGeometry  # noqa: E402
from thick_ptycho_b200.cn3d import CN3D  # noqa: E402
from thick_ptycho_b200.solver import PWEGpuSolver  # noqa: E402

TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def c64(x):
    return torch.from_numpy(np.ascontiguousarray(x).astype(np.complex64)).cuda()


def run(eng, n, P, mode="forward", **kw):
    store = eng.new_store(P)
    eng.march(torch.from_numpy(np.ascontiguousarray(n.reshape(eng.N, eng.nz))).cuda(), P, mode, u_store=store,
              tol=kw.pop("tol", 1e-6), **kw)
    return store.permute(0, 2, 1).cpu().numpy().astype(np.complex128)  # (P, N, nz)


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet"])
@pytest.mark.parametrize("nx", [8, 16])
def test_kat3d_golden(golden, bc, nx):
    g = golden("kat3d")
    key = f"{bc}_{nx}"
    N, nz, dz, dx, dy, k = (int(g[key + "_nx"]), int(g[key + "_nz"]), float(g[key + "_dz"]), float(g[key + "_dx"]),
                            float(g[key + "_dy"]), float(g[key + "_k"]))
    eng = CN3D(N, N, nz, k, dx, dy, dz, bc)
    n = np.ones((N * N, nz), dtype=complex)
    kw = {}
    if key + "_test_rhs" in g:
        kw["src_shared"] = c64(g[key + "_test_rhs"])
    u = run(eng, n, 1, probes=c64(g[key + "_probe"].reshape(1, -1)), **kw)[0]
    assert rel(u.reshape(N, N, nz), g[key + "_u"]) < TOL
    st = eng.read_stats()
    assert st["failed"] == 0 and st["solves"] == nz - 1


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet"])
def test_random3d_golden(golden, bc):
    g = golden("random3d")
    N, nz, dz, dx, dy, k = (int(g["nx"]), int(g["nz"]), float(g["dz"]), float(g["dx"]), float(g["dy"]), float(g["k"]))
    eng = CN3D(N, N, nz, k, dx, dy, dz, bc)
    P = g["probes"].shape[0]
    u = run(eng, g["n"], P, probes=c64(g["probes"].reshape(P, -1)))
    for p in range(P):
        assert rel(u[p].reshape(N, N, nz), g[f"{bc}_forward"][p]) < TOL, p
    # the reference adjoint reads rhs_block column -j at step j and flips its output
    src = c64(g["rhs_block"][:, ::-1].T)
    lam = run(eng, g["n"], 1, "adjoint", src_shared=src)[0]
    assert rel(lam, g[f"{bc}_adjoint"]) < TOL


def _field(rng, N, nz, scale=5e-3):
    return 1 + scale * (rng.standard_normal((N, nz)) + 0.2j * rng.standard_normal((N, nz)))


def _gauss(nf, nb, centres, w):
    f = np.arange(nf)[None, :]
    b = np.arange(nb)[:, None]
    return np.array([np.exp(-((f - cf) ** 2 + (b - cb) ** 2) / w**2).ravel() for cf, cb in centres]).astype(complex)


@pytest.mark.parametrize("bc", ["impedance", "neumann", "dirichlet"])
@pytest.mark.parametrize("precond", [True, False])
def test_fft_preconditioned_against_oracle(bc, precond):
    """64×64 transverse (FFT preconditioner active), 12 nodes, 6 probes."""
    rng = np.random.default_rng(11)
    nf = nb = 64
    nz, k, dx, dz, P = 12, 2 * np.pi / 0.5, 1.0, 1.0, 6
    n = _field(rng, nf * nb, nz)
    probes = _gauss(nf, nb, rng.uniform(20, 44, (P, 2)), 8.0)
    eng = CN3D(nf, nb, nz, k, dx, dx, dz, bc)
    u = run(eng, n, P, probes=c64(probes), precond=precond)
    st = eng.read_stats()
    assert st["failed"] == 0
    co = po.bc_coefficients(k, dx, dz, dy=dx, bc_type=bc, dimension=3)
    A, B = po.step_matrices_2d(nf, nb, co, bc, dz)
    C = po.object_contribution(n, k, dz)
    for p in (0, 3, 5):
        ref = po.march(A, B, C, probes[p])
        assert rel(u[p], ref) < TOL, (p, rel(u[p], ref))


@pytest.mark.parametrize("bc,dz", [("neumann", 1.0), ("impedance", 0.5)])
def test_reverse_mode_against_oracle(bc, dz):
    """Reverse (σ = −1) march.  With impedance edges the reversed corner
    diagonal is 1 + Kc = 1 − dz/dx + O(μ): at dz = dx it is ≈ −0.08i, the
    corner amplification per step is |1 − Kc|/|1 + Kc| ≈ 25, and complex64
    round-off grows like 25^L (the complex128 march is no reference there);
    dz = dx/2 keeps the amplification at ≈ 3.  The amplification also acts
    on each step's Krylov residual: at the default 1e-6 the impedance case
    reaches 2.3e-5 after 8 steps, at 1e-7 it stays near 2e-6."""
    rng = np.random.default_rng(3)
    nf = nb = 32
    nz, k, P = 9, 4 * np.pi, 3
    n = _field(rng, nf * nb, nz)
    probes = _gauss(nf, nb, rng.uniform(10, 22, (P, 2)), 5.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, dz, bc)
    u = run(eng, n, P, "reverse", probes=c64(probes), tol=1e-7, max_iter=40)
    co = po.bc_coefficients(k, 1.0, dz, dy=1.0, bc_type=bc, dimension=3)
    A, B = po.step_matrices_2d(nf, nb, co, bc, dz)
    C = po.object_contribution(n, k, dz)
    for p in range(P):
        assert rel(u[p], po.march(A, B, C, probes[p], "reverse")) < TOL


@pytest.mark.parametrize("exact", [False, True])
def test_exact_adjoint_gradient_against_oracle(exact):
    rng = np.random.default_rng(21)
    nf = nb = 32
    nz, k, dz, P = 10, 4 * np.pi, 1.0, 4
    N = nf * nb
    n = _field(rng, N, nz)
    probes = _gauss(nf, nb, rng.uniform(10, 22, (P, 2)), 5.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, dz, "impedance", exact_ref_coeff=exact)
    field = torch.from_numpy(n).cuda()
    store = eng.new_store(P)
    eng.march(field, P, "forward", probes=c64(probes), u_store=store, tol=1e-7)
    srcs = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    gc = torch.zeros((nz - 1, N), dtype=torch.complex64, device="cuda")
    eng.march(field, P, "adjoint_exact", src_exit=c64(srcs), u_fwd=store, grad_c=gc, tol=1e-7)
    gn = eng.grad_to_n(gc, field).cpu().numpy()

    co = po.bc_coefficients(k, 1.0, dz, dy=1.0, bc_type="impedance", dimension=3)
    A, B = po.step_matrices_2d(nf, nb, co, "impedance", dz)
    C = po.object_contribution(n, k, dz, exact_ref_coeff=exact)
    u = np.array([po.march(A, B, C, probes[p]) for p in range(P)])
    src = np.zeros((P, N, nz - 1), dtype=complex)
    src[:, :, -1] = srcs
    lam = po.exact_adjoint_many(A, B, C, src)
    gcr = sum(po.grad_c_from_adjoint(u[p], lam[p]) for p in range(P))
    assert rel(gc.cpu().numpy().T, gcr) < TOL
    gnr = po.chain_grad_to_n(gcr, k, dz, n=n, exact_ref_coeff=exact)
    assert rel(gn, gnr) < TOL


def test_src_shared_and_src_exit_adjoint():
    """ADJOINT_EXACT with a shared per-step source and an exit source together."""
    rng = np.random.default_rng(8)
    nf = nb = 16
    nz, k, P = 7, 4 * np.pi, 2
    N = nf * nb
    n = _field(rng, N, nz)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, "neumann")
    sh = rng.standard_normal((nz - 1, N)) + 1j * rng.standard_normal((nz - 1, N))
    ex = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    store = eng.new_store(P)
    # shared source rows are in step order: step t solves slice L+1-t
    eng.march(torch.from_numpy(n).cuda(), P, "adjoint_exact", src_exit=c64(ex), src_shared=c64(sh[::-1]),
              u_store=store, tol=1e-7)
    lam = store.permute(0, 2, 1).cpu().numpy()
    co = po.bc_coefficients(k, 1.0, 1.0, dy=1.0, bc_type="neumann", dimension=3)
    A, B = po.step_matrices_2d(nf, nb, co, "neumann", 1.0)
    C = po.object_contribution(n, k, 1.0)
    src = np.repeat(sh.T[None], P, axis=0).astype(complex)
    src[:, :, -1] += ex
    ref = po.exact_adjoint_many(A, B, C, src)
    for p in range(P):
        # node t holds step t, i.e. slice L+1-t (node 0 holds the zero start state)
        assert rel(lam[p][:, 1:][:, ::-1], ref[p]) < TOL


def test_dropin_solver_3d():
    geo = SimulationGeometry.grid_3d(24, 10, 0.5, 2, 8)
    rng = np.random.default_rng(2)
    n = 1 + 2e-3 * (rng.standard_normal(geo.effective_shape) + 0.1j * rng.standard_normal(geo.effective_shape))
    N = geo.block_size
    centres = [(8 + 8 * (p // 2), 8 + 8 * (p % 2)) for p in range(geo.num_probes)]
    probes = _gauss(geo.effective_shape[0], geo.effective_shape[1], centres, 4.0).reshape(
        1, geo.num_probes, *geo.effective_shape[:2])
    s = PWEGpuSolver(geo, probes, bc_type="impedance")
    u = s.solve(n=n)
    assert u.shape == (1, 1, geo.num_probes, *geo.effective_shape)
    nf = geo.effective_shape[0]
    co = po.bc_coefficients(geo.k, geo.dx, geo.dz, dy=geo.dy, bc_type="impedance", dimension=3)
    A, B = po.step_matrices_2d(nf, nf, co, "impedance", geo.dz)
    C = po.object_contribution(n, geo.k, geo.dz).reshape(N, -1)
    for p in range(geo.num_probes):
        ref = po.march(A, B, C, probes[0, p].ravel())
        assert rel(u[0, 0, p].reshape(N, -1), ref) < TOL
    rhs = rng.standard_normal((N, geo.nz - 1)) + 1j * rng.standard_normal((N, geo.nz - 1))
    lam = s._solve_single_probe(n=n, mode="adjoint", rhs_block=rhs)
    assert rel(lam, po.march(A, B, C, None, "adjoint", rhs_block=rhs)) < TOL


def test_rejects_bad_arguments():
    eng = CN3D(8, 8, 4, 4 * np.pi, 1.0, 1.0, 1.0, "impedance")
    f = torch.ones((64, 4), dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError):
        eng.march(f, 2, probes=torch.zeros((2, 63), dtype=torch.complex64, device="cuda"))
    with pytest.raises(Exception, match="gradient"):
        eng.march(f, 1, "forward", u_fwd=eng.new_store(1),
                  grad_c=torch.zeros((3, 64), dtype=torch.complex64, device="cuda"))


@pytest.mark.parametrize("mode", ["forward", "adjoint_exact", "adjoint", "reverse"])
def test_graph_march_matches_step_by_step(mode):
    """The march recorded as one CUDA graph (conditional WHILE nodes for the
    step and BiCGStab loops, no host round trip) against the same kernels
    launched step by step with a host check per iteration: the same iteration
    counts (up to a convergence decision that round-off may tip), fields equal
    to fp32 round-off (the fp64 dot products are summed with atomics in
    varying order), and the gradient likewise."""
    rng = np.random.default_rng(31)
    nf = nb = 32
    nz, k, P = 12, 4 * np.pi, 3
    N = nf * nb
    n = _field(rng, N, nz)
    field = torch.from_numpy(n).cuda()
    dz = 0.5 if mode == "reverse" else 1.0
    probes = c64(_gauss(nf, nb, rng.uniform(10, 22, (P, 2)), 5.0))
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, dz, "impedance")
    fwd = eng.new_store(P)
    eng.march(field, P, "forward", probes=probes, u_store=fwd, tol=1e-7)
    src = c64(rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N)))
    out = {}
    for launch in (0, 1):
        eng.launch = launch
        eng.read_stats()
        store = eng.new_store(P)
        gc = torch.zeros((nz - 1, N), dtype=torch.complex64, device="cuda")
        if mode == "adjoint_exact":
            eng.march(field, P, mode, src_exit=src, u_fwd=fwd, grad_c=gc, u_store=store, tol=1e-7)
        elif mode == "adjoint":
            eng.march(field, P, mode, src_exit=src, u_store=store, tol=1e-7)
        else:
            eng.march(field, P, mode, probes=probes, u_store=store, tol=1e-7)
        st = eng.read_stats()
        assert st["graph"] == (launch == 0), st
        out[launch] = (store.cpu().numpy(), gc.cpu().numpy(), st)
    eng.launch = 0
    assert abs(out[0][2]["iterations"] - out[1][2]["iterations"]) <= 2
    assert out[0][2]["solves"] == out[1][2]["solves"] == P * (nz - 1)
    assert rel(out[0][0], out[1][0]) < 1e-6
    if mode == "adjoint_exact":
        assert rel(out[0][1], out[1][1]) < 1e-6


def _apply_i_minus_p(eng, x, diag):
    """(I - P_s) x in complex128 from the engine's forward diagonals plus the
    slice's object diagonal (vector index b * nf + f)."""
    kc, kw, ke, ks, kn = (d.cpu().numpy().astype(np.complex128) for d in eng._diags)
    nf, N = eng.nx, eng.N
    f = np.arange(N) % nf
    px = (kc + diag) * x
    px[f > 0] += kw[f > 0] * x[np.arange(N)[f > 0] - 1]
    px[f < nf - 1] += ke[f < nf - 1] * x[np.arange(N)[f < nf - 1] + 1]
    px[nf:] += ks[nf:] * x[:-nf]
    px[:-nf] += kn[:-nf] * x[nf:]
    return x - px


@pytest.mark.parametrize("nf,nb", [(64, 64), (128, 128), (192, 192), (256, 256), (96, 96), (64, 128)])
def test_fft_preconditioner_against_numpy(nf, nb):
    """The plain preconditioner M0^{-1} v = IFFT2(FFT2(v) / lambda) through the
    white-noise training pairs (x noise, v = (I - P_s) x, z0 = M0^{-1} v),
    against numpy's complex128 FFT: the register four-step kernels (square 64,
    128, 192, 256) and the shared-memory Stockham kernels (96 x 96 and 64 x 128,
    and forced at the four-step sizes) give the same operator."""
    from thick_ptycho_b200.cn3d import generate_pairs

    rng = np.random.default_rng(nf + nb)
    nz, k, P = 3, 2 * np.pi / 0.5, 3
    N = nf * nb
    field = torch.from_numpy(_field(rng, N, nz)).cuda()
    probes = c64(_gauss(nf, nb, rng.uniform(10, min(nf, nb) - 10, (P, 2)), 6.0))
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, "impedance")
    fb, ff = np.meshgrid(np.arange(nb), np.arange(nf), indexing="ij")
    mx, my = complex(eng.co.mu_x), complex(eng.co.mu_y)
    lam = 1 - (mx * (2 * np.cos(2 * np.pi * ff / nf) - 2) + my * (2 * np.cos(2 * np.pi * fb / nb) - 2))
    z0 = {}
    for kern in (0, 1):
        eng.kernels = kern
        pairs = generate_pairs(eng, field, probes, every=1, kind="noise")
        z0[kern] = pairs.z0.cpu().numpy().astype(np.complex128)
        sol = pairs.sol.cpu().numpy().astype(np.complex128)
        diag = pairs.diag.cpu().numpy().astype(np.complex128)
        for s in range(nz - 1):
            for p in range(P):
                v = _apply_i_minus_p(eng, sol[s, p], diag[s]).reshape(nb, nf)
                ref = np.fft.ifft2(np.fft.fft2(v) / lam).ravel()
                assert rel(z0[kern][s, p], ref) < 5e-6, (kern, s, p, rel(z0[kern][s, p], ref))
    eng.kernels = 0
    assert rel(z0[0], z0[1]) < 2e-6


_TAPS = [(0, 0), (0, -1), (0, 1), (-1, 0), (1, 0), (-1, -1), (-1, 1), (1, -1), (1, 1), (0, -2), (0, 2), (-2, 0), (2, 0)]


def _slice_operator(eng, diag):
    """P_s of one slice (forward orientation) as a sparse matrix: the engine's
    operator diagonals plus the slice's object diagonal."""
    import scipy.sparse as sp

    kc, kw, ke, ks, kn = (d.cpu().numpy().astype(np.complex128) for d in eng._diags)
    nf, N = eng.nx, eng.N
    f = np.arange(N) % nf
    w_ = np.where(f[1:] > 0, kw[1:], 0)       # (i, i-1)
    e_ = np.where(f[:-1] < nf - 1, ke[:-1], 0)  # (i, i+1)
    return sp.diags([kc + diag, w_, e_, ks[nf:], kn[:-nf]], [0, -1, 1, -nf, nf], format="csr")


def _learned_filter_np(z, F, nf, nb):
    Z = z.reshape(nb, nf)
    Zp = np.zeros((nb + 4, nf + 4), complex)
    Zp[2:-2, 2:-2] = Z
    y = Z.copy()
    for t, (dy, dx) in enumerate(_TAPS):
        y = y + F[t].reshape(nb, nf) * Zp[2 + dy:2 + dy + nb, 2 + dx:2 + dx + nf]
    return y.ravel()


@pytest.mark.parametrize("nf,nb,learned,mode", [
    (64, 64, False, "forward"), (256, 256, False, "forward"), (64, 64, True, "forward"),
    (256, 256, True, "forward"), (192, 192, True, "adjoint"), (96, 80, True, "forward"), (320, 40, True, "adjoint"),
])
def test_one_bicgstab_iteration_against_numpy(nf, nb, learned, mode):
    """One preconditioned BiCGStab iteration of one step (nz = 2, max_iter = 1)
    against numpy in complex128: right-hand side 2 P u, y = M p, v = A y,
    s = r - alpha v, z = M s, t = A z, x = alpha y + omega z, u + x.  M is
    the FFT preconditioner, and for the learned form M followed by the
    per-pixel 13-tap filter with random taps written into the learned
    workspace (the march reuses them: the network is not run).  The cases
    cover both transform kernels (four-step at 64, 192, 256; Stockham at
    96 x 80 and 320 x 40), the filter's image edges, several row pairs per CTA
    (64, 96), two column blocks (320) and the adjoint's conjugated operator,
    symbol and taps.  The update x is compared at 5e-5 (it is ~5 % of u, held
    in complex64)."""
    import ctypes

    from thick_ptycho_b200.cn3d import generate_pairs
    from thick_ptycho_b200.learned import LearnedPreconditioner

    rng = np.random.default_rng(nf * 7 + nb)
    nz, k, P = 2, 2 * np.pi / 0.5, 3
    N = nf * nb
    field = torch.from_numpy(_field(rng, N, nz, scale=2e-2)).cuda()
    probes = _gauss(nf, nb, np.column_stack([rng.uniform(8, nf - 8, P), rng.uniform(8, nb - 8, P)]), 6.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, "impedance")
    diag = generate_pairs(eng, field, c64(probes), every=1, kind="noise").diag[0].cpu().numpy().astype(np.complex128)
    Pf = _slice_operator(eng, diag)
    adj = mode == "adjoint"
    Pm = Pf.conj().T.tocsr() if adj else Pf
    fb, ff = np.meshgrid(np.arange(nb), np.arange(nf), indexing="ij")
    mx, my = complex(eng.co.mu_x), complex(eng.co.mu_y)
    lam = 1 - (mx * (2 * np.cos(2 * np.pi * ff / nf) - 2) + my * (2 * np.cos(2 * np.pi * fb / nb) - 2))
    if adj:
        lam = lam.conj()
    model = None
    F = None
    if learned:
        model = LearnedPreconditioner(nf, nb, 1.0, seed=0)
        lws = eng.learned_workspace(P)
        off = (int(eng.lib.tp_cnn_forward_ws_bytes(nf, nb, 1)) + 255) // 256 * 256
        F = 0.05 * (rng.standard_normal((13, N)) + 1j * rng.standard_normal((13, N)))
        lws[off:off + 13 * N * 8].view(torch.complex64).copy_(torch.from_numpy(F.astype(np.complex64)).cuda().ravel())
        if adj:
            F = F.conj()

    def M(v):
        z = np.fft.ifft2(np.fft.fft2(v.reshape(nb, nf)) / lam).ravel()
        return _learned_filter_np(z, F, nf, nb) if learned else z

    ex = torch.empty((P, N), dtype=torch.complex64, device="cuda")
    eng.read_stats()
    eng.march(field, P, mode, probes=c64(probes), exit_out=ex, precond="learned" if learned else True, model=model,
              reuse_filters=learned, fallback=False, max_iter=1, tol=1e-12)
    assert eng.read_stats()["iterations"] == P
    got = ex.cpu().numpy().astype(np.complex128)
    for p in range(P):
        u0 = probes[p]
        r0 = 2 * (Pm @ u0)
        y = M(r0)
        v = y - Pm @ y
        alpha = np.vdot(r0, r0) / np.vdot(r0, v)
        s = r0 - alpha * v
        z = M(s)
        t = z - Pm @ z
        omega = np.vdot(t, s) / np.vdot(t, t)
        x = alpha * y + omega * z
        assert rel(got[p] - u0, x) < 5e-5, (p, rel(got[p] - u0, x))


@pytest.mark.parametrize("nf,nb,mode", [(64, 64, "forward"), (256, 32, "adjoint"), (192, 45, "forward"),
                                         (128, 60, "adjoint_exact")])
def test_bulk_staged_filter_matches_shuffle_filter(nf, nb, mode):
    """The learned filter with each probe's rows staged by bulk copies (the
    default for widths 64, 128, 192, 256) against the register-shuffle kernel
    (`kernels = 4`) over a five-step march with random per-slice taps written
    into the learned workspace: 11 probes (a full and a partial probe group),
    solves converging after different iteration counts (probes leaving the
    filter's pending set), an odd row count (a last row pair of one row), the
    adjoint's conjugated taps.  Both kernels run the same multiply-adds in the
    same order, so the fields agree to the round-off of the fp64 dot products'
    summation order, and the iteration counts match."""
    from thick_ptycho_b200.learned import LearnedPreconditioner

    rng = np.random.default_rng(nf + 3 * nb)
    nz, k, P = 6, 2 * np.pi / 0.5, 11
    N, L = nf * nb, nz - 1
    field = torch.from_numpy(_field(rng, N, nz, scale=1e-2)).cuda()
    probes = _gauss(nf, nb, np.column_stack([rng.uniform(8, nf - 8, P), rng.uniform(8, nb - 8, P)]), 5.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, "impedance")
    model = LearnedPreconditioner(nf, nb, 1.0, seed=0)
    lws = eng.learned_workspace(P)
    off = (int(eng.lib.tp_cnn_forward_ws_bytes(nf, nb, L)) + 255) // 256 * 256
    F = 0.01 * (rng.standard_normal((13, L * N)) + 1j * rng.standard_normal((13, L * N)))
    lws[off:off + 13 * L * N * 8].view(torch.complex64).copy_(torch.from_numpy(F.astype(np.complex64)).cuda().ravel())
    fwd = eng.new_store(P)
    eng.march(field, P, "forward", probes=c64(probes), u_store=fwd, tol=1e-7)
    src = c64(rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N)))
    out = {}
    for kern in (0, 4):
        eng.kernels = kern
        eng.read_stats()
        store = eng.new_store(P)
        gc = torch.zeros((L, N), dtype=torch.complex64, device="cuda")
        kw = dict(precond="learned", model=model, reuse_filters=True, fallback=False, tol=1e-6, u_store=store)
        if mode == "adjoint_exact":
            eng.march(field, P, mode, src_exit=src, u_fwd=fwd, grad_c=gc, **kw)
        elif mode == "adjoint":
            eng.march(field, P, mode, src_exit=src, **kw)
        else:
            eng.march(field, P, mode, probes=c64(probes), **kw)
        eng.device_status()
        st = eng.read_stats()
        assert st["failed"] == 0, st
        out[kern] = (store.cpu().numpy(), gc.cpu().numpy(), st)
    eng.kernels = 0
    assert out[0][2]["iterations"] == out[4][2]["iterations"], (out[0][2], out[4][2])
    assert out[0][2]["iterations"] > P * L, out[0][2]  # some solves took more than one iteration
    assert rel(out[0][0], out[4][0]) < 1e-6
    if mode == "adjoint_exact":
        assert rel(out[0][1], out[4][1]) < 1e-6


@pytest.mark.parametrize("nf,nb,mode,bc", [(64, 64, "forward", "impedance"), (256, 32, "adjoint_exact", "neumann"),
                                           (192, 48, "forward", "dirichlet"), (128, 66, "adjoint", "impedance")])
def test_tma_stencils_match_per_thread_loads(nf, nb, mode, bc):
    """The stencil kernels with their inputs staged by tensor-memory copies
    (right-hand side, matvecs, finish; widths 64, 128, 192, 256) against the
    same arithmetic with per-thread loads (`kernels = 2`): fields and the
    exact-adjoint gradient equal to fp32 round-off (the fp64 dot products are
    summed in a different order), the same iteration counts up to a
    convergence decision that round-off may tip, and both within 1e-5 of the
    oracle."""
    rng = np.random.default_rng(nf + nb)
    nz, k, P = 7, 2 * np.pi / 0.5, 6
    N = nf * nb
    n = _field(rng, N, nz, scale=1e-2)
    field = torch.from_numpy(n).cuda()
    probes = _gauss(nf, nb, np.column_stack([rng.uniform(8, nf - 8, P), rng.uniform(8, nb - 8, P)]), 5.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, bc)
    fwd = eng.new_store(P)
    eng.march(field, P, "forward", probes=c64(probes), u_store=fwd, tol=1e-7)
    src = c64(rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N)))
    out = {}
    for kern in (0, 2):
        eng.kernels = kern
        eng.read_stats()
        store = eng.new_store(P)
        gc = torch.zeros((nz - 1, N), dtype=torch.complex64, device="cuda")
        if mode == "adjoint_exact":
            eng.march(field, P, mode, src_exit=src, u_fwd=fwd, grad_c=gc, u_store=store, tol=1e-7)
        elif mode == "adjoint":
            eng.march(field, P, mode, src_exit=src, u_store=store, tol=1e-7)
        else:
            eng.march(field, P, mode, probes=c64(probes), u_store=store, tol=1e-7)
        eng.device_status()
        st = eng.read_stats()
        assert st["failed"] == 0, st
        out[kern] = (store.cpu().numpy(), gc.cpu().numpy(), st)
    eng.kernels = 0
    assert abs(out[0][2]["iterations"] - out[2][2]["iterations"]) <= 2
    assert rel(out[0][0], out[2][0]) < 1e-6
    if mode == "adjoint_exact":
        assert rel(out[0][1], out[2][1]) < 1e-6
    if mode == "forward":
        co = po.bc_coefficients(k, 1.0, 1.0, dy=1.0, bc_type=bc, dimension=3)
        A, B = po.step_matrices_2d(nf, nb, co, bc, 1.0)
        C = po.object_contribution(n, k, 1.0)
        for p in (0, P - 1):
            assert rel(out[0][0][p].T, po.march(A, B, C, probes[p])) < TOL
