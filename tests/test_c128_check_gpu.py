"""The complex128 check build (``libtpcuda_c128.so``) against the complex128 oracle.

The check build compiles the 2D factorisation and marches with complex128
state, factor sets and fields (``TP_C128_CHECK``), so the algorithms that the
complex64 build rounds -- the partitioned tridiagonal solve with its spike
vectors and "1 + eps" deviation storage, parallel cyclic reduction or its
skip, the Cayley step, the pair-sum store and the fused exact-adjoint
gradient -- are compared with the oracle's per-slice SuperLU march far below
complex64 round-off.  Cases: the 256 x 128 geometry of the CPU-runnable
benchmark (warp path; every mode), N = 512 (team path, PCR kept), N = 1024 at
λ = 0.1 (team path: every separator coupling below 1e-17, so the PCR levels
are skipped; checked on the factor set), and a subset of the 2048 x 1024
batched workload: its central 1024 columns, 129 nodes and 64 of its probes
(stride 3).

The same library holds the 3D march in complex128 (BiCGStab with the FFT
preconditioner, fp64 vectors and dots), run at a Krylov tolerance of 1e-13
against the oracle's per-slice sparse LU: 64 x 64 (register four-step
transforms, 8 x 8), 128 x 128 (16 x 8) in the adjoint, 48 x 40 (runtime
Stockham plan) and 32 x 32 (compile-time Stockham plan) with the exact
adjoint and its gradient, and the reverse march.

Tolerance: ≤ 1e-12 relative L2 for fields, exit waves and gradients.
"""

import struct

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200.cn2d import CN2D  # noqa: E402
from thick_ptycho_b200.cn3d import CN3D  # noqa: E402
from thick_ptycho_b200.workloads import CONFIG0, CONFIG1, gaussian_probes_2d  # noqa: E402

TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def c128(x):
    return torch.from_numpy(np.ascontiguousarray(x).astype(np.complex128)).cuda()


def _coupling(eng, fs):
    """The factor set's PCR coupling bound (float bits in the tail word)."""
    off = eng.factor_bytes - 256
    return struct.unpack("<f", bytes(fs.buf[off:off + 4].cpu().numpy().tobytes()))[0]


def _check_case(N, nz, k, n, probes, bc, grad=True, sums=False, two_slice=True):
    eng = CN2D(N, nz, k, 1.0, 1.0, bc, check=True)
    assert eng.cdtype == torch.complex128
    P = probes.shape[0]
    co = po.bc_coefficients(k, 1.0, 1.0, bc_type=bc)
    A, B = po.step_matrices_1d(N, co, bc, 1.0)
    C = po.object_contribution(n, k, 1.0)
    lus, Bs = po.build_lu_factors(A, B, C)
    u_ref = np.array([po.march_with_lu(lus, Bs, np.zeros(N, complex), probes[p]) for p in range(P)])
    field = c128(n)
    ff = eng.factor(field, "forward")
    st = eng.new_store(P)
    ex = torch.empty((P, N), dtype=torch.complex128, device="cuda")
    eng.march(ff, P, probes=c128(probes), u_store=st, exit_out=ex)
    eng.device_status()
    assert rel(ex.cpu().numpy(), u_ref[:, :, -1]) < TOL, rel(ex.cpu().numpy(), u_ref[:, :, -1])
    assert rel(eng.unchunk(st).cpu().numpy(), u_ref) < TOL
    out = {"engine": eng, "forward_factors": ff}
    if not grad:
        return out
    rng = np.random.default_rng(N + nz)
    e = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    srcs = np.zeros((P, N, nz - 1), dtype=complex)
    srcs[:, :, -1] = e
    lam = po.exact_adjoint_many(A, B, C, srcs)
    gref = sum(po.grad_c_from_adjoint(u_ref[p], lam[p]) for p in range(P))
    fa = eng.factor(field, "adjoint_exact")
    if two_slice:
        # the exact adjoint reading two stored forward slices per step
        gc = eng.new_grad_buffer()
        eng.march(fa, P, src_exit=c128(e), u_fwd=st, grad_c=gc)
        eng.device_status()
        got = eng.unchunk_rows(gc).cpu().numpy().T
        assert rel(got, gref) < TOL, rel(got, gref)
        gn = eng.grad_to_n(gc).cpu().numpy()
        assert rel(gn, po.chain_grad_to_n(gref, k, 1.0)) < TOL
    if sums:
        # forward storing the half pair sums, Cayley-form exact adjoint reading them
        hs, gs = eng.new_store(P), eng.new_grad_buffer()
        eng.march(ff, P, probes=c128(probes), u_store=hs, store_sums=True)
        eng.march(fa, P, src_exit=c128(e), u_fwd=hs, grad_c=gs, store_sums=True)
        eng.device_status()
        half = 0.5 * (u_ref[:, :, 1:] + u_ref[:, :, :-1])
        assert rel(eng.unchunk(hs).cpu().numpy()[:, :, 1:], half) < TOL
        got_s = eng.unchunk_rows(gs).cpu().numpy().T
        assert rel(got_s, gref) < TOL, rel(got_s, gref)
    return out


def test_c128_config0_geometry_every_mode():
    """Warp path (32 chunks of 8 rows) at N = 256, nz = 128, 32 probes."""
    w = CONFIG0
    geo = w.geometry()
    n = 1 - w.delta_n()
    probes = w.probes(geo)
    _check_case(w.nx, w.nz, geo.k, n, probes, "impedance")
    eng = CN2D(w.nx, w.nz, geo.k, 1.0, 1.0, "neumann", check=True)
    co = po.bc_coefficients(geo.k, 1.0, 1.0, bc_type="neumann")
    A, B = po.step_matrices_1d(w.nx, co, "neumann", 1.0)
    C = po.object_contribution(n, geo.k, 1.0)
    rng = np.random.default_rng(3)
    P = 4
    rhs = rng.standard_normal((P, w.nx, w.nz - 1)) + 1j * rng.standard_normal((P, w.nx, w.nz - 1))
    src = c128(rhs.transpose(0, 2, 1))
    field = c128(n)
    for mode, use_probe, use_src in (("forward", True, True), ("adjoint", False, True), ("reverse", True, False)):
        st = eng.new_store(P)
        eng.march(eng.factor(field, mode), P, probes=c128(probes[:P]) if use_probe else None,
                  src_probe=src if use_src else None, u_store=st)
        eng.device_status()
        got = eng.unchunk(st).cpu().numpy()
        for p in range(P):
            ref = po.march(A, B, C, probes[p] if use_probe else None, mode, rhs_block=rhs[p] if use_src else None)
            assert rel(got[p], ref) < TOL, (mode, p, rel(got[p], ref))


@pytest.mark.parametrize("bc", ["impedance", "dirichlet"])
def test_c128_team_path_with_pcr(bc):
    """Team path at N = 512 (128 chunks of 4 rows): the separators keep their
    7 PCR levels; pair-sum store and Cayley-form exact adjoint."""
    N, nz, P, k = 512, 48, 6, 4 * np.pi
    rng = np.random.default_rng(1)
    n = 1 + 1e-3 * (rng.standard_normal((N, nz)) + 0.1j * rng.standard_normal((N, nz)))
    probes = gaussian_probes_2d(N, np.linspace(60, 450, P), 8.0)
    res = _check_case(N, nz, k, n, probes, bc, sums=True)
    assert _coupling(res["engine"], res["forward_factors"]) >= 1e-17  # PCR kept


def test_c128_team_path_pcr_skipped():
    """N = 1024 at λ = 0.1 (k = 20π): |μ| = dz/(4k dx²) ≈ 0.004 makes every
    separator coupling of the 8-row chunks smaller than 1e-17, so the march
    solves the reduced system directly (the PCR skip)."""
    N, nz, P, k = 1024, 40, 5, 20 * np.pi
    rng = np.random.default_rng(2)
    n = 1 + 1e-3 * (rng.standard_normal((N, nz)) + 0.1j * rng.standard_normal((N, nz)))
    probes = gaussian_probes_2d(N, np.linspace(100, 900, P), 8.0)
    # (in complex128 the two-slice adjoint's factor double buffer and stencil
    # rows exceed 227 KB of shared memory at N = 1024: Cayley form only)
    res = _check_case(N, nz, k, n, probes, "impedance", sums=True, two_slice=False)
    assert _coupling(res["engine"], res["forward_factors"]) < 1e-17  # PCR skipped


def test_c128_batched_workload_subset():
    """The 2048 x 1024 batched workload's central 1024 columns over its first
    129 nodes, with 64 of its probes (stride 3 px, waist 8 px) that lie in the
    crop: team path at N = 1024, exit waves and the fused gradient."""
    w = CONFIG1
    geo = w.geometry()
    dn = w.delta_n()[512:1536, :129]
    centres = np.asarray(geo.centres, dtype=float)
    inside = centres[(centres >= 512 + 40) & (centres < 1536 - 40)][:64] - 512
    probes = gaussian_probes_2d(1024, inside, w.waist)
    _check_case(1024, 129, geo.k, 1 - dn, probes, "impedance", sums=True, two_slice=False)


# ------------------------------------------------------------------ 3D march
KTOL3 = 1e-13  # BiCGStab stopping residual of the complex128 3D march


def _field3(rng, N, nz, scale=5e-3):
    return 1 + scale * (rng.standard_normal((N, nz)) + 0.2j * rng.standard_normal((N, nz)))


def _gauss3(nf, nb, centres, w):
    f = np.arange(nf)[None, :]
    b = np.arange(nb)[:, None]
    return np.array([np.exp(-((f - cf) ** 2 + (b - cb) ** 2) / w**2).ravel() for cf, cb in centres]).astype(complex)


def _oracle3(nf, nb, nz, k, dz, bc, n):
    co = po.bc_coefficients(k, 1.0, dz, dy=1.0, bc_type=bc, dimension=3)
    A, B = po.step_matrices_2d(nf, nb, co, bc, dz)
    return A, B, po.object_contribution(n, k, dz)


@pytest.mark.parametrize("nf,nb,bc", [(64, 64, "impedance"), (64, 64, "neumann"), (64, 64, "dirichlet"),
                                      (48, 40, "impedance")])
def test_c128_3d_forward(nf, nb, bc):
    """Forward march of 4 probes over 12 nodes in complex128."""
    rng = np.random.default_rng(nf + nb)
    nz, k, P = 12, 2 * np.pi / 0.5, 4
    N = nf * nb
    n = _field3(rng, N, nz)
    probes = _gauss3(nf, nb, np.column_stack([rng.uniform(10, nf - 10, P), rng.uniform(10, nb - 10, P)]), 6.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, bc, check=True)
    assert eng.cdtype == torch.complex128
    store = eng.new_store(P)
    eng.march(torch.from_numpy(n).cuda(), P, "forward", probes=c128(probes), u_store=store, tol=KTOL3, max_iter=60)
    st = eng.read_stats()
    assert st["failed"] == 0 and st["solves"] == P * (nz - 1), st
    u = store.permute(0, 2, 1).cpu().numpy()
    A, B, C = _oracle3(nf, nb, nz, k, 1.0, bc, n)
    for p in range(P):
        ref = po.march(A, B, C, probes[p])
        assert rel(u[p], ref) < TOL, (p, rel(u[p], ref))


def test_c128_3d_adjoint_128():
    """The reference adjoint with a right-hand-side block at 128 x 128."""
    rng = np.random.default_rng(5)
    nf = nb = 128
    nz, k, P = 8, 2 * np.pi / 0.5, 2
    N = nf * nb
    n = _field3(rng, N, nz)
    rhs = rng.standard_normal((P, N, nz - 1)) + 1j * rng.standard_normal((P, N, nz - 1))
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, "impedance", check=True)
    A, B, C = _oracle3(nf, nb, nz, k, 1.0, "impedance", n)
    field = torch.from_numpy(n).cuda()
    for p in range(P):
        store = eng.new_store(1)
        # the adjoint's source rows by step: step t solves slice L+1-t
        sh = c128(rhs[p].T[::-1])
        eng.march(field, 1, "adjoint", src_shared=sh, u_store=store, tol=KTOL3, max_iter=60)
        assert eng.read_stats()["failed"] == 0
        ref = po.march(A, B, C, None, "adjoint", rhs_block=rhs[p])
        got = store[0].T.cpu().numpy()
        assert rel(got, ref) < TOL, rel(got, ref)


@pytest.mark.parametrize("exact", [False, True])
def test_c128_3d_exact_adjoint_gradient(exact):
    """Forward + exact adjoint with the fused gradient at 32 x 32 x 10."""
    rng = np.random.default_rng(21)
    nf = nb = 32
    nz, k, P = 10, 4 * np.pi, 3
    N = nf * nb
    n = _field3(rng, N, nz)
    probes = _gauss3(nf, nb, rng.uniform(10, 22, (P, 2)), 5.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 1.0, "impedance", exact_ref_coeff=exact, check=True)
    field = torch.from_numpy(n).cuda()
    store = eng.new_store(P)
    eng.march(field, P, "forward", probes=c128(probes), u_store=store, tol=KTOL3, max_iter=60)
    srcs = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    gc = torch.zeros((nz - 1, N), dtype=torch.complex128, device="cuda")
    eng.march(field, P, "adjoint_exact", src_exit=c128(srcs), u_fwd=store, grad_c=gc, tol=KTOL3, max_iter=60)
    assert eng.read_stats()["failed"] == 0
    co = po.bc_coefficients(k, 1.0, 1.0, dy=1.0, bc_type="impedance", dimension=3)
    A, B = po.step_matrices_2d(nf, nb, co, "impedance", 1.0)
    C = po.object_contribution(n, k, 1.0, exact_ref_coeff=exact)
    u = np.array([po.march(A, B, C, probes[p]) for p in range(P)])
    assert rel(store.permute(0, 2, 1).cpu().numpy(), u) < TOL
    src = np.zeros((P, N, nz - 1), dtype=complex)
    src[:, :, -1] = srcs
    lam = po.exact_adjoint_many(A, B, C, src)
    gcr = sum(po.grad_c_from_adjoint(u[p], lam[p]) for p in range(P))
    assert rel(gc.cpu().numpy().T, gcr) < TOL, rel(gc.cpu().numpy().T, gcr)
    gn = eng.grad_to_n(gc, field).cpu().numpy()
    assert rel(gn, po.chain_grad_to_n(gcr, k, 1.0, n=n, exact_ref_coeff=exact)) < TOL


def test_c128_3d_reverse_and_learned_rejected():
    """Reverse march (sigma = -1, dz = 0.5) in complex128; the check build has
    no learned correction and says so."""
    rng = np.random.default_rng(9)
    nf = nb = 32
    nz, k, P = 8, 4 * np.pi, 2
    N = nf * nb
    n = _field3(rng, N, nz)
    probes = _gauss3(nf, nb, rng.uniform(10, 22, (P, 2)), 5.0)
    eng = CN3D(nf, nb, nz, k, 1.0, 1.0, 0.5, "neumann", check=True)
    store = eng.new_store(P)
    eng.march(torch.from_numpy(n).cuda(), P, "reverse", probes=c128(probes), u_store=store, tol=KTOL3, max_iter=60)
    assert eng.read_stats()["failed"] == 0
    A, B, C = _oracle3(nf, nb, nz, k, 0.5, "neumann", n)
    u = store.permute(0, 2, 1).cpu().numpy()
    for p in range(P):
        ref = po.march(A, B, C, probes[p], "reverse")
        assert rel(u[p], ref) < TOL, (p, rel(u[p], ref))
    from thick_ptycho_b200.learned import LearnedPreconditioner

    model = LearnedPreconditioner(nf, nb, 1.0, seed=0)
    with pytest.raises(Exception, match="check build"):
        eng.march(torch.from_numpy(n).cuda(), P, "forward", probes=c128(probes), precond="learned", model=model,
                  fallback=False)
