"""GPU parity of the 3D multislice (the reference's multislice is 2D only):
against the complex128 restatement `ms_forward_3d` (itself pinned to the
reference's 2D MSForwardModelSolver by a y-invariant reduction), on runtime
and compile-time FFT plans, through the drop-in solver with a 3D space, and
the adjoint gradient against finite differences of the oracle.

Tolerance: relative L2 ≤ 1e-5 for fields (complex64 vs complex128).
"""

from types import SimpleNamespace

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200.ms2d import MSGpuSolver  # noqa: E402
from thick_ptycho_b200.ms3d import MS3D, MS3DFunction  # noqa: E402

TOL = 1e-5
K = 4 * np.pi


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _object(n1, n2, nz, seed, amp=1e-3):
    rng = np.random.default_rng(seed)
    return 1 + amp * (rng.standard_normal((n1, n2, nz)) + 0.1j * rng.standard_normal((n1, n2, nz)))


def _probes(n1, n2, P, seed, waist=6.0):
    rng = np.random.default_rng(seed)
    a = np.arange(n1)[:, None]
    b = np.arange(n2)[None, :]
    out = []
    for _ in range(P):
        ca, cb = rng.uniform(0.3 * n1, 0.7 * n1), rng.uniform(0.3 * n2, 0.7 * n2)
        out.append(np.exp(-((a - ca) ** 2 + (b - cb) ** 2) / (2 * waist**2)) * np.exp(1j * rng.uniform(0, 6.28)))
    return np.array(out)


@pytest.mark.parametrize("n1,n2,d2", [(64, 48, 0.8), (128, 128, 1.0), (256, 32, 1.0)])
def test_ms3d_against_oracle(n1, n2, d2):
    """Runtime plan (48), compile-time plans (32, 64, 128, 256), dx != dy."""
    nz, P = 24, 3
    n = _object(n1, n2, nz, 1)
    probes = _probes(n1, n2, P, 2)
    eng = MS3D(n1, n2, nz, K, 1.0, d2, 1.0)
    T = eng.transmission(torch.from_numpy(n).cuda())
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    st = torch.empty((P, nz, n1 * n2), dtype=torch.complex64, device="cuda")
    ex = torch.empty((P, n1 * n2), dtype=torch.complex64, device="cuda")
    eng.march(T, pr, u_store=st, exit_out=ex)
    got = st.cpu().numpy().reshape(P, nz, n1, n2)
    exit_ = ex.cpu().numpy().reshape(P, n1, n2)
    for p in range(P):
        ref = po.ms_forward_3d(n, probes[p], K, 1.0, d2, 1.0)
        assert rel(got[p].transpose(1, 2, 0), ref) < TOL, (p, rel(got[p].transpose(1, 2, 0), ref))
        assert np.array_equal(exit_[p], got[p, -1])


def test_ms3d_y_invariant_matches_2d_oracle():
    """A y-invariant object and probe: every line equals the 2D multislice."""
    n1, n2, nz, P = 256, 32, 40, 2
    rng = np.random.default_rng(5)
    n2d = 1 + 1e-3 * (rng.standard_normal((n1, nz)) + 0.1j * rng.standard_normal((n1, nz)))
    x = np.arange(n1)
    pr2d = np.array([np.exp(-((x - c) ** 2) / 64.0) for c in (90.0, 170.0)]).astype(complex)
    n = np.repeat(n2d[:, None, :], n2, axis=1)
    probes = np.repeat(pr2d[:, :, None], n2, axis=2)
    eng = MS3D(n1, n2, nz, K, 1.0, 1.0, 1.0)
    T = eng.transmission(torch.from_numpy(n).cuda())
    ex = torch.empty((P, n1 * n2), dtype=torch.complex64, device="cuda")
    eng.march(T, torch.from_numpy(probes.astype(np.complex64)).cuda(), exit_out=ex)
    ex = ex.cpu().numpy().reshape(P, n1, n2)
    for p in range(P):
        ref = po.ms_forward(n2d, pr2d[p], K, 1.0, 1.0)[:, -1]
        for j in (0, 17, 31):
            assert rel(ex[p, :, j], ref) < TOL, (p, j)


def test_ms3d_256_squared_subset():
    """256 x 256 x 128 nodes, 8 probes; two probes checked in complex128."""
    n1 = n2 = 256
    nz, P = 128, 8
    n = _object(n1, n2, nz, 7, amp=5e-4)
    probes = _probes(n1, n2, P, 8, waist=12.0)
    eng = MS3D(n1, n2, nz, K, 1.0, 1.0, 1.0)
    T = eng.transmission(torch.from_numpy(n).cuda())
    ex = torch.empty((P, n1 * n2), dtype=torch.complex64, device="cuda")
    eng.march(T, torch.from_numpy(probes.astype(np.complex64)).cuda(), exit_out=ex)
    ex = ex.cpu().numpy().reshape(P, n1, n2)
    for p in (0, 5):
        ref = po.ms_forward_3d(n, probes[p], K, 1.0, 1.0, 1.0)[:, :, -1]
        assert rel(ex[p], ref) < TOL, (p, rel(ex[p], ref))


def test_ms3d_adjoint_gradient_matches_finite_differences():
    n1 = n2 = 32
    nz, P = 8, 2
    n = _object(n1, n2, nz, 11)
    probes = _probes(n1, n2, P, 12, waist=4.0)
    rng = np.random.default_rng(13)
    target = (rng.standard_normal((P, n1, n2)) + 1j * rng.standard_normal((P, n1, n2))) * 0.1
    eng = MS3D(n1, n2, nz, K, 1.0, 1.0, 1.0)
    field = torch.from_numpy(n.reshape(n1 * n2, nz)).cuda().requires_grad_(True)
    pr = torch.from_numpy(probes.reshape(P, -1).astype(np.complex64)).cuda()
    ex = MS3DFunction.apply(field, pr, eng)
    tg = torch.from_numpy(target.reshape(P, -1)).cuda()
    loss = torch.sum((ex.to(torch.complex128) - tg).abs() ** 2)
    loss.backward()
    g = field.grad.cpu().numpy().reshape(n1, n2, nz)

    def oloss(nn):
        e = np.array([po.ms_forward_3d(nn, probes[p], K, 1.0, 1.0, 1.0)[:, :, -1] for p in range(P)])
        return float(np.sum(np.abs(e - target) ** 2))

    assert abs(loss.item() - oloss(n)) < 1e-5 * oloss(n)
    h = 1e-6
    scale = np.abs(g).max()
    for (a, b, t) in [(16, 16, 0), (12, 18, 3), (20, 10, 6), (15, 15, 5)]:
        for d, part in ((1.0, 0), (1j, 1)):
            e = np.zeros_like(n)
            e[a, b, t] = h * d
            fd = (oloss(n + e) - oloss(n - e)) / (2 * h)
            an = g[a, b, t].real if part == 0 else g[a, b, t].imag
            assert abs(fd - an) <= 2e-3 * max(abs(fd), 1e-2 * scale), (a, b, t, part, fd, an)
    assert np.all(g[:, :, -1] == 0)  # the last plane does not enter the multislice model


def test_ms_solver_accepts_3d_space():
    """The drop-in solver runs a 3D simulation space (which the reference's
    MSForwardModelSolver rejects) with the reference's field layout."""
    nx = ny = 64
    nz, P = 16, 3
    n = _object(nx, ny, nz, 21)
    probes = _probes(nx, ny, P, 22)
    ss = SimpleNamespace(dimension=3, effective_shape=(nx, ny, nz), block_size=nx * ny, nz=nz, nx=nx,
                         effective_nx=nx, effective_ny=ny, num_probes=P, num_projections=1, probe_angles=[0.0],
                         n_medium=1.0, k=K, dx=1.0, dy=1.0, dz=1.0, total_scans=P,
                         refractive_index_empty=np.ones((nx, ny, nz), dtype=complex))
    s = MSGpuSolver(ss, probes[None])
    u = s.solve(n=n)
    assert u.shape == (1, 1, P, nx, ny, nz)
    for p in range(P):
        ref = po.ms_forward_3d(n, probes[p], K, 1.0, 1.0, 1.0)
        assert rel(u[0, 0, p], ref) < TOL, p
    single = s._solve_single_probe(n=n, probe=probes[1])
    assert single.shape == (nx, ny, nz) and rel(single, po.ms_forward_3d(n, probes[1], K, 1.0, 1.0, 1.0)) < TOL
    ff = s.get_farfield_intensities(u, poisson_noise=False)
    assert ff.shape == (P, nx * ny)
    ex = np.array([po.ms_forward_3d(n, probes[p], K, 1.0, 1.0, 1.0)[:, :, -1].reshape(-1) for p in range(P)])
    assert rel(ff, po.farfield_intensity(ex, dimension=3)) < 1e-5
