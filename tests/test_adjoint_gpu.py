"""GPU exact adjoint + fused gradient against the complex128 oracle and
central finite differences.

Tolerance: relative L2 ≤ 1e-5 for adjoint fields and for the fused gradient
(which sums the probe contributions in fp32), and against finite differences
of the complex128 oracle loss at ≤ 1e-3 relative per sampled voxel (the
finite differences themselves carry ~1e-4 truncation and round-off error).
"""

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200.cn2d import CN2D  # noqa: E402

GRAD_TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _problem(N=64, nz=24, P=6, seed=3, bc="impedance"):
    rng = np.random.default_rng(seed)
    k, dx, dz = 4 * np.pi, 1.0, 1.0
    n = 1 + 1e-3 * (rng.standard_normal((N, nz)) + 0.2j * rng.standard_normal((N, nz)))
    x = np.arange(N)
    cents = np.linspace(10, N - 10, P)
    probes = np.exp(-((x[None] - cents[:, None]) ** 2) / 36.0).astype(complex)
    amp = np.abs(np.fft.fft(probes, axis=-1)) * 1.05 + 0.01
    return k, dx, dz, n, probes, amp, bc


def _oracle_grad(k, dx, dz, n, probes, amp, bc):
    co = po.bc_coefficients(k, dx, dz, bc_type=bc)
    A, B = po.step_matrices_1d(n.shape[0], co, bc, dz)
    C = po.object_contribution(n, k, dz)
    gc = np.zeros((n.shape[0], n.shape[1] - 1), dtype=complex)
    loss = 0.0
    lams = []
    for p in range(probes.shape[0]):
        u = po.march(A, B, C, probes[p])
        l, ge = po.amplitude_loss_and_grad(u[:, -1][None], amp[p][None])
        loss += l
        src = np.zeros_like(gc)
        src[:, -1] = ge[0]
        lam = po.exact_adjoint(A, B, C, src)
        lams.append(lam)
        gc += po.grad_c_from_adjoint(u, lam)
    return loss, gc, po.chain_grad_to_n(gc, k, dz), lams


def _gpu_grad(k, dx, dz, n, probes, amp, bc, N, nz):
    P = probes.shape[0]
    eng = CN2D(N, nz, k, dx, dz, bc)
    field = torch.from_numpy(n).cuda()
    ff = eng.factor(field, "forward")
    fa = eng.factor(field, "adjoint_exact")
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    st = eng.new_store(P)
    ex = torch.empty((P, N), dtype=torch.complex64, device="cuda")
    eng.march(ff, P, probes=pr, u_store=st, exit_out=ex)
    U = torch.fft.fft(ex.to(torch.complex128), dim=-1)
    mag = U.abs()
    a = torch.from_numpy(amp).cuda()
    ge = N * torch.fft.ifft(2 * (mag - a) * U / mag, dim=-1)
    gc = eng.new_grad_buffer()
    lam_st = eng.new_store(P)
    eng.march(fa, P, src_exit=ge.to(torch.complex64).contiguous(), u_store=lam_st, u_fwd=st, grad_c=gc)
    gn = eng.grad_to_n(gc)
    eng.device_status()
    return eng.unchunk_rows(gc).cpu().numpy().T, gn.cpu().numpy(), eng, lam_st


@pytest.mark.parametrize("bc", ["impedance", "neumann", "dirichlet"])
def test_exact_adjoint_gradient_matches_oracle(bc):
    k, dx, dz, n, probes, amp, bc = _problem(bc=bc)
    N, nz = n.shape
    loss, gc_ref, gn_ref, lams = _oracle_grad(k, dx, dz, n, probes, amp, bc)
    gc, gn, eng, lam_st = _gpu_grad(k, dx, dz, n, probes, amp, bc, N, nz)
    assert rel(gc, gc_ref) < GRAD_TOL, rel(gc, gc_ref)
    assert rel(gn, gn_ref) < GRAD_TOL, rel(gn, gn_ref)
    # adjoint fields themselves (store index t holds slice L+1-t's λ for t>=1)
    lam = eng.unchunk(lam_st).cpu().numpy()
    L = nz - 1
    for p in range(probes.shape[0]):
        got = lam[p][:, 1:][:, ::-1]  # → columns slice 1..L
        assert rel(got, lams[p]) < 1e-5


def test_gradient_matches_finite_differences():
    k, dx, dz, n, probes, amp, bc = _problem(N=40, nz=12, P=3, seed=11)
    N, nz = n.shape
    _, gn, _, _ = _gpu_grad(k, dx, dz, n, probes, amp, bc, N, nz)
    co = po.bc_coefficients(k, dx, dz, bc_type=bc)
    A, B = po.step_matrices_1d(N, co, bc, dz)

    def loss(nn):
        C = po.object_contribution(nn, k, dz)
        ex = np.array([po.march(A, B, C, probes[p])[:, -1] for p in range(probes.shape[0])])
        return po.amplitude_loss_and_grad(ex, amp)[0]

    rng = np.random.default_rng(0)
    h = 1e-7
    scale = np.abs(gn).max()
    for _ in range(8):
        x, t = int(rng.integers(0, N)), int(rng.integers(0, nz))
        for d, part in ((1.0, 0), (1j, 1)):
            e = np.zeros_like(n)
            e[x, t] = h * d
            fd = (loss(n + e) - loss(n - e)) / (2 * h)
            an = gn[x, t].real if part == 0 else gn[x, t].imag
            assert abs(fd - an) <= 1e-3 * max(abs(fd), 1e-2 * scale), (x, t, part, fd, an)
