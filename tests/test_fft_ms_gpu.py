"""GPU FFT heads and the multislice march against NumPy and the complex128
oracle (whose multislice is pinned to the reference's golden vectors).

Tolerances: FFTs ≤ 2e-6 relative L2 (complex64, fp64 twiddles); far field
and amplitude residual ≤ 1e-5; multislice exit waves / fields ≤ 1e-5
relative L2 after 127–1023 slices; multislice gradient ≤ 1e-4 against the
oracle's adjoint and finite differences (h = 1e-7, complex128) within 1e-3.
"""

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200 import SimulationGeometry, heads  # noqa: E402
from thick_ptycho_b200.ms2d import MS2D, MSFunction, MSGpuSolver  # noqa: E402
from thick_ptycho_b200.workloads import CONFIG0, CONFIG1  # noqa: E402


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("n", [2048, 1024, 256, 192, 240, 12, 4096, 3])
def test_fft1d_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = (rng.standard_normal((7, n)) + 1j * rng.standard_normal((7, n))).astype(np.complex64)
    xd = torch.from_numpy(x).cuda()
    f = heads.fft1d(xd).cpu().numpy()
    assert rel(f, np.fft.fft(x.astype(np.complex128), axis=-1)) < 2e-6
    i = heads.fft1d(xd, inverse=True).cpu().numpy()
    assert rel(i, np.fft.ifft(x.astype(np.complex128), axis=-1)) < 2e-6


def test_fft_rejects_unsupported_lengths():
    x = torch.zeros((1, 257), dtype=torch.complex64, device="cuda")
    with pytest.raises(Exception, match="257"):
        heads.fft1d(x)


def test_farfield_and_amplitude_residual():
    rng = np.random.default_rng(1)
    P, N = 40, 2048
    e = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    amp = np.abs(np.fft.fft(e, axis=-1)) * 1.03
    ed = torch.from_numpy(e.astype(np.complex64)).cuda()
    ff = heads.farfield_intensity(ed).cpu().numpy()
    assert rel(ff, po.farfield_intensity(e)) < 1e-5
    loss, g = heads.amplitude_residual(ed, torch.from_numpy(amp).cuda())
    lref, gref = po.amplitude_loss_and_grad(e, amp)
    assert abs(loss.item() - lref) < 1e-5 * lref
    assert rel(g.cpu().numpy(), gref) < 1e-5


@pytest.mark.parametrize("w", [CONFIG0, CONFIG1])
def test_multislice_against_oracle(w):
    """CONFIG0 (N=256, 127 slices, 32 probes) fully; CONFIG1 (N=2048, 1023
    slices, 512 probes) with three probes checked in complex128."""
    geo = w.geometry()
    dn = w.delta_n()
    probes = w.probes(geo)
    eng = MS2D(w.nx, w.nz, geo.k, 1.0, 1.0)
    T = eng.transmission(torch.from_numpy(1 + dn).cuda())
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    ex = torch.empty_like(pr)
    eng.march(T, pr, exit_out=ex)
    ex = ex.cpu().numpy()
    check = range(w.num_probes) if w.num_probes <= 32 else (0, 255, 511)
    for p in check:
        ref = po.ms_forward(1 + dn, probes[p], geo.k, 1.0, 1.0)[:, -1]
        assert rel(ex[p], ref) < 1e-5, (p, rel(ex[p], ref))


def test_multislice_dropin_solver_and_farfield():
    w = CONFIG0
    geo = w.geometry()
    dn = w.delta_n()
    probes = w.probes(geo)
    s = MSGpuSolver(geo, probes[None])
    u = s.solve(n=1 + dn)
    assert u.shape == (1, 1, 32, 256, 128)
    ref = po.ms_forward(1 + dn, probes[5], geo.k, 1.0, 1.0)
    assert rel(u[0, 0, 5], ref) < 1e-5
    ff = s.get_farfield_intensities(u, poisson_noise=False)
    assert rel(ff[5], np.abs(np.fft.fft(ref[:, -1])) ** 2) < 1e-5


def test_multislice_adjoint_gradient():
    rng = np.random.default_rng(4)
    N, nz, P, k = 256, 20, 5, 4 * np.pi
    n = 1 + 1e-3 * (rng.standard_normal((N, nz)) + 0.1j * rng.standard_normal((N, nz)))
    x = np.arange(N)
    probes = np.exp(-((x[None] - rng.uniform(60, 200, (P, 1))) ** 2) / 64.0).astype(complex)
    amp = np.abs(np.fft.fft(probes, axis=-1)) * 1.05
    eng = MS2D(N, nz, k, 1.0, 1.0)
    field = torch.from_numpy(n).cuda().requires_grad_(True)
    ex = MSFunction.apply(field, torch.from_numpy(probes.astype(np.complex64)).cuda(), eng)
    loss = torch.sum((torch.fft.fft(ex.to(torch.complex128), dim=-1).abs() - torch.from_numpy(amp).cuda()) ** 2)
    loss.backward()
    g = field.grad.cpu().numpy()

    def oloss(nn):
        e = np.array([po.ms_forward(nn, probes[p], k, 1.0, 1.0)[:, -1] for p in range(P)])
        return po.amplitude_loss_and_grad(e, amp)[0]

    assert abs(loss.item() - oloss(n)) < 1e-5 * oloss(n)
    h = 1e-7
    scale = np.abs(g).max()
    for (xx, t) in [(100, 0), (130, 7), (180, 18), (90, 12), (150, 3)]:
        for d, part in ((1.0, 0), (1j, 1)):
            e = np.zeros_like(n)
            e[xx, t] = h * d
            fd = (oloss(n + e) - oloss(n - e)) / (2 * h)
            an = g[xx, t].real if part == 0 else g[xx, t].imag
            assert abs(fd - an) <= 1e-3 * max(abs(fd), 1e-2 * scale), (xx, t, part, fd, an)
    assert np.all(g[:, -1] == 0)  # the last plane does not enter the multislice model


def test_ms_3pie_against_reference_golden(golden):
    """The multislice 3PIE kernel against ReconstructorMS.reconstruct (1 and 2 epochs).
    Tolerance: complex64 fields and FFTs against the reference's complex128,
    measured relative to the total update ‖n_k − 1‖: ≤ 1e-4 (1 epoch), ≤ 3e-4 (2)."""
    from thick_ptycho_b200.ms2d import ReconstructorMSGpu

    g = golden("ms3pie_ref")
    N, nz = int(g["nx"]), int(g["nz"])
    rec = ReconstructorMSGpu(N, nz, float(g["k"]), float(g["dx"]), float(g["dz"]), g["data"], g["probes"],
                             phase_retrieval=True, n_medium=complex(g["n_medium"]))
    for it, tol in ((1, 1e-4), (2, 3e-4)):
        n, loss = rec.reconstruct(max_iters=it, alpha_obj=0.1)
        ref = g[f"n_{it}"]
        err = np.linalg.norm(n - ref) / np.linalg.norm(ref - 1)
        assert err <= tol, (it, err)
        assert np.allclose(loss, g[f"loss_{it}"], rtol=tol, atol=0), (loss, g[f"loss_{it}"])
