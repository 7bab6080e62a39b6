"""Learned 3D preconditioner end to end: solver-generated pairs, training on the
GPU with the project's own kernels, and what the trained network gains over
the plain FFT preconditioner on a held-out index field.

Tolerances: exit waves of the learned march ≤ 1e-5 relative L2 against the
complex128 oracle (the same bound as the plain BiCGStab march, both at the
default stopping residual); the trained correction must at least halve the
plain preconditioner's error on the held-out field and must not need more
Krylov iterations than the plain form.
"""

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200.cn3d import CN3D, generate_pairs  # noqa: E402
from thick_ptycho_b200.learned import LearnedPreconditioner, default_kappa  # noqa: E402
from thick_ptycho_b200.workloads import ellipsoid_field_3d  # noqa: E402

NF = NB = 32
NZ = 33
K = 4 * np.pi
AMP = 5e-3


def _index(seed):
    dn = ellipsoid_field_3d(NF, NB, NZ, 40, seed, semi=(2.0, 6.0), amplitude=(0.0, AMP), absorption=1e-5)
    return (1 - dn).reshape(NF * NB, NZ)


def _probes(P, seed):
    rng = np.random.default_rng(seed)
    f = np.arange(NF)[None, :]
    b = np.arange(NB)[:, None]
    cs = rng.uniform(10, 22, (P, 2))
    return np.array([np.exp(-((f - cf) ** 2 + (b - cb) ** 2) / 36.0).ravel() for cf, cb in cs]).astype(complex)


@pytest.fixture(scope="module")
def trained():
    eng = CN3D(NF, NB, NZ, K, 1.0, 1.0, 1.0, "impedance")
    P = 6
    pr = torch.from_numpy(_probes(P, 1).astype(np.complex64)).cuda()
    # white-noise pairs teach the correction as an operator (every spatial
    # frequency); pairs of smooth right-hand sides alone give a filter that
    # amplifies the rough Krylov search directions
    noise = generate_pairs(eng, torch.from_numpy(_index(101)).cuda(), pr, every=1, kind="noise")
    model = LearnedPreconditioner(NF, NB, default_kappa(K, 1.0, AMP), seed=0)
    log = model.train(noise, steps=1500, slices_per_batch=4, lr=1e-3, log_every=50)
    return eng, model, log


def test_training_reduces_the_loss(trained):
    _, _, log = trained
    # 1 = the plain preconditioner
    assert log.losses[-1] < 0.05 * log.losses[0], log.losses


def test_trained_correction_beats_plain_on_held_out_field(trained):
    eng, model, _ = trained
    pr = torch.from_numpy(_probes(5, 2).astype(np.complex64)).cuda()
    for kind in ("rhs", "noise"):
        pairs = generate_pairs(eng, torch.from_numpy(_index(202)).cuda(), pr, every=2, kind=kind)
        err = model.relative_error(pairs)
        assert err["learned"] < 0.5 * err["plain"], (kind, err)


@pytest.mark.parametrize("mode", ["forward", "adjoint_exact"])
def test_learned_march_against_oracle_and_iterations(trained, mode):
    eng, model, _ = trained
    n = _index(303)
    P = 4
    probes = _probes(P, 3)
    field = torch.from_numpy(n).cuda()
    co = po.bc_coefficients(K, 1.0, 1.0, dy=1.0, bc_type="impedance", dimension=3)
    A, B = po.step_matrices_2d(NF, NB, co, "impedance", 1.0)
    C = po.object_contribution(n, K, 1.0)
    its = {}
    eng.read_stats()  # drop the counts of earlier marches (pair generation)
    for pc in ("learned", True):
        ex = torch.empty((P, NF * NB), dtype=torch.complex64, device="cuda")
        if mode == "forward":
            eng.march(field, P, "forward", probes=torch.from_numpy(probes.astype(np.complex64)).cuda(), exit_out=ex,
                      precond=pc, model=model)
        else:
            # exit_out of an adjoint march holds the state after the last step: lambda at slice 1
            src = torch.from_numpy(probes.astype(np.complex64)).cuda()
            eng.march(field, P, "adjoint_exact", src_exit=src, exit_out=ex, precond=pc, model=model)
        s = eng.read_stats()
        assert s["failed"] == 0
        its[pc] = s["iterations"]
        got = ex.cpu().numpy().astype(complex)
        for p in range(P):
            if mode == "forward":
                ref = po.march(A, B, C, probes[p])[:, -1]
            else:
                srcm = np.zeros((NF * NB, NZ - 1), dtype=complex)
                srcm[:, -1] = probes[p]
                ref = po.exact_adjoint(A, B, C, srcm)[:, 0]
            assert np.linalg.norm(got[p] - ref) <= 1e-5 * np.linalg.norm(ref), (pc, p, np.linalg.norm(got[p] - ref) / np.linalg.norm(ref))
    assert eng.fallbacks == 0
    assert its["learned"] <= its[True], its


def test_gradient_descent_learned_matches_plain(trained):
    """Config-4-style reconstruction at small size: gradient descent on the 3D
    amplitude loss with the learned preconditioner in the forward and the
    adjoint marches lowers the loss as the plain run does (final losses within
    1 %) and needs no more Krylov iterations.  The trajectories are compared
    at the level the Krylov tolerance allows: at δn = 0 the gradient is a small
    difference of large per-probe terms, and a 1e-6 relative residual per
    solve moves it by ~1.6 % (measured between the plain FFT-preconditioned and
    the unpreconditioned march as well), so after 4 steps the two n differ by
    ~8 % of the total update; the bound is 15 %."""
    from types import SimpleNamespace

    from thick_ptycho_b200 import heads
    from thick_ptycho_b200.cn3d import PWEGradient3D
    from thick_ptycho_b200.reconstruct import gradient_descent_3d

    _, model, _ = trained
    geo = SimpleNamespace(effective_shape=(NF, NB, NZ), nz=NZ, k=K, dx=1.0, dy=1.0, dz=1.0, exact_ref_coeff=False)
    P = 4
    probes = torch.from_numpy(_probes(P, 6).astype(np.complex64)).cuda()
    truth = PWEGradient3D(geo)
    ex = truth.forward(torch.from_numpy(_index(505)).cuda(), probes)
    amp = heads.fft2_last(ex.reshape(P, NF, NB).contiguous()).abs().to(torch.float64)
    n0 = np.ones((NF * NB, NZ), dtype=complex)
    runs = {}
    for pc in (True, "learned"):
        g3 = PWEGradient3D(geo, precond=pc, model=model)
        n, losses, its = gradient_descent_3d(g3, n0, probes, amp, iters=4)
        assert losses[-1] < 0.95 * losses[0], (pc, losses)
        assert g3.engine.fallbacks == 0
        runs[pc] = (n.cpu().numpy(), sum(its), losses[-1])
    assert abs(runs["learned"][2] - runs[True][2]) <= 1e-2 * runs[True][2]
    diff = np.linalg.norm(runs["learned"][0] - runs[True][0]) / np.linalg.norm(runs[True][0] - n0)
    assert diff <= 0.15, diff
    assert runs["learned"][1] <= runs[True][1], (runs["learned"][1], runs[True][1])


def test_learned_filters_reused_by_the_adjoint(trained):
    """The adjoint march reusing the forward march's per-slice filters
    (reuse_filters: the network is not run again for the same field) gives
    the gradient of the march that recomputes them, to fp32 round-off."""
    eng, model, _ = trained
    P = 3
    field = torch.from_numpy(_index(404)).cuda()
    pr = torch.from_numpy(_probes(P, 4).astype(np.complex64)).cuda()
    store = eng.new_store(P)
    ex = torch.empty((P, NF * NB), dtype=torch.complex64, device="cuda")
    eng.march(field, P, "forward", probes=pr, u_store=store, exit_out=ex, precond="learned", model=model)
    grads = []
    for reuse in (True, False):
        gc = torch.zeros((NZ - 1, NF * NB), dtype=torch.complex64, device="cuda")
        eng.march(field, P, "adjoint_exact", src_exit=ex, u_fwd=store, grad_c=gc, precond="learned", model=model,
                  reuse_filters=reuse)
        grads.append(gc.cpu().numpy())
    assert eng.fallbacks == 0
    assert np.linalg.norm(grads[0] - grads[1]) <= 1e-6 * np.linalg.norm(grads[1])
