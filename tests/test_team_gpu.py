"""GPU parity of the team path (N in {512, 1024, 2048}: 128 chunks, several
probes per thread) against the complex128 oracle: every boundary condition
and mode, groups of 1 and 4 probes per CTA with a partial last group, and
the fused exact-adjoint gradient summed over hundreds of probes.

Tolerances as in the other GPU tests: relative L2 ≤ 1e-5 for fields and for
the fp32-summed gradient.
"""

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200.cn2d import CN2D  # noqa: E402

TOL = 1e-5
GRAD_TOL = 1e-5
K, DX, DZ = 4 * np.pi, 1.0, 1.0


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _field(N, nz, seed):
    rng = np.random.default_rng(seed)
    return 1 + 1e-3 * (rng.standard_normal((N, nz)) + 0.1j * rng.standard_normal((N, nz)))


def _probes(N, P, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(N)[None]
    c = rng.uniform(0.1 * N, 0.9 * N, (P, 1))
    return (np.exp(-((x - c) ** 2) / 64.0) * np.exp(1j * rng.uniform(0, 6.28, (P, 1)))).astype(complex)


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet", "impedance2"])
def test_team_modes_against_oracle(bc):
    N, nz, P = 512, 33, 3
    n = _field(N, nz, 1)
    probes = _probes(N, P, 2)
    eng = CN2D(N, nz, K, DX, DZ, bc)
    assert eng.chunks == 128
    co = po.bc_coefficients(K, DX, DZ, bc_type=bc)
    A, B = po.step_matrices_1d(N, co, bc, DZ)
    C = po.object_contribution(n, K, DZ)
    field = torch.from_numpy(n).cuda()
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal((P, N, nz - 1)) + 1j * rng.standard_normal((P, N, nz - 1))
    src = torch.from_numpy(np.ascontiguousarray(rhs.transpose(0, 2, 1)).astype(np.complex64)).cuda()
    for mode, use_probe, use_src in (("forward", True, False), ("forward", True, True), ("adjoint", False, True),
                                     ("reverse", True, False), ("adjoint", True, False)):
        fs = eng.factor(field, mode)
        st = eng.new_store(P)
        eng.march(fs, P, probes=pr if use_probe else None, src_probe=src if use_src else None, u_store=st)
        eng.device_status()
        got = eng.unchunk(st).cpu().numpy()
        for p in range(P):
            ref = po.march(A, B, C, probes[p] if use_probe else None, mode, rhs_block=rhs[p] if use_src else None)
            assert rel(got[p], ref) < TOL, (bc, mode, p, rel(got[p], ref))


def test_team_groups_of_four_with_partial_group_and_gradient():
    N, nz, P = 1024, 24, 457  # 115 CTAs of 4 probes, the last one partial
    n = _field(N, nz, 5)
    probes = _probes(N, P, 6)
    eng = CN2D(N, nz, K, DX, DZ, "impedance")
    co = po.bc_coefficients(K, DX, DZ, bc_type="impedance")
    A, B = po.step_matrices_1d(N, co, "impedance", DZ)
    C = po.object_contribution(n, K, DZ)
    field = torch.from_numpy(n).cuda()
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    st = eng.new_store(P)
    ex = torch.empty((P, N), dtype=torch.complex64, device="cuda")
    eng.march(eng.factor(field, "forward"), P, probes=pr, u_store=st, exit_out=ex)
    # exit-wave source for the adjoint: a fixed random field per probe
    rng = np.random.default_rng(7)
    e = (rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))).astype(np.complex64)
    gc = eng.new_grad_buffer()
    eng.march(eng.factor(field, "adjoint_exact"), P, src_exit=torch.from_numpy(e).cuda(), u_fwd=st, grad_c=gc)
    eng.device_status()
    lus, Bs = po.build_lu_factors(A, B, C)
    u_ref = np.array([po.march_with_lu(lus, Bs, np.zeros(N, complex), probes[p]) for p in range(P)])
    assert rel(ex.cpu().numpy(), u_ref[:, :, -1]) < TOL
    assert rel(eng.unchunk(st).cpu().numpy()[[0, 228, 456]], u_ref[[0, 228, 456]]) < TOL
    srcs = np.zeros((P, N, nz - 1), dtype=complex)
    srcs[:, :, -1] = e
    lam = po.exact_adjoint_many(A, B, C, srcs)
    gref = sum(po.grad_c_from_adjoint(u_ref[p], lam[p]) for p in range(P))
    got = eng.unchunk_rows(gc).cpu().numpy().T
    assert rel(got, gref) < GRAD_TOL, rel(got, gref)
    # the same with stored half pair sums and the Cayley-form adjoint: staged
    # half-sum loads and the CTA sum of the teams' contributions, the last
    # CTA holding one probe and three padded teams
    sums, gs = eng.new_store(P), eng.new_grad_buffer()
    eng.march(eng.factor(field, "forward"), P, probes=pr, u_store=sums, store_sums=True)
    eng.march(eng.factor(field, "adjoint_exact"), P, src_exit=torch.from_numpy(e).cuda(), u_fwd=sums, grad_c=gs,
              store_sums=True)
    eng.device_status()
    got_s = eng.unchunk_rows(gs).cpu().numpy().T
    assert rel(got_s, gref) < GRAD_TOL, rel(got_s, gref)


@pytest.mark.parametrize("N,k", [(512, K), (1024, K), (2048, K), (2048, 0.5)])
def test_team_pair_sums_store_and_cayley_adjoint(N, k):
    """store_sums: the forward store holds (u_t + u_{t-1})/2; the exact adjoint
    reading those sums (one slice per step, Cayley-form step) gives the same
    lambda and gradient as the two-slice form and as the oracle.  N = 512
    (4-row chunks) keeps parallel cyclic reduction; N = 2048 at
    k = 4 pi keeps 8 spike rows (the shared-memory staged bulk stores, bulk
    half-sum loads and CTA gradient accumulator); k = 0.5 couples the chunks
    strongly (all 15 spike rows, parallel cyclic reduction), where the staging
    does not fit and the direct per-thread path runs."""
    from thick_ptycho_b200._native import NativeLibraryError

    nz, P = 24, 9
    n = _field(N, nz, 11)
    probes = _probes(N, P, 12)
    eng = CN2D(N, nz, k, DX, DZ, "impedance")
    co = po.bc_coefficients(k, DX, DZ, bc_type="impedance")
    A, B = po.step_matrices_1d(N, co, "impedance", DZ)
    C = po.object_contribution(n, k, DZ)
    field = torch.from_numpy(n).cuda()
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    ff = eng.factor(field, "forward")
    st, sums = eng.new_store(P), eng.new_store(P)
    eng.march(ff, P, probes=pr, u_store=st)
    eng.march(ff, P, probes=pr, u_store=sums, store_sums=True)
    eng.device_status()
    u = eng.unchunk(st).cpu().numpy()
    w = eng.unchunk(sums).cpu().numpy()
    assert rel(w[:, :, 1:], 0.5 * (u[:, :, 1:] + u[:, :, :-1])) < 1e-6
    rng = np.random.default_rng(13)
    e = torch.from_numpy((rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))).astype(np.complex64)).cuda()
    fa = eng.factor(field, "adjoint_exact")
    g1, g2 = eng.new_grad_buffer(), eng.new_grad_buffer()
    s1 = torch.empty((P, eng.npad), dtype=torch.complex64, device="cuda")
    s2 = torch.empty_like(s1)
    eng.march(fa, P, src_exit=e, u_fwd=st, grad_c=g1, state_out=s1)
    eng.march(fa, P, src_exit=e, u_fwd=sums, grad_c=g2, state_out=s2, store_sums=True)
    eng.device_status()
    assert rel(s2.cpu().numpy(), s1.cpu().numpy()) < TOL
    got = eng.unchunk_rows(g2).cpu().numpy().T
    assert rel(got, eng.unchunk_rows(g1).cpu().numpy().T) < TOL
    lus, Bs = po.build_lu_factors(A, B, C)
    u_ref = np.array([po.march_with_lu(lus, Bs, np.zeros(N, complex), probes[p]) for p in range(P)])
    srcs = np.zeros((P, N, nz - 1), dtype=complex)
    srcs[:, :, -1] = e.cpu().numpy()
    lam = po.exact_adjoint_many(A, B, C, srcs)
    gref = sum(po.grad_c_from_adjoint(u_ref[p], lam[p]) for p in range(P))
    assert rel(got, gref) < GRAD_TOL, rel(got, gref)
    # exact adjoint without a gradient (Cayley step): the stored lambda
    # (index t holds slice L+1-t) against the oracle
    lam_st = eng.new_store(P)
    eng.march(fa, P, src_exit=e, u_store=lam_st)
    eng.device_status()
    lg = eng.unchunk(lam_st).cpu().numpy()
    for p in range(P):
        assert rel(lg[p][:, 1:][:, ::-1], lam[p]) < TOL, (p, rel(lg[p][:, 1:][:, ::-1], lam[p]))
    # checkpoint stores keep states; the warp path (N = 256) has no pair sums
    with pytest.raises(NativeLibraryError):
        eng.march(ff, P, probes=pr, u_store=eng.new_store(P, 4), store_every=8, store_sums=True)
    small = CN2D(256, nz, k, DX, DZ, "impedance")
    with pytest.raises(NativeLibraryError):
        small.march(small.factor(torch.from_numpy(n[:256]).cuda(), "forward"), 1, u_store=small.new_store(1),
                    store_sums=True)


def test_team_rejects_misaligned_slice_buffers():
    """The team kernels move whole slices with 16-byte vectors and bulk copies:
    a store buffer 8 bytes off a 16-byte boundary is refused on the host
    (nothing is launched), and the aligned buffer works."""
    from thick_ptycho_b200._native import NativeLibraryError

    N, nz, P = 512, 12, 3
    eng = CN2D(N, nz, K, DX, DZ, "impedance")
    field = torch.from_numpy(_field(N, nz, 21)).cuda()
    pr = torch.from_numpy(_probes(N, P, 22).astype(np.complex64)).cuda()
    fs = eng.factor(field, "forward")
    st = eng.new_store(P)
    flat = torch.empty(st.numel() + 1, dtype=torch.complex64, device="cuda")
    off = flat[1:].view(st.shape)  # 8 bytes past the allocation's 256-byte boundary
    assert off.data_ptr() % 16 == 8
    with pytest.raises(NativeLibraryError, match="16-byte aligned"):
        eng.march(fs, P, probes=pr, u_store=off)
    eng.march(fs, P, probes=pr, u_store=st)
    eng.device_status()
