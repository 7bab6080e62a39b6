"""GPU parity of the 2D Crank–Nicolson path (libtpcuda) against the reference
golden vectors and the complex128 oracle.

Tolerances (complex64 arithmetic with fp64 factorisation): relative L2 error
≤ 1e-5 against complex128 results (the target stated for the complex64
form); bit-exact where the result is an index or must not depend on the
batch composition.
"""

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200 import PWEGpuSolver, SimulationGeometry  # noqa: E402
from thick_ptycho_b200.cn2d import CN2D  # noqa: E402
from thick_ptycho_b200.workloads import CONFIG0, CONFIG1  # noqa: E402

TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


class _TestBCs:
    """Carries precomputed exact boundary data in the reference's interface."""

    def __init__(self, rows):
        self.rows = rows

    def test_exact_impedance_rhs_step(self, j):
        return self.rows[j - 1]


def geometry_from(g, prefix="", num_probes=1, **kw):
    return SimulationGeometry(dimension=2, nx=int(g[prefix + "nx"]), nz=int(g[prefix + "nz"]), dx=float(g[prefix + "dx"]),
                              dz=float(g[prefix + "dz"]), k=float(g[prefix + "k"]), num_probes=num_probes, **kw)


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet"])
def test_kat2d_against_reference(golden, bc):
    g = golden("kat2d")
    errs = []
    for nx in (16, 32, 64):
        key = f"{bc}_{nx}_"
        geo = geometry_from(g, key)
        tb = _TestBCs(g[key + "test_rhs"]) if bc == "impedance" else None
        probes = g[key + "probe"][None, None]
        solver = PWEGpuSolver(geo, probes, bc_type=bc, test_bcs=tb)
        u = solver.solve().squeeze()
        assert rel(u, g[key + "u"]) < TOL, (bc, nx, rel(u, g[key + "u"]))
        X, Z = np.meshgrid(g[key + "x"], g[key + "z"], indexing="ij")
        a = 1j / (2 * float(g[key + "k"]))
        if bc == "dirichlet":
            ex = sum(c * np.exp(-a * m * m * np.pi**2 * Z) * np.sin(m * np.pi * X) for c, m in ((1, 1), (0.5, 5), (0.2, 9)))
        else:
            ex = sum(c * np.exp(-a * m * m * np.pi**2 * Z) * np.cos(m * np.pi * X) for c, m in ((1, 1), (0.5, 2), (0.2, 5)))
        errs.append(np.max(np.abs(u - ex)))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert all(errs[i] < errs[i - 1] for i in range(1, 3)), errs
    assert 1.5 <= np.mean(rates) <= 2.5, rates


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet", "impedance2"])
def test_random2d_modes_against_reference(golden, bc):
    g = golden("random2d")
    geo = geometry_from(g, num_probes=4)
    probes = g["probes"][None]
    s = PWEGpuSolver(geo, probes, bc_type=bc)
    n = g["n"]
    u = s.solve(n=n)[0, 0]
    assert rel(u, g[f"{bc}_forward"]) < TOL
    rhs = g["rhs_block"]
    lam = s._solve_single_probe(scan_idx=1, n=n, mode="adjoint", rhs_block=rhs, probe=None)
    assert rel(lam, g[f"{bc}_adjoint"]) < TOL
    r = s._solve_single_probe(scan_idx=2, n=n, mode="reverse", probe=probes[0, 2])
    assert rel(r, g[f"{bc}_reverse"]) < TOL
    f = s._solve_single_probe(scan_idx=3, n=n, mode="forward", rhs_block=rhs, probe=probes[0, 3])
    assert rel(f, g[f"{bc}_forward_src"]) < TOL


def test_exact_coeff_and_padding_against_reference(golden):
    g = golden("random2d")
    geo = geometry_from(g, num_probes=4, exact_ref_coeff=True)
    u = PWEGpuSolver(geo, g["probes"][None], bc_type="impedance").solve(n=g["n"])[0, 0]
    assert rel(u, g["exact_forward"]) < TOL
    e = (int(g["pad_block_size"]) - int(g["nx"])) // 2
    geo2 = geometry_from(g, num_probes=4, empty_space_px=e)
    assert geo2.block_size == int(g["pad_block_size"])
    u2 = PWEGpuSolver(geo2, g["pad_probes"][None], bc_type="impedance").solve(n=g["n"])[0, 0]
    assert rel(u2, g["pad_forward"]) < TOL


def test_config0_reference_geometry_exit_and_farfield(golden):
    """N = 257 (ragged rows), 32 probes: exit waves and |FFT|² vs the reference."""
    g = golden("config0_ref")
    geo = geometry_from(g, num_probes=32)
    s = PWEGpuSolver(geo, g["probes"][None], bc_type="impedance")
    u = s.solve(n=1 - g["delta_n"])
    ex = s.get_exit_waves(u)
    assert rel(ex, g["exit"]) < TOL
    assert rel(u[0, 0, 0][:, ::8], g["u_p0"]) < TOL
    assert rel(u[0, 0, 31][:, ::8], g["u_p31"]) < TOL
    ff = s.get_farfield_intensities(exit_waves=ex, poisson_noise=False)
    assert rel(ff, g["farfield"]) < 2 * TOL


def test_config0_exact_size_against_oracle():
    """N = 256, Nz = 128, 32 probes (the CPU-runnable configuration)."""
    w = CONFIG0
    geo = w.geometry()
    dn = w.delta_n()
    probes = w.probes(geo)
    s = PWEGpuSolver(geo, probes[None], bc_type="impedance")
    ex = s.get_exit_waves(s.solve(n=1 - dn))
    co = po.bc_coefficients(geo.k, 1.0, 1.0, bc_type="impedance")
    A, B = po.step_matrices_1d(256, co, "impedance", 1.0)
    lus, Bs = po.build_lu_factors(A, B, po.object_contribution(1 - dn, geo.k, 1.0))
    ref = np.array([po.march_with_lu(lus, Bs, np.zeros(256, complex), probes[p])[:, -1] for p in range(32)])
    assert rel(ex, ref) < TOL
    assert rel(np.abs(np.fft.fft(ex)) ** 2, np.abs(np.fft.fft(ref)) ** 2) < 2 * TOL


def test_config1_full_size_subset_against_oracle():
    """N = 2048, Nz = 1024, all 512 probes on the GPU; 3 of them checked in complex128."""
    w = CONFIG1
    geo = w.geometry()
    dn = w.delta_n()
    probes = w.probes(geo)
    eng = CN2D(2048, 1024, geo.k, 1.0, 1.0, "impedance")
    field = torch.from_numpy(1 - dn).cuda()
    fs = eng.factor(field, "forward")
    pr = torch.from_numpy(probes.astype(np.complex64)).cuda()
    ex = torch.empty((512, 2048), dtype=torch.complex64, device="cuda")
    eng.march(fs, 512, probes=pr, exit_out=ex)
    eng.device_status()
    ex = ex.cpu().numpy()
    co = po.bc_coefficients(geo.k, 1.0, 1.0, bc_type="impedance")
    A, B = po.step_matrices_1d(2048, co, "impedance", 1.0)
    lus, Bs = po.build_lu_factors(A, B, po.object_contribution(1 - dn, geo.k, 1.0))
    for p in (0, 255, 511):
        ref = po.march_with_lu(lus, Bs, np.zeros(2048, complex), probes[p])[:, -1]
        assert rel(ex[p], ref) < TOL, (p, rel(ex[p], ref))


def test_batch_composition_and_linearity():
    """A probe's result is identical whatever the batch around it (scan order
    exact), and the march is linear in the probe."""
    w = CONFIG0
    geo = w.geometry()
    dn = w.delta_n()
    probes = w.probes(geo).astype(np.complex64)
    eng = CN2D(256, 128, geo.k, 1.0, 1.0, "impedance")
    fs = eng.factor(torch.from_numpy(1 - dn).cuda(), "forward")
    pr = torch.from_numpy(probes).cuda()
    full = torch.empty((32, 256), dtype=torch.complex64, device="cuda")
    eng.march(fs, 32, probes=pr, exit_out=full)
    perm = torch.randperm(32, generator=torch.Generator().manual_seed(0))
    sub = torch.empty((32, 256), dtype=torch.complex64, device="cuda")
    eng.march(fs, 32, probes=pr[perm.cuda()].contiguous(), exit_out=sub)
    assert torch.equal(sub, full[perm.cuda()])
    one = torch.empty((1, 256), dtype=torch.complex64, device="cuda")
    eng.march(fs, 1, probes=pr[7:8].contiguous(), exit_out=one)
    assert torch.equal(one[0], full[7])
    a, b = 0.3 - 0.2j, -1.1 + 0.5j
    comb = (a * pr[3] + b * pr[11])[None].contiguous()
    eng.march(fs, 1, probes=comb, exit_out=one)
    expect = a * full[3] + b * full[11]
    assert (torch.linalg.norm(one[0] - expect) / torch.linalg.norm(expect)).item() < 1e-5


def test_full_field_store_matches_exit():
    w = CONFIG0
    geo = w.geometry()
    probes = w.probes(geo).astype(np.complex64)
    eng = CN2D(256, 128, geo.k, 1.0, 1.0, "neumann")
    fs = eng.factor(torch.from_numpy(1 - w.delta_n()).cuda(), "forward")
    pr = torch.from_numpy(probes).cuda()
    st = eng.new_store(32)
    ex = torch.empty((32, 256), dtype=torch.complex64, device="cuda")
    eng.march(fs, 32, probes=pr, u_store=st, exit_out=ex)
    u = eng.unchunk(st)
    assert torch.equal(u[..., -1], ex)
    assert torch.equal(u[..., 0], pr)
