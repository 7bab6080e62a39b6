"""The GPU solver plugged into the unmodified reference.

When the reference package is installed in ``baseline/_ref`` (``pip install
--target baseline/_ref`` of the reference checkout; its two display-only
imports, matplotlib and scikit-image, are satisfied by the stub packages in
``tests/golden/refstubs``), this builds the reference's own simulation space
and probes and checks that ``PWEGpuSolver``

* takes them unchanged and reproduces ``PWEIterativeLUSolver``'s ``solve``,
  its adjoint ``_solve_single_probe`` with a right-hand side, its
  ``get_gradient`` operator and its far-field intensities;
* serves as ``ReconstructorPWE.forward_model``: two iterations of the
  reference's own NLCG ``reconstruct`` (``pwe_reconstructor.py:229-368``)
  with the GPU solver swapped in land where the unmodified run lands.

Tolerances: fields and intensities ≤ 1e-5 relative L2 (complex64 against the
reference's complex128); the reconstructed n relative to the total update
‖n_k − n_0‖ ≤ 1e-4 after one iteration and ≤ 2e-3 after two (as for the
committed NLCG golden vectors: the reference's first step is large, so the
second iteration amplifies the first one's round-off).
"""

import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")
STUBS = os.path.join(ROOT, "tests", "golden", "refstubs")

TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def ref():
    if not os.path.isdir(os.path.join(REF, "thick_ptycho")):
        pytest.skip("the reference package is not installed in baseline/_ref")
    for p in (REF, STUBS):
        if p not in sys.path:
            sys.path.insert(0, p)
    import thick_ptycho.forward_model as fm
    import thick_ptycho.reconstruction as rc
    import thick_ptycho.simulation.config as cfg
    import thick_ptycho.simulation.ptycho_probe as pp
    import thick_ptycho.simulation.scan_frame as sf
    import thick_ptycho.simulation.simulation_space as spc

    return {"fm": fm, "rc": rc, "cfg": cfg, "pp": pp, "sf": sf, "spc": spc}


def _space(ref, nz):
    cfg = ref["cfg"]
    c = cfg.SimulationConfig(
        probe_config=cfg.ProbeConfig(type=cfg.ProbeType.GAUSSIAN, wave_length=0.5, diameter=12.0),
        scan_points=4, step_size_px=7, pad_factor=1.2, nz=nz,
        spatial_limits=ref["sf"].Limits(x=(0.0, 33.0), z=(0.0, float(nz - 1)), units="meters"),
        use_logging=False,
    )
    return ref["spc"].create_simulation_space(c)


def test_gpu_solver_takes_the_reference_objects(ref):
    from thick_ptycho_b200.solver import PWEGpuSolver

    ss = _space(ref, 24)
    probes = ref["pp"].create_ptycho_probes(ss)
    rng = np.random.default_rng(11)
    n = 1 + 2e-3 * (rng.standard_normal((ss.nx, ss.nz)) + 0.1j * rng.standard_normal((ss.nx, ss.nz)))
    cpu = ref["fm"].PWEIterativeLUSolver(ss, probes, bc_type="impedance")
    gpu = PWEGpuSolver(ss, probes, bc_type="impedance")
    u_ref = cpu.solve(n=n)
    u = gpu.solve(n=n)
    assert u.shape == u_ref.shape
    assert rel(u, u_ref) < TOL, rel(u, u_ref)
    rhs = rng.standard_normal((ss.block_size, ss.nz - 1)) + 1j * rng.standard_normal((ss.block_size, ss.nz - 1))
    cpu.reset_cache()
    a_ref = cpu._solve_single_probe(scan_idx=1, n=n, mode="adjoint", rhs_block=rhs, probe=None)
    a = gpu._solve_single_probe(scan_idx=1, n=n, mode="adjoint", rhs_block=rhs, probe=None)
    assert rel(a, a_ref) < TOL, rel(a, a_ref)
    g_ref, g = cpu.get_gradient(n=n), gpu.get_gradient(n=n)
    assert g.shape == g_ref.shape
    assert abs((g - g_ref).tocsr()).max() <= 1e-12 * abs(g_ref.tocsr()).max()
    ff_ref = cpu.get_farfield_intensities(u_ref, poisson_noise=False)
    ff = gpu.get_farfield_intensities(u, poisson_noise=False)
    assert rel(ff, ff_ref) < TOL, rel(ff, ff_ref)


def test_reference_nlcg_with_the_gpu_forward_model(ref):
    from thick_ptycho_b200.solver import PWEGpuSolver

    ss = _space(ref, 16)
    probes = ref["pp"].create_ptycho_probes(ss)
    rng = np.random.default_rng(2024)
    n_true = 1 + 1e-3 * (rng.standard_normal((ss.nx, ss.nz)) + 0.05j * np.abs(rng.standard_normal((ss.nx, ss.nz))))
    fwd = ref["fm"].PWEIterativeLUSolver(ss, probes, bc_type="impedance")
    data = fwd.get_farfield_intensities(fwd.solve(n=n_true), poisson_noise=False)
    n0 = (1 + 2e-4 * rng.standard_normal((ss.nx, ss.nz))).astype(complex)
    for iters, tol in ((1, 1e-4), (2, 2e-3)):
        runs = {}
        for name in ("reference", "gpu"):
            rec = ref["rc"].ReconstructorPWE(ss, data, phase_retrieval=True, solver_type="iterative",
                                             bc_type="impedance", verbose=False)
            if name == "gpu":
                rec.forward_model = PWEGpuSolver(ss, rec.ptycho_probes, bc_type="impedance")
            nk, _, residual = rec.reconstruct(max_iters=iters, n_initial=n0.copy())
            runs[name] = (np.asarray(nk), np.asarray(residual))
        err = np.linalg.norm(runs["gpu"][0] - runs["reference"][0]) / np.linalg.norm(runs["reference"][0] - n0)
        assert err <= tol, (iters, err)
        assert np.allclose(runs["gpu"][1], runs["reference"][1], rtol=tol, atol=0)
