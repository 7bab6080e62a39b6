"""Generate the golden fixtures from the unmodified reference implementation.

Run in a container that holds the reference checkout (read-only) at
``REF`` below::

    python tests/golden/make_golden.py [/path/to/reference [section ...]]

With section names (the function names below) only those fixtures are
regenerated.

The reference is imported as-is; its two display-only imports (matplotlib,
scikit-image) are satisfied by the stub packages in ``tests/golden/refstubs``.
The fixtures are small ``.npz`` files committed next to this script; tests on
machines without the reference read only those files.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
sys.path.insert(0, os.path.join(HERE, "refstubs"))
sys.path.insert(1, REF)
sys.path.insert(2, os.path.dirname(os.path.dirname(HERE)))

from thick_ptycho.forward_model import MSForwardModelSolver, PWEFullLUSolver, PWEIterativeLUSolver  # noqa: E402
from thick_ptycho.forward_model.pwe.operators.finite_differences.boundary_condition_test import (  # noqa: E402
    BoundaryConditionsTest,
)
from thick_ptycho.reconstruction import ReconstructorPWE  # noqa: E402
from thick_ptycho.simulation.config import ProbeConfig, ProbeType, SimulationConfig  # noqa: E402
from thick_ptycho.simulation.ptycho_probe import create_ptycho_probes  # noqa: E402
from thick_ptycho.simulation.scan_frame import Limits, ScanPath  # noqa: E402
from thick_ptycho.simulation.simulation_space import create_simulation_space  # noqa: E402

from thick_ptycho_b200.workloads import CONFIG0, blob_field_2d, gaussian_probes_2d  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}.npz ({os.path.getsize(path) / 1024:.1f} KiB)")


def sim_params(ss):
    out = dict(
        nx=ss.nx, nz=ss.nz, dx=float(ss.dx), dz=float(ss.dz), k=float(ss.k),
        block_size=ss.block_size, num_probes=ss.num_probes,
    )
    if ss.dimension == 3:
        out["dy"] = float(ss.dy)
    return out


# ---------------------------------------------------------------------------
# 1. Known-answer convergence cases (test_boundary_conditions_2d.py:146-183)
# ---------------------------------------------------------------------------
def kat_2d():
    k = 100
    limits = Limits(x=(0, 1), z=(0, 2), units="meters")
    out = {}
    for bc, ptype in (("neumann", ProbeType.NEUMANN_TEST), ("impedance", ProbeType.NEUMANN_TEST),
                      ("dirichlet", ProbeType.DIRICHLET_TEST)):
        for nx in (16, 32, 64):
            cfg = SimulationConfig(probe_config=ProbeConfig(type=ptype, wave_length=2 * np.pi / k),
                                   step_size_px=nx, nz=nx, spatial_limits=limits)
            ss = create_simulation_space(cfg)
            probes = create_ptycho_probes(ss)
            tb = BoundaryConditionsTest(ss) if bc == "impedance" else None
            solver = PWEIterativeLUSolver(ss, probes, bc_type=bc, test_bcs=tb)
            u = solver.solve().squeeze()
            key = f"{bc}_{nx}"
            out[key + "_u"] = u
            out[key + "_probe"] = probes[0, 0]
            if tb is not None:
                out[key + "_test_rhs"] = np.stack([tb.test_exact_impedance_rhs_step(j) for j in range(1, ss.nz)])
            for kk, v in sim_params(ss).items():
                out[key + "_" + kk] = v
            out[key + "_x"] = np.linspace(0, 1, ss.nx)
            out[key + "_z"] = ss.z
    save("kat2d", **out)


def kat_3d():
    k = 100
    limits = Limits(x=(0, 1), y=(0, 1), z=(0, 2), units="meters")
    out = {}
    for bc, ptype in (("neumann", ProbeType.NEUMANN_TEST), ("impedance", ProbeType.NEUMANN_TEST),
                      ("dirichlet", ProbeType.DIRICHLET_TEST)):
        for nx in (8, 16):
            cfg = SimulationConfig(probe_config=ProbeConfig(type=ptype, wave_length=2 * np.pi / k),
                                   step_size_px=nx, nz=nx, spatial_limits=limits, solve_reduced_domain=False)
            ss = create_simulation_space(cfg)
            probes = create_ptycho_probes(ss)
            tb = BoundaryConditionsTest(ss) if bc == "impedance" else None
            solver = PWEIterativeLUSolver(ss, probes, bc_type=bc, test_bcs=tb)
            u = solver.solve().squeeze()
            key = f"{bc}_{nx}"
            out[key + "_u"] = u
            out[key + "_probe"] = probes[0, 0]
            if tb is not None:
                out[key + "_test_rhs"] = np.stack([tb.test_exact_impedance_rhs_step(j) for j in range(1, ss.nz)])
            if nx == 8:
                fl = PWEFullLUSolver(ss, probes, bc_type=bc, test_bcs=tb).solve().squeeze()
                out[key + "_fulllu_u"] = fl
            for kk, v in sim_params(ss).items():
                out[key + "_" + kk] = v
    save("kat3d", **out)


# ---------------------------------------------------------------------------
# 2. Random small 2D cases: every BC, every mode, exact_ref_coeff, padding
# ---------------------------------------------------------------------------
def small_space_2d(nz=24, exact_ref_coeff=False, empty_space_px=0):
    cfg = SimulationConfig(
        probe_config=ProbeConfig(type=ProbeType.GAUSSIAN, wave_length=0.5, diameter=12.0),
        scan_points=4, step_size_px=7, pad_factor=1.2, nz=nz,
        spatial_limits=Limits(x=(0.0, 33.0), z=(0.0, float(nz - 1)), units="meters"),
        exact_ref_coeff=exact_ref_coeff, empty_space_px=empty_space_px, use_logging=False,
    )
    return create_simulation_space(cfg)


def random_2d():
    rng = np.random.default_rng(1234)
    out = {}
    ss = small_space_2d()
    assert ss.nx == 34, ss.nx
    probes = create_ptycho_probes(ss)
    n = 1 + 2e-3 * (rng.standard_normal((ss.nx, ss.nz)) + 1j * 0.1 * rng.standard_normal((ss.nx, ss.nz)))
    out["n"] = n
    out["probes"] = probes[0]
    for kk, v in sim_params(ss).items():
        out[kk] = v
    rhs = rng.standard_normal((ss.block_size, ss.nz - 1)) + 1j * rng.standard_normal((ss.block_size, ss.nz - 1))
    out["rhs_block"] = rhs
    for bc in ("neumann", "impedance", "dirichlet", "impedance2"):
        solver = PWEIterativeLUSolver(ss, probes, bc_type=bc)
        out[f"{bc}_forward"] = solver.solve(n=n)[0, 0]
        solver.reset_cache()
        out[f"{bc}_adjoint"] = solver._solve_single_probe(scan_idx=1, n=n, mode="adjoint", rhs_block=rhs, probe=None)
        solver.reset_cache()
        out[f"{bc}_reverse"] = solver._solve_single_probe(scan_idx=2, n=n, mode="reverse", probe=probes[0, 2])
        solver.reset_cache()
        out[f"{bc}_forward_src"] = solver._solve_single_probe(scan_idx=3, n=n, mode="forward", rhs_block=rhs,
                                                              probe=probes[0, 3])
        full = PWEFullLUSolver(ss, probes, bc_type=bc)
        out[f"{bc}_fulllu"] = full.solve(n=n)[0, 0]
    # exact_ref_coeff and transverse zero padding
    ss2 = small_space_2d(exact_ref_coeff=True)
    out["exact_forward"] = PWEIterativeLUSolver(ss2, probes, bc_type="impedance").solve(n=n)[0, 0]
    ss3 = small_space_2d(empty_space_px=5)
    probes3 = create_ptycho_probes(ss3)
    out["pad_probes"] = probes3[0]
    out["pad_block_size"] = ss3.block_size
    out["pad_forward"] = PWEIterativeLUSolver(ss3, probes3, bc_type="impedance").solve(n=n)[0, 0]
    # multislice with the same n (reference MS convention n = 1 + δn)
    ms = MSForwardModelSolver(ss, probes)
    out["ms_forward"] = ms.solve(n=n)[0, 0]
    # step operator rows for the 4 BCs
    save("random2d", **out)


# ---------------------------------------------------------------------------
# 3. Config-0 geometry through the reference (N = 257: the reference's parity
#    rule makes an even stride produce an odd width)
# ---------------------------------------------------------------------------
def config0_reference():
    nz = CONFIG0.nz
    cfg = SimulationConfig(
        probe_config=ProbeConfig(type=ProbeType.GAUSSIAN, wave_length=CONFIG0.wave_length, diameter=16.0),
        scan_points=CONFIG0.scan_points, step_size_px=CONFIG0.step, pad_factor=4.0 / 3.0, nz=nz,
        spatial_limits=Limits(x=(0.0, 256.0), z=(0.0, float(nz - 1)), units="meters"), use_logging=False,
    )
    ss = create_simulation_space(cfg)
    assert ss.nx == 257 and abs(ss.dx - 1) < 1e-12 and abs(ss.dz - 1) < 1e-12, (ss.nx, ss.dx, ss.dz)
    centres = [f.probe_centre_discrete.x for f in ss.scan_frame_info]
    dn = blob_field_2d(ss.nx, nz, CONFIG0.n_shapes, CONFIG0.seed)
    probes = gaussian_probes_2d(ss.nx, centres, CONFIG0.waist)[None]
    solver = PWEIterativeLUSolver(ss, probes, bc_type="impedance")
    u = solver.solve(n=1 - dn, probes=probes)
    exit_w = solver.get_exit_waves(u)
    ff = solver.get_farfield_intensities(exit_waves=exit_w, poisson_noise=False)
    ms = MSForwardModelSolver(ss, probes)
    u_ms = ms.solve(n=1 + dn, probes=probes)
    save("config0_ref", delta_n=dn, probes=probes[0], centres=np.array(centres), exit=exit_w, farfield=ff,
         u_p0=u[0, 0, 0][:, ::8], u_p31=u[0, 0, 31][:, ::8], ms_exit=ms.get_exit_waves(u_ms),
         **sim_params(ss))


# ---------------------------------------------------------------------------
# 4. Reference least-squares gradient (pwe_reconstructor.py:100-164)
# ---------------------------------------------------------------------------
def gradient_reference():
    ss = small_space_2d(nz=16)
    rng = np.random.default_rng(99)
    probes = create_ptycho_probes(ss)
    n_true = 1 + 1e-3 * (rng.standard_normal((ss.nx, ss.nz)) + 0.05j * np.abs(rng.standard_normal((ss.nx, ss.nz))))
    fwd = PWEIterativeLUSolver(ss, probes, bc_type="impedance")
    data = fwd.get_farfield_intensities(fwd.solve(n=n_true), poisson_noise=False)
    rec = ReconstructorPWE(ss, data, phase_retrieval=True, solver_type="iterative", bc_type="impedance",
                           verbose=False)
    n0 = 1 + 5e-4 * (rng.standard_normal((ss.nx, ss.nz)))
    rec.nk = n0.astype(complex)
    uk = rec.compute_forward_model(probes=rec.forward_model.probes)
    err = rec.get_error_in_exit_wave(uk)
    grad_A = -rec.forward_model.get_gradient(n=rec.nk)
    gre, gim = rec.compute_grad_least_squares(err, uk, grad_A)
    save("gradient_ref", n=rec.nk, data=data, probes=rec.ptycho_probes[0], uk=uk,
         exit_error=err[0, 0][..., -1], grad_re=gre, grad_im=gim, **sim_params(ss))


# ---------------------------------------------------------------------------
# 4a. Far-field intensities of 2D and 3D spaces (base/base_solver.py:213-249)
# ---------------------------------------------------------------------------
def farfield_reference():
    from types import SimpleNamespace

    from thick_ptycho.forward_model.base.base_solver import BaseForwardModelSolver

    rng = np.random.default_rng(77)
    out = {}
    for dim, scans, block in ((2, 5, 40), (3, 4, 36)):
        obj = SimpleNamespace(simulation_space=SimpleNamespace(dimension=dim, total_scans=scans, block_size=block))
        ex = rng.standard_normal((scans, block)) + 1j * rng.standard_normal((scans, block))
        out[f"ex_{dim}d"] = ex
        out[f"intensity_{dim}d"] = BaseForwardModelSolver.get_farfield_intensities(obj, exit_waves=ex,
                                                                                  poisson_noise=False)
    save("farfield_ref", **out)


# ---------------------------------------------------------------------------
# 4b. Reference NLCG reconstruction (pwe_reconstructor.py:166-368)
# ---------------------------------------------------------------------------
def nlcg_reference():
    """n after 1, 2 and 3 iterations of ReconstructorPWE.reconstruct (phase
    retrieval, computed step sizes) from the same start, and the residuals."""
    ss = small_space_2d(nz=16)
    rng = np.random.default_rng(2024)
    probes = create_ptycho_probes(ss)
    n_true = 1 + 1e-3 * (rng.standard_normal((ss.nx, ss.nz)) + 0.05j * np.abs(rng.standard_normal((ss.nx, ss.nz))))
    fwd = PWEIterativeLUSolver(ss, probes, bc_type="impedance")
    data = fwd.get_farfield_intensities(fwd.solve(n=n_true), poisson_noise=False)
    n0 = (1 + 2e-4 * rng.standard_normal((ss.nx, ss.nz))).astype(complex)
    out = {"n0": n0, "data": data, "probes": np.asarray(probes)[0], **sim_params(ss)}
    for iters in (1, 2, 3):
        rec = ReconstructorPWE(ss, data, phase_retrieval=True, solver_type="iterative", bc_type="impedance",
                               verbose=False)
        nk, _, residual = rec.reconstruct(max_iters=iters, n_initial=n0.copy())
        out[f"n_{iters}"] = np.asarray(nk)
        out[f"residual_{iters}"] = np.asarray(residual)
    save("nlcg_ref", **out)


# ---------------------------------------------------------------------------
# 4c. Reference multislice 3PIE reconstruction (ms_reconstructor.py:40-190)
# ---------------------------------------------------------------------------
def ms3pie_reference():
    """n after 1 and 2 epochs of ReconstructorMS.reconstruct (phase retrieval,
    alpha_obj = 0.1: with 1 the reference's update diverges on this problem)
    on a 40-pixel-wide space (a length the GPU FFT plans)."""
    from thick_ptycho.reconstruction.ms_reconstructor import ReconstructorMS

    cfg = SimulationConfig(
        probe_config=ProbeConfig(type=ProbeType.GAUSSIAN, wave_length=0.5, diameter=12.0),
        scan_points=4, step_size_px=5, pad_factor=2.0, nz=16,
        spatial_limits=Limits(x=(0.0, 33.0), z=(0.0, 15.0), units="meters"), use_logging=False,
    )
    ss = create_simulation_space(cfg)
    assert ss.nx == 40, ss.nx
    probes = create_ptycho_probes(ss)
    # a smooth object: its scattering stays inside the probes' band, so the
    # modulus projection never takes its phase from round-off (a white-noise
    # object scatters into frequencies where the model's spectrum is zero)
    n_true = 1 + blob_field_2d(ss.nx, ss.nz, 4, 31, sigma=(3.0, 6.0), amplitude=(-1e-3, 1e-3), absorption=1e-5)
    ms = MSForwardModelSolver(ss, probes)
    data = ms.get_farfield_intensities(ms.solve(n=n_true), poisson_noise=False)
    out = {"data": data, "probes": np.asarray(probes)[0], "n_medium": complex(ss.n_medium), **sim_params(ss)}
    for iters in (1, 2):
        rec = ReconstructorMS(ss, data, phase_retrieval=True, verbose=False)
        n_est, loss = rec.reconstruct(max_iters=iters, alpha_obj=0.1)
        out[f"n_{iters}"] = np.asarray(n_est)
        out[f"loss_{iters}"] = np.asarray(loss)
    save("ms3pie_ref", **out)


# ---------------------------------------------------------------------------
# 5. Random small 3D cases and scan orders
# ---------------------------------------------------------------------------
def pit_reference():
    """PWEFullPinTSolver (full_pint.py): α-circulant right-preconditioned GMRES
    on the space-time system, defaults (α = 1e-2, atol = 1e-8) and α = 0.1, on
    the random 2D case; the FullLU solution of the same system beside it."""
    from thick_ptycho.forward_model import PWEFullPinTSolver

    g = np.load(os.path.join(HERE, "random2d.npz"))
    ss = small_space_2d()
    probes = create_ptycho_probes(ss)
    n = g["n"]
    out = {"n": n, "probes": probes[0], **sim_params(ss)}
    for bc in ("neumann", "impedance", "dirichlet"):
        out[f"pit_{bc}"] = PWEFullPinTSolver(ss, probes, bc_type=bc).solve(n=n)[0, 0]
        out[f"pit_{bc}_alpha01"] = PWEFullPinTSolver(ss, probes, bc_type=bc, alpha=0.1).solve(n=n)[0, 0]
        out[f"fulllu_{bc}"] = PWEFullLUSolver(ss, probes, bc_type=bc).solve(n=n)[0, 0]
    save("pit2d", **out)


def pit_adjoint_reference():
    """PWEFullPinTSolver in mode "adjoint" (full_pint.py:140-166, _pint_utils.py:
    27-54): GMRES on the block-bidiagonal system with conjugate-transposed A, B
    and the z-flipped conjugate C, right-preconditioned by the forward
    α-circulant preconditioner, for a given right-hand side (the flat
    column-major (N, L) space-time vector) and for the probe right-hand side."""
    from thick_ptycho.forward_model import PWEFullPinTSolver

    g = np.load(os.path.join(HERE, "random2d.npz"))
    ss = small_space_2d()
    probes = create_ptycho_probes(ss)
    n = g["n"]
    rhs = g["rhs_block"]
    out = {"n": n, "probes": probes[0], "rhs_block": rhs, **sim_params(ss)}
    for bc in ("neumann", "impedance", "dirichlet"):
        s = PWEFullPinTSolver(ss, probes, bc_type=bc)
        out[f"adj_rhs_{bc}"] = s._solve_single_probe(scan_idx=1, n=n, mode="adjoint",
                                                     rhs_block=rhs.ravel(order="F"), probe=probes[0, 1])
        s = PWEFullPinTSolver(ss, probes, bc_type=bc)
        out[f"adj_probe_{bc}"] = s._solve_single_probe(scan_idx=2, n=n, mode="adjoint", probe=probes[0, 2])
    save("pit2d_adjoint", **out)


def random_3d():
    rng = np.random.default_rng(77)
    cfg = SimulationConfig(
        probe_config=ProbeConfig(type=ProbeType.GAUSSIAN, wave_length=0.5, diameter=6.0),
        scan_points=2, step_size_px=5, pad_factor=1.0, nz=7,
        spatial_limits=Limits(x=(0.0, 9.0), y=(0.0, 9.0), z=(0.0, 6.0), units="meters"), use_logging=False,
    )
    ss = create_simulation_space(cfg)
    probes = create_ptycho_probes(ss)
    shape = (ss.nx, ss.ny, ss.nz)
    n = 1 + 2e-3 * (rng.standard_normal(shape) + 0.1j * rng.standard_normal(shape))
    out = dict(n=n, probes=probes[0], **sim_params(ss))
    rhs = rng.standard_normal((ss.block_size, ss.nz - 1)) + 1j * rng.standard_normal((ss.block_size, ss.nz - 1))
    out["rhs_block"] = rhs
    for bc in ("neumann", "impedance", "dirichlet"):
        solver = PWEIterativeLUSolver(ss, probes, bc_type=bc)
        out[f"{bc}_forward"] = solver.solve(n=n)[0, 0]
        solver.reset_cache()
        out[f"{bc}_adjoint"] = solver._solve_single_probe(scan_idx=1, n=n, mode="adjoint", rhs_block=rhs, probe=None)
    save("random3d", **out)


def geometry():
    out = {}
    for sp_, step, pad in ((32, 6, 4.0 / 3.0), (512, 3, 2048 / 1536), (256, 4, 1024 / 1024), (5, 7, 1.3)):
        cfg = SimulationConfig(probe_config=ProbeConfig(type=ProbeType.GAUSSIAN, wave_length=0.5, diameter=8.0),
                               scan_points=sp_, step_size_px=step, pad_factor=pad, nz=4,
                               spatial_limits=Limits(x=(0.0, 1.0), z=(0.0, 1.0), units="meters"), use_logging=False)
        ss = create_simulation_space(cfg)
        out[f"2d_{sp_}_{step}_nx"] = ss.nx
        out[f"2d_{sp_}_{step}_centres"] = np.array([f.probe_centre_discrete.x for f in ss.scan_frame_info])
    for path in (ScanPath.SERPENTINE, ScanPath.RASTER, ScanPath.SPIRAL):
        for sp_, step, pad in ((8, 16, 2.0), (16, 10, 1.2), (3, 5, 1.0)):
            cfg = SimulationConfig(probe_config=ProbeConfig(type=ProbeType.GAUSSIAN, wave_length=0.5, diameter=8.0),
                                   scan_points=sp_, step_size_px=step, pad_factor=pad, nz=4, scan_path=path,
                                   spatial_limits=Limits(x=(0.0, 1.0), y=(0.0, 1.0), z=(0.0, 1.0), units="meters"),
                                   use_logging=False)
            ss = create_simulation_space(cfg)
            key = f"3d_{path.value}_{sp_}_{step}"
            out[key + "_nx"] = ss.nx
            out[key + "_cx"] = np.array([f.probe_centre_discrete.x for f in ss.scan_frame_info])
            out[key + "_cy"] = np.array([f.probe_centre_discrete.y for f in ss.scan_frame_info])
    save("geometry", **out)


if __name__ == "__main__":
    sections = [geometry, kat_2d, random_2d, config0_reference, gradient_reference, farfield_reference,
                nlcg_reference, ms3pie_reference, kat_3d, random_3d, pit_reference, pit_adjoint_reference]
    wanted = set(sys.argv[2:])
    for fn in sections:
        if not wanted or fn.__name__ in wanted:
            fn()
