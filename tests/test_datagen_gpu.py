"""Far-field intensities, Poisson noise and the simulated-data file of the
drop-in solver (base/base_solver.py:213-249, generate_data.py:185-197),
against the reference's own outputs (golden) and the complex128 oracle.

Tolerances: intensities from complex64 exit waves ≤ 1e-5 relative (2D FFT head
and the 3D fft2); Poisson noise: the same generator seed gives identical
counts, and over 200 000 draws the sample mean and variance match the
intensity to 1 % (6σ of the estimator at this size).
"""

import os
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import pwe_oracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200 import SimulationGeometry  # noqa: E402
from thick_ptycho_b200.solver import PWEGpuSolver  # noqa: E402


def _fake(dim, scans, block):
    return SimpleNamespace(device=torch.device("cuda"), dimension=dim, block_size=block,
                           simulation_space=SimpleNamespace(total_scans=scans))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def test_farfield_matches_reference_2d_and_3d(golden):
    g = golden("farfield_ref")
    for dim, (scans, block) in ((2, (5, 40)), (3, (4, 36))):
        I = PWEGpuSolver.get_farfield_intensities(_fake(dim, scans, block), exit_waves=g[f"ex_{dim}d"],
                                                  poisson_noise=False)
        assert rel(I, g[f"intensity_{dim}d"]) < 1e-5, dim


def test_poisson_noise_seeded_and_unbiased():
    fake = _fake(2, 2, 50)
    ex = np.full((2, 50), 0.0, dtype=complex)
    ex[:, 0] = 3.0  # |FFT|^2 = 9 in every bin
    a = PWEGpuSolver.get_farfield_intensities(fake, exit_waves=ex, generator=torch.Generator(device="cuda").manual_seed(1))
    b = PWEGpuSolver.get_farfield_intensities(fake, exit_waves=ex, generator=torch.Generator(device="cuda").manual_seed(1))
    assert a.dtype == np.int64 and np.array_equal(a, b)
    big = _fake(2, 2000, 100)
    exb = np.zeros((2000, 100), dtype=complex)
    exb[:, 0] = 3.0
    draws = PWEGpuSolver.get_farfield_intensities(big, exit_waves=exb, generator=torch.Generator(device="cuda").manual_seed(2))
    assert abs(draws.mean() - 9.0) < 0.09 and abs(draws.var() - 9.0) < 0.09 * 9


def test_simulated_data_file(tmp_path):
    geo = SimulationGeometry.grid_2d(64, 16, 0.5, 4, 6)
    rng = np.random.default_rng(3)
    n = 1 + 1e-3 * rng.standard_normal(geo.shape) + 1e-5j
    x = np.arange(64)
    probes = np.exp(-((x[None] - np.array(geo.centres)[:, None]) ** 2) / 25.0).astype(complex)[None]
    s = PWEGpuSolver(geo, probes, bc_type="impedance")
    path = os.path.join(tmp_path, "simulated_data.npz")
    data, ex = s.save_simulated_data(path, n=n, poisson_noise=False)
    with np.load(path) as f:
        assert set(f.files) == {"intensity", "exit_waves"}
        assert f["intensity"].shape == (4, 64) and f["exit_waves"].shape == (4, 64)
        assert rel(f["intensity"], po.farfield_intensity(f["exit_waves"])) < 1e-5
