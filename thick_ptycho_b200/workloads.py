"""Seeded synthetic workloads (refractive-index perturbations and probes).

The benchmark workloads are defined by their shapes and value
distributions: 2D fields are sums of Gaussian blobs (σ uniform in px, peak
amplitude uniform, centres uniform over the grid) plus a uniform absorption
``i·absorption``; 3D fields are sums of axis-aligned ellipsoids (semi-axes
uniform in px, amplitude uniform) plus absorption.  Probes are Gaussians of a
given 1/e amplitude waist centred at the reference's scan centres.

``δn`` here is the physical perturbation ``n_phys − 1``.  The reference PWE
solvers expect ``n_ref = 1 − δn`` (their object term has the opposite sign to
their multislice transmission), the multislice solver ``n = 1 + δn``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import SimulationGeometry


def blob_field_2d(nx, nz, n_blobs, seed, sigma=(4.0, 12.0), amplitude=(-1e-3, 1e-3), absorption=1e-5):
    """δn(x, z) = Σ Gaussian blobs + i·absorption, complex128 of shape (nx, nz)."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx, dtype=np.float64)[:, None]
    z = np.arange(nz, dtype=np.float64)[None, :]
    dn = np.zeros((nx, nz), dtype=np.float64)
    for _ in range(n_blobs):
        cx = rng.uniform(0, nx)
        cz = rng.uniform(0, nz)
        s = rng.uniform(*sigma)
        a = rng.uniform(*amplitude)
        dn += a * np.exp(-((x - cx) ** 2 + (z - cz) ** 2) / (2 * s * s))
    return dn + 1j * absorption


def ellipsoid_field_3d(nx, ny, nz, n_ell, seed, semi=(3.0, 15.0), amplitude=(0.0, 5e-4), absorption=1e-6):
    """δn(x, y, z) = Σ uniform ellipsoids + i·absorption, complex128 (nx, ny, nz)."""
    rng = np.random.default_rng(seed)
    dn = np.zeros((nx, ny, nz), dtype=np.float64)
    for _ in range(n_ell):
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
        ax = rng.uniform(*semi, 3)
        a = rng.uniform(*amplitude)
        lo = np.maximum(np.floor(c - ax).astype(int), 0)
        hi = np.minimum(np.ceil(c + ax).astype(int) + 1, [nx, ny, nz])
        if np.any(hi <= lo):
            continue
        xs = np.arange(lo[0], hi[0])[:, None, None]
        ys = np.arange(lo[1], hi[1])[None, :, None]
        zs = np.arange(lo[2], hi[2])[None, None, :]
        inside = ((xs - c[0]) / ax[0]) ** 2 + ((ys - c[1]) / ax[1]) ** 2 + ((zs - c[2]) / ax[2]) ** 2 <= 1.0
        dn[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += a * inside
    return dn + 1j * absorption


def gaussian_probes_2d(nx, centres, waist):
    """(P, nx) complex probes ``exp(−(x − c)²/w²)`` (flat phase)."""
    x = np.arange(nx, dtype=np.float64)[None, :]
    c = np.asarray(centres, dtype=np.float64)[:, None]
    return np.exp(-((x - c) ** 2) / waist**2).astype(np.complex128)


def gaussian_probes_3d(nx, ny, centres, waist):
    """(P, nx, ny) complex probes ``exp(−r²/w²)`` (flat phase)."""
    x = np.arange(nx, dtype=np.float64)[:, None]
    y = np.arange(ny, dtype=np.float64)[None, :]
    out = np.empty((len(centres), nx, ny), dtype=np.complex128)
    for p, (cx, cy) in enumerate(centres):
        out[p] = np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / waist**2)
    return out


@dataclass(frozen=True)
class Workload:
    """One benchmark configuration."""

    name: str
    dimension: int
    nx: int
    nz: int
    scan_points: int
    step: int
    waist: float
    n_shapes: int
    seed: int
    wave_length: float = 0.5

    @property
    def num_probes(self):
        return self.scan_points ** (self.dimension - 1)

    def geometry(self, bc_free=True) -> SimulationGeometry:
        if self.dimension == 2:
            return SimulationGeometry.grid_2d(self.nx, self.nz, self.wave_length, self.scan_points, self.step)
        return SimulationGeometry.grid_3d(self.nx, self.nz, self.wave_length, self.scan_points, self.step)

    def delta_n(self):
        if self.dimension == 2:
            return blob_field_2d(self.nx, self.nz, self.n_shapes, self.seed)
        return ellipsoid_field_3d(self.nx, self.nx, self.nz, self.n_shapes, self.seed)

    def probes(self, geom: SimulationGeometry = None):
        geom = geom or self.geometry()
        if self.dimension == 2:
            return gaussian_probes_2d(self.nx, geom.centres, self.waist)
        return gaussian_probes_3d(self.nx, self.nx, geom.centres, self.waist)


# The benchmark configurations (sizes, seeds and distributions as specified).
CONFIG0 = Workload("2d-forward-256x128-p32", 2, 256, 128, 32, 6, 8.0, 12, 0)
CONFIG1 = Workload("2d-fwd-adj-2048x1024-p512", 2, 2048, 1024, 512, 3, 8.0, 200, 0)
CONFIG2 = Workload("3d-forward-256x256x256-p64", 3, 256, 256, 8, 16, 12.0, 400, 1)
CONFIG3 = Workload("2d-grad-1024x512-p256", 2, 1024, 512, 256, 4, 8.0, 300, 0)
CONFIG4 = Workload("3d-recon-192x192x192-p256", 3, 192, 192, 16, 10, 12.0, 600, 1)
# Reduced-depth case of the CONFIG1 kernels (same N and probe count, 128 nodes):
# small enough for full profiler captures, larger than L2 (1.07 GB field).
PROFILE1 = Workload("2d-fwd-adj-2048x128-p512", 2, 2048, 128, 512, 3, 8.0, 200, 0)
CONFIGS = {w.name: w for w in (CONFIG0, CONFIG1, CONFIG2, CONFIG3, CONFIG4, PROFILE1)}
