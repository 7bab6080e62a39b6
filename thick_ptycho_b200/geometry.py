"""Simulation geometry used by the GPU solvers.

``SimulationGeometry`` carries exactly the attributes that the reference's
solvers read from a ``SimulationSpace2D/3D``
(``thick_ptycho/simulation/simulation_space/``), so either object can be
handed to :class:`thick_ptycho_b200.PWEGpuSolver`.  Its constructor restates
the reference's grid and scan arithmetic:

* z axis: ``base_simulation_space.py:192-202``
* transverse width, padding and parity rule: ``base_simulation_space.py:204-234``
* 2D scan centres: ``simulation_space_2d.py:80-130``
* 3D scan centres and serpentine / spiral / raster orders:
  ``simulation_space_3d.py:167-307``

Scan-centre indices are integer results and must match the reference exactly
(Python ``round`` is half-to-even, as in the reference).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np


def scan_centres_1d(nx: int, scan_points: int, step_size: int) -> List[int]:
    """Probe centre pixels along one axis (``simulation_space_2d.py:104-110``)."""
    if scan_points == 1:
        return [nx // 2]
    mid = (nx - 1) / 2.0
    return [int(round(mid + (i - (scan_points - 1) / 2) * step_size)) for i in range(scan_points)]


def order_scan_2d(x_coords, y_coords, scan_path: str):
    """Scan order over a 2D grid of centres (``simulation_space_3d.py:243-307``)."""
    cx, cy = [], []
    if scan_path == "serpentine":
        xs = list(np.flip(x_coords))
        ys = list(y_coords)
        for x in xs:
            for y in ys:
                cx.append(int(x))
                cy.append(int(y))
            ys = list(np.flip(ys))
    elif scan_path == "raster":
        for y in y_coords:
            for x in x_coords:
                cx.append(int(x))
                cy.append(int(y))
    elif scan_path == "spiral":
        left, right = 0, len(x_coords) - 1
        top, bottom = 0, len(y_coords) - 1
        while left <= right and top <= bottom:
            for i in range(left, right + 1):
                cx.append(int(x_coords[i]))
                cy.append(int(y_coords[top]))
            top += 1
            for i in range(top, bottom + 1):
                cx.append(int(x_coords[right]))
                cy.append(int(y_coords[i]))
            right -= 1
            if top <= bottom:
                for i in range(right, left - 1, -1):
                    cx.append(int(x_coords[i]))
                    cy.append(int(y_coords[bottom]))
                bottom -= 1
            if left <= right:
                for i in range(bottom, top - 1, -1):
                    cx.append(int(x_coords[left]))
                    cy.append(int(y_coords[i]))
                left += 1
    else:
        raise ValueError(f"Unknown scan path: {scan_path}")
    return cx, cy


def domain_width(scan_points: int, step_size: int, pad_factor: float) -> int:
    """Transverse grid size with the reference's padding/parity rules.

    Restates ``base_simulation_space.py:207-220``: ``nx = int(pad·min_nx)``,
    made to have even padding, then odd when the step is even (even when odd).
    """
    min_nx = scan_points * step_size
    nx = int(pad_factor * min_nx)
    if (nx - min_nx) % 2 != 0:
        nx += 1
    desired_parity = 1 if (step_size % 2 == 0) else 0
    if nx % 2 != desired_parity:
        nx += 1
    return nx


@dataclass
class SimulationGeometry:
    """Duck-typed stand-in for the reference ``SimulationSpace2D/3D``.

    Only full-domain solves are modelled (``solve_reduced_domain`` False).
    """

    dimension: int
    nx: int
    nz: int
    dx: float
    dz: float
    k: float
    num_probes: int
    ny: Optional[int] = None
    dy: Optional[float] = None
    probe_angles: Tuple[float, ...] = (0.0,)
    exact_ref_coeff: bool = False
    empty_space_px: int = 0
    n_medium: complex = 1.0 + 0j
    x0: float = 0.0
    z0: float = 0.0
    y0: float = 0.0
    centres: List = field(default_factory=list)
    solve_reduced_domain: bool = False
    num_projections: int = 1
    results_dir: Optional[str] = None
    verbose: bool = False
    use_logging: bool = False

    def __post_init__(self):
        self.num_angles = len(self.probe_angles)
        self.total_scans = self.num_angles * self.num_probes * self.num_projections
        e = self.empty_space_px
        if self.dimension == 2:
            self.effective_nx = self.nx
            self.shape = (self.nx, self.nz)
            self.effective_shape = (self.nx + 2 * e, self.nz)
            self.block_size = self.nx + 2 * e
        else:
            if self.ny is None:
                self.ny = self.nx
            if self.dy is None:
                self.dy = self.dx
            self.effective_nx = self.nx
            self.effective_ny = self.ny
            self.shape = (self.nx, self.ny, self.nz)
            self.effective_shape = (self.nx + 2 * e, self.ny + 2 * e, self.nz)
            self.block_size = (self.nx + 2 * e) * (self.ny + 2 * e)
        self.z = self.z0 + self.dz * np.arange(self.nz)
        self.x = self.x0 + self.dx * np.arange(self.nx)
        if self.dimension == 3:
            self.y = self.y0 + self.dy * np.arange(self.ny)
        self.wave_length = 2 * np.pi / self.k

    @property
    def refractive_index_empty(self):
        return np.ones(self.shape, dtype=complex) * self.n_medium

    @classmethod
    def grid_2d(cls, nx, nz, wave_length, scan_points, step_size_px, dx=1.0, dz=1.0, **kw):
        """2D geometry of an explicit grid with reference-formula scan centres."""
        k = 2 * np.pi / wave_length
        centres = scan_centres_1d(nx, scan_points, step_size_px)
        return cls(dimension=2, nx=nx, nz=nz, dx=dx, dz=dz, k=k, num_probes=scan_points, centres=centres, **kw)

    @classmethod
    def grid_3d(cls, nx, nz, wave_length, scan_points, step_size_px, dx=1.0, dz=1.0, scan_path="raster", **kw):
        """3D geometry (nx = ny) with reference-formula centres in ``scan_path`` order."""
        k = 2 * np.pi / wave_length
        c1 = scan_centres_1d(nx, scan_points, step_size_px)
        if scan_points == 1:
            centres = [(nx // 2, nx // 2)]
        else:
            cx, cy = order_scan_2d(c1, c1, scan_path)
            centres = list(zip(cx, cy))
        return cls(
            dimension=3, nx=nx, ny=nx, nz=nz, dx=dx, dy=dx, dz=dz, k=k, num_probes=scan_points**2, centres=centres, **kw
        )

    @classmethod
    def from_reference_parameters(
        cls,
        wave_length,
        limits_x,
        limits_z,
        scan_points=1,
        step_size_px=10,
        pad_factor=1.0,
        nz=None,
        points_per_wavelength=8,
        limits_y=None,
        scan_path="serpentine",
        **kw,
    ):
        """Geometry computed from the reference's ``SimulationConfig`` fields."""
        if nz is None:
            dz0 = wave_length / points_per_wavelength
            nz = int((limits_z[1] - limits_z[0]) / dz0)
        z = np.linspace(limits_z[0], limits_z[1], nz)
        dz = z[1] - z[0]
        nx = domain_width(scan_points, int(step_size_px), pad_factor)
        x = np.linspace(limits_x[0], limits_x[1], nx)
        dx = x[1] - x[0]
        k = 2 * np.pi / wave_length
        c1 = scan_centres_1d(nx, scan_points, int(step_size_px))
        if limits_y is None:
            return cls(dimension=2, nx=nx, nz=nz, dx=dx, dz=dz, k=k, num_probes=scan_points, centres=c1,
                       x0=limits_x[0], z0=limits_z[0], **kw)
        y = np.linspace(limits_y[0], limits_y[1], nx)
        if scan_points == 1:
            centres = [(nx // 2, nx // 2)]
        else:
            cx, cy = order_scan_2d(c1, c1, scan_path)
            centres = list(zip(cx, cy))
        return cls(dimension=3, nx=nx, ny=nx, nz=nz, dx=dx, dy=y[1] - y[0], dz=dz, k=k, num_probes=scan_points**2,
                   centres=centres, x0=limits_x[0], y0=limits_y[0], z0=limits_z[0], **kw)
