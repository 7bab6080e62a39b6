"""The seeded synthetic workloads every benchmark line and the reference arm
are measured on (no GPU): the configurations' sizes and probe counts, the
2D fields and probes reproduced bit for bit from their seeds, values inside
the stated distributions, and the 3D generator on a reduced grid."""

import numpy as np
import pytest

from thick_ptycho_b200.workloads import (CONFIG0, CONFIG1, CONFIG2, CONFIG3, CONFIG4, CONFIGS, PROFILE1,
                                         ellipsoid_field_3d, gaussian_probes_3d)

SIZES = {  # name: (transverse unknowns N, nz, probes)
    CONFIG0.name: (256, 128, 32),
    CONFIG1.name: (2048, 1024, 512),
    CONFIG2.name: (256 * 256, 256, 64),
    CONFIG3.name: (1024, 512, 256),
    CONFIG4.name: (192 * 192, 192, 256),
    PROFILE1.name: (2048, 128, 512),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_configuration_sizes(name):
    w = CONFIGS[name]
    g = w.geometry()
    N, nz, P = SIZES[name]
    assert (g.block_size, g.nz, w.num_probes, len(g.centres)) == (N, nz, P, P)
    assert g.dx == 1.0 and g.dz == 1.0


@pytest.mark.parametrize("w", [CONFIG0, CONFIG1, CONFIG3, PROFILE1], ids=lambda w: w.name)
def test_2d_fields_and_probes_are_reproducible(w):
    dn1, dn2 = w.delta_n(), w.delta_n()
    assert dn1.shape == (w.nx, w.nz) and dn1.dtype == np.complex128
    assert np.array_equal(dn1, dn2)
    assert np.all(dn1.imag == 1e-5)  # uniform absorption
    assert np.max(np.abs(dn1.real)) <= w.n_shapes * 1e-3  # blobs of peak amplitude in [-1e-3, 1e-3]
    assert np.max(np.abs(dn1.real)) > 0
    g = w.geometry()
    p1, p2 = w.probes(g), w.probes(g)
    assert p1.shape == (w.num_probes, w.nx) and np.array_equal(p1, p2)
    # Gaussians of unit peak at the scan centres (integer centres here)
    peaks = np.abs(p1[np.arange(w.num_probes), np.round(np.asarray(g.centres)).astype(int)])
    assert np.allclose(peaks, 1.0, atol=1e-2)


def test_3d_generator_reduced_grid():
    dn1 = ellipsoid_field_3d(24, 20, 16, 30, seed=3)
    dn2 = ellipsoid_field_3d(24, 20, 16, 30, seed=3)
    assert dn1.shape == (24, 20, 16) and np.array_equal(dn1, dn2)
    assert np.all(dn1.imag == 1e-6)
    assert dn1.real.min() >= 0.0 and dn1.real.max() <= 30 * 5e-4
    assert not np.array_equal(dn1, ellipsoid_field_3d(24, 20, 16, 30, seed=4))
    pr = gaussian_probes_3d(24, 20, [(5.0, 6.0), (12.0, 9.0)], 4.0)
    assert pr.shape == (2, 24, 20) and abs(pr[0, 5, 6] - 1.0) < 1e-12 and abs(pr[1, 12, 9] - 1.0) < 1e-12
