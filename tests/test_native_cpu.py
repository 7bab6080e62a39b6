"""CPU-side checks: the C-ABI library loads and exports every declared symbol,
and the host-side operator/geometry logic matches the oracle and the
reference's golden geometry.  No compute call runs here (no GPU)."""

import ctypes
import os
import re

import numpy as np
import pytest

from oracle import pwe_oracle as po
from thick_ptycho_b200 import _native
from thick_ptycho_b200.geometry import SimulationGeometry, domain_width, order_scan_2d, scan_centres_1d
from thick_ptycho_b200.operators import BCCoefficients, normalize_bc, operator_1d
from thick_ptycho_b200.workloads import CONFIG0, CONFIG1, blob_field_2d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "tpcuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:TP_API\s+)?(?:const\s+)?\w+\s*\*?\s*(tp_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = declared_functions()
    assert len(names) >= 8, names
    for name in names:
        assert hasattr(lib, name), name
    bound = {n for n, _, _ in _native.SIGNATURES}
    assert set(names) <= bound, set(names) - bound
    assert lib.tp_version() >= 100


def test_pure_host_queries():
    lib = _native.load()
    c, m, npad = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    args = (ctypes.byref(c), ctypes.byref(m), ctypes.byref(npad))
    assert lib.tp_cn2d_layout(2048, *args) == 0
    assert (c.value, m.value, npad.value) == (128, 16, 2048)          # team path
    assert lib.tp_cn2d_layout(256, *args) == 0
    assert (c.value, m.value, npad.value) == (32, 8, 256)             # warp path
    assert lib.tp_cn2d_layout(257, *args) == 0
    assert npad.value >= 257 and npad.value == 32 * m.value
    assert lib.tp_cn2d_layout(4097, *args) != 0
    assert b"4097" in lib.tp_last_error_string()
    # 1023 slices of (5 M + 17 records) x 128 chunks float2, then a 256-byte tail (the PCR coupling bound)
    assert lib.tp_cn2d_factor_bytes(2048, 1024) == 1023 * (5 * 16 + 17) * 128 * 8 + 256
    assert lib.tp_cn2d_factor_bytes(2048, 1) == 0


def test_struct_layout_matches_header():
    # tp_cn2d_op: 6 int32 + 2 double + 6 complex doubles
    assert ctypes.sizeof(_native.TpCn2dOp) == 6 * 4 + 2 * 8 + 12 * 8
    assert ctypes.sizeof(_native.TpCn2dMarchArgs) == 8 + 8 * 8 + 8 + 2 * 8 + 6 * 4


@pytest.mark.parametrize("bc", ["neumann", "impedance", "dirichlet", "impedance2"])
def test_operator_matches_oracle_matrices(bc):
    k, dx, dz, n = 4 * np.pi, 0.7, 1.3, 12
    co = BCCoefficients.make(k, dx, dz, bc)
    K = operator_1d(n, co, bc, dz).dense()
    A, B = po.step_matrices_1d(n, po.bc_coefficients(k, dx, dz, bc_type=bc), bc, dz)
    assert np.allclose(np.eye(n) - K, A.toarray(), rtol=0, atol=1e-15)
    assert np.allclose(np.eye(n) + K, B.toarray(), rtol=0, atol=1e-15)


def test_bc_normalisation():
    from enum import Enum

    class BT(Enum):
        IMPEDANCE = "impedance"

    assert normalize_bc(BT.IMPEDANCE) == "impedance"
    assert normalize_bc("Dirichlet") == "dirichlet"
    with pytest.raises(ValueError):
        normalize_bc("robin")


def test_geometry_matches_reference_golden(golden):
    g = golden("geometry")
    for sp_, step, pad in ((32, 6, 4.0 / 3.0), (512, 3, 2048 / 1536), (256, 4, 1.0), (5, 7, 1.3)):
        nx = domain_width(sp_, step, pad)
        assert nx == int(g[f"2d_{sp_}_{step}_nx"])
        assert scan_centres_1d(nx, sp_, step) == list(g[f"2d_{sp_}_{step}_centres"])
    for path in ("serpentine", "raster", "spiral"):
        for sp_, step, pad in ((8, 16, 2.0), (16, 10, 1.2), (3, 5, 1.0)):
            key = f"3d_{path}_{sp_}_{step}"
            nx = domain_width(sp_, step, pad)
            assert nx == int(g[key + "_nx"])
            c = scan_centres_1d(nx, sp_, step)
            cx, cy = order_scan_2d(c, c, path)
            assert cx == list(g[key + "_cx"]) and cy == list(g[key + "_cy"])


def test_workloads_are_seeded_and_shaped():
    a = blob_field_2d(64, 32, 5, seed=3)
    b = blob_field_2d(64, 32, 5, seed=3)
    assert np.array_equal(a, b) and a.shape == (64, 32) and np.all(a.imag == 1e-5)
    geo = CONFIG1.geometry()
    assert geo.num_probes == 512 and geo.block_size == 2048 and len(geo.centres) == 512
    assert min(geo.centres) >= 0 and max(geo.centres) < 2048
    assert CONFIG0.geometry().centres == scan_centres_1d(256, 32, 6)


def test_geometry_from_reference_parameters(golden):
    g = golden("config0_ref")
    geo = SimulationGeometry.from_reference_parameters(0.5, (0.0, 256.0), (0.0, 127.0), scan_points=32, step_size_px=6,
                                                       pad_factor=4.0 / 3.0, nz=128)
    assert geo.nx == int(g["nx"]) == 257
    assert abs(geo.dx - float(g["dx"])) < 1e-12 and abs(geo.dz - float(g["dz"])) < 1e-12
    assert geo.centres == list(g["centres"])
