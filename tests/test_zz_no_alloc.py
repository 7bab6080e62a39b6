"""The allocation-free entry point ``tp_cn2d_march_noalloc``.

Some callers cannot allocate device memory: a host that owns the whole device
budget as a pre-reserved pool and passes only its input and output buffers,
or a latency-bounded loop where cudaMalloc (which may synchronise the device)
is not allowed.  ``tp_cn2d_march_noalloc`` serves them by keeping the
per-slice factor set in a fixed 32 MiB device array inside the library.

This test calls it through the C ABI twice in a row, with different inputs,
and compares each result with the allocating entry points (``tp_cn2d_factor``
into a caller workspace + ``tp_cn2d_march``).  Both run the same kernels on
the same inputs, so the exit waves and stored fields must be bit-identical.
It covers N = 256 (the per-warp march) and N = 512 (the team march, whose
16-byte bulk copies also read the factor set from the static array).  It also
checks that a problem whose factor set exceeds the 32 MiB limit is rejected
with a clear error.  The file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200 import _native  # noqa: E402
from thick_ptycho_b200.cn2d import CN2D  # noqa: E402
from thick_ptycho_b200.workloads import CONFIG0, blob_field_2d, gaussian_probes_2d  # noqa: E402


def _args(P, mode, probes, exit_out, u_store=None):
    a = _native.TpCn2dMarchArgs()
    a.num_probes, a.mode = P, mode
    a.probes = ctypes.c_void_p(probes.data_ptr())
    a.exit_out = ctypes.c_void_p(exit_out.data_ptr())
    if u_store is not None:
        a.u_store = ctypes.c_void_p(u_store.data_ptr())
    return a


def _run_noalloc(eng, field, probes, P):
    lib = _native.load()
    ex = torch.zeros((P, eng.n), dtype=torch.complex64, device="cuda")
    st = eng.new_store(P)
    o = eng.op()
    a = _args(P, _native.MODE_FORWARD, probes, ex, st)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.tp_cn2d_march_noalloc(ctypes.byref(o), ctypes.c_void_p(field.data_ptr()), _native.C128, ctypes.byref(a),
                                   stream)
    _native.check(rc, "tp_cn2d_march_noalloc")
    eng.device_status()
    return ex, st


def _run_allocating(eng, field, probes, P):
    fs = eng.factor(field, "forward")
    ex = torch.zeros((P, eng.n), dtype=torch.complex64, device="cuda")
    st = eng.new_store(P)
    eng.march(fs, P, probes=probes, u_store=st, exit_out=ex)
    eng.device_status()
    return ex, st


def _case(n):
    """(N, nz, k, n field, probes) of the 256 x 128 config-0 workload, or of a
    512 x 96 workload of the same kind (seeded blobs, 24 Gaussian probes)."""
    if n == 256:
        w = CONFIG0
        geo = w.geometry()
        return w.nx, w.nz, geo.k, w.delta_n(), w.probes(geo)
    nz = 96
    centres = np.linspace(40, n - 40, 24)
    return n, nz, 4 * np.pi, blob_field_2d(n, nz, 30, 5), gaussian_probes_2d(n, centres, 8.0)


@pytest.mark.parametrize("n", [256, 512])
def test_noalloc_matches_allocating_path_on_two_calls(n):
    N, nz, k, dn, pr = _case(n)
    eng = CN2D(N, nz, k, 1.0, 1.0, "impedance")
    P = pr.shape[0]
    probes = torch.from_numpy(pr.astype(np.complex64)).cuda()
    fields = [torch.from_numpy(1 - dn).cuda(), torch.from_numpy(1 - 0.5 * dn[:, ::-1].copy()).cuda()]
    for field in fields:  # two calls in a row, different inputs
        ex_n, st_n = _run_noalloc(eng, field, probes, P)
        ex_a, st_a = _run_allocating(eng, field, probes, P)
        assert torch.equal(ex_n, ex_a)
        assert torch.equal(st_n, st_a)
        assert torch.isfinite(torch.view_as_real(ex_n)).all() and ex_n.abs().max() > 0


def test_noalloc_rejects_sizes_beyond_its_static_limit():
    lib = _native.load()
    eng = CN2D(2048, 1024, 4 * np.pi, 1.0, 1.0, "impedance")
    assert eng.factor_bytes > 32 << 20
    field = torch.ones((2048, 1024), dtype=torch.complex128, device="cuda")
    probes = torch.zeros((1, 2048), dtype=torch.complex64, device="cuda")
    ex = torch.zeros((1, 2048), dtype=torch.complex64, device="cuda")
    o = eng.op()
    a = _args(1, _native.MODE_FORWARD, probes, ex)
    rc = lib.tp_cn2d_march_noalloc(ctypes.byref(o), ctypes.c_void_p(field.data_ptr()), _native.C128, ctypes.byref(a),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 5  # TP_ERR_WORKSPACE
    assert b"static scratch" in lib.tp_last_error_string()
