"""The 3D BiCGStab march at the full benchmark geometries against complex128.

Geometries: 256 x 256 transverse x 256 nodes (400 seeded ellipsoids, 8 x 8
probe raster, stride 16, waist 12) and 192 x 192 x 192 (600 ellipsoids,
16 x 16 raster, stride 10), impedance edges, n = 1 − δn.  The fixtures
(``tests/golden/config{2,4}_3d_full.npz``, made by ``make_golden_3d_full.py``
with the oracle's per-slice SuperLU march) hold three probes' exit waves and,
for a fixed exit-plane source on probe 0, the exact-adjoint gradient at three
slices and its norm at every slice.

Tolerances: relative L2 ≤ 1e-5 for exit waves and gradient slices, and each
slice's gradient norm within 1e-5 relative; plain FFT-preconditioned and
learned (trained briefly on solver-generated white-noise pairs of another
seeded field) forms, both at the march's default stopping residual.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from thick_ptycho_b200.cn3d import CN3D, generate_pairs  # noqa: E402
from thick_ptycho_b200.learned import LearnedPreconditioner, default_kappa  # noqa: E402
from thick_ptycho_b200.workloads import CONFIG2, CONFIG4, ellipsoid_field_3d  # noqa: E402

TOL = 1e-5
WORKLOADS = {"config2": CONFIG2, "config4": CONFIG4}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _setup(name, golden):
    g = golden(f"{name}_3d_full")
    w = WORKLOADS[name]
    geo = w.geometry()
    n = w.nx
    assert (int(g["nx"]), int(g["nz"])) == (n, w.nz)
    eng = CN3D(n, n, w.nz, geo.k, 1.0, 1.0, 1.0, "impedance")
    field = torch.from_numpy((1 - w.delta_n()).reshape(n * n, w.nz)).cuda()
    idx = [int(i) for i in g["probe_idx"]]
    probes = torch.from_numpy(w.probes(geo).reshape(w.num_probes, n * n)[idx].astype(np.complex64)).cuda()
    return g, w, eng, field, probes


def _check(g, eng, field, probes, **kw):
    P = probes.shape[0]
    store = eng.new_store(P)
    ex = torch.empty((P, eng.N), dtype=torch.complex64, device="cuda")
    eng.read_stats()
    eng.march(field, P, "forward", probes=probes, u_store=store, exit_out=ex, **kw)
    st_f = eng.read_stats()
    ex = ex.cpu().numpy()
    for j in range(P):
        assert rel(ex[j], g["exit"][j]) < TOL, (j, rel(ex[j], g["exit"][j]))
    # exact adjoint of probe 0 from the fixture's exit-plane source
    gc = torch.zeros((eng.L, eng.N), dtype=torch.complex64, device="cuda")
    src = torch.from_numpy(g["src"][None]).cuda()
    eng.march(field, 1, "adjoint_exact", src_exit=src, u_fwd=store[:1].contiguous(), grad_c=gc, **kw)
    st_a = eng.read_stats()
    gc = gc.cpu().numpy()
    for s, ref in zip(g["grad_s"], g["grad_slices"]):
        assert rel(gc[s - 1], ref) < TOL, (int(s), rel(gc[s - 1], ref))
    norms = np.linalg.norm(gc.astype(np.complex128), axis=1)
    assert np.max(np.abs(norms - g["grad_norms"]) / g["grad_norms"]) < TOL
    assert st_f["failed"] == 0 and st_a["failed"] == 0
    return st_f, st_a


@pytest.mark.parametrize("name", ["config2", "config4"])
def test_plain_march_full_geometry(golden, name):
    g, w, eng, field, probes = _setup(name, golden)
    _check(g, eng, field, probes, precond=True)


def test_learned_march_full_geometry(golden):
    g, w, eng, field, probes = _setup("config2", golden)
    geo = w.geometry()
    n = w.nx
    # a short training run on white-noise pairs of another seeded field (8 probes)
    other = torch.from_numpy((1 - ellipsoid_field_3d(n, n, w.nz, w.n_shapes, 1001)).reshape(n * n, w.nz)).cuda()
    tr_probes = torch.from_numpy(w.probes(geo).reshape(w.num_probes, n * n)[::8].astype(np.complex64)).cuda()
    pairs = generate_pairs(eng, other, tr_probes.contiguous(), every=4, kind="noise")
    model = LearnedPreconditioner(n, n, default_kappa(geo.k, 1.0, 5e-4), seed=0)
    model.train(pairs, steps=300, slices_per_batch=2, lr=1e-3)
    del pairs, other
    _check(g, eng, field, probes, precond="learned", model=model)
    assert eng.fallbacks == 0
