"""complex128 oracle fixtures of the full 3D benchmark geometries.

    python tests/golden/make_golden_3d_full.py [config2] [config4]

For the 256 x 256 x 256-node geometry (64 probes, 400 ellipsoids, seed 1) and
the 192 x 192 x 192-node one (256 probes, 600 ellipsoids, seed 1), impedance
edges, n = 1 − δn (the reference PWE's index convention), this computes with
the complex128 restatement of the reference's per-slice SuperLU march
(``oracle.pwe_oracle``, one slice factorised at a time):

* ``exit``: the exit waves of the probes ``probe_idx`` (stored complex64: the
  rounding, ~6e-8 relative, is far below the 1e-5 parity bound);
* ``src``: a seeded unit-norm complex64 exit-plane source for probe 0;
* ``grad_slices`` / ``grad_norms``: the exact-adjoint gradient
  ``g_s = λ_s conj(u_s + u_{s−1})`` of that source and probe 0's forward field,
  at the slices ``grad_s`` (1-based), and ``‖g_s‖`` for every slice.

The forward and the adjoint are independent (the source is fixed), so the four
marches run in four processes, one thread each (SuperLU's BLAS calls would
otherwise start a thread pool per process and oversubscribe the cores).  Takes
~5 minutes on 4 host cores.  The
fixtures are committed; the GPU tests only read them.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

for _v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_v] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# probes checked at each geometry (first, a middle one, last)
PROBES = {"config2": (0, 27, 63), "config4": (0, 119, 255)}


def _setup(name):
    from oracle import pwe_oracle as po
    from thick_ptycho_b200.workloads import CONFIG2, CONFIG4

    w = {"config2": CONFIG2, "config4": CONFIG4}[name]
    geo = w.geometry()
    n = w.nx
    co = po.bc_coefficients(geo.k, 1.0, 1.0, dy=1.0, bc_type="impedance", dimension=3)
    A, B = po.step_matrices_2d(n, n, co, "impedance", 1.0)
    field = (1 - w.delta_n()).reshape(n * n, w.nz)
    C = po.object_contribution(field, geo.k, 1.0)
    return w, geo, A, B, C


def source(N, seed=7):
    rng = np.random.default_rng(seed)
    s = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    return (s / np.float32(np.linalg.norm(s))).astype(np.complex64)


def job(args):
    name, kind, tmp = args
    from oracle import pwe_oracle as po

    w, geo, A, B, C = _setup(name)
    N, L = A.shape[0], C.shape[1]
    t0 = time.time()
    if kind == "forward":
        probes = w.probes(geo).reshape(w.num_probes, N)
        idx = list(PROBES[name])
        # the gradient needs probe 0's whole field: march it with the others and keep every node
        exit_w, kept = po.march_streamed(A, B, C, probes[idx], keep=range(L + 1))
        u0 = np.stack([kept[t][0] for t in range(L + 1)], axis=1)  # (N, nz)
        np.save(os.path.join(tmp, f"{name}_u0.npy"), u0)
        np.save(os.path.join(tmp, f"{name}_exit.npy"), exit_w)
    else:
        src = np.zeros((1, N, L), dtype=complex)
        src[0, :, L - 1] = source(N).astype(complex)
        lam = po.exact_adjoint_many(A, B, C, src)[0]  # (N, L)
        np.save(os.path.join(tmp, f"{name}_lam.npy"), lam)
    return name, kind, time.time() - t0


def main(names):
    import tempfile

    from oracle import pwe_oracle as po

    with tempfile.TemporaryDirectory() as tmp:
        jobs = [(n, k, tmp) for n in names for k in ("forward", "adjoint")]
        with mp.get_context("spawn").Pool(len(jobs)) as pool:
            for name, kind, dt in pool.imap_unordered(job, jobs):
                print(f"{name} {kind}: {dt:.0f} s", flush=True)
        for name in names:
            w, geo, A, B, C = _setup(name)
            N, L = A.shape[0], C.shape[1]
            u0 = np.load(os.path.join(tmp, f"{name}_u0.npy"))
            lam = np.load(os.path.join(tmp, f"{name}_lam.npy"))
            g = po.grad_c_from_adjoint(u0, lam)  # (N, L), column s-1 = slice s
            grad_s = np.array([1, L // 2, L])
            out = dict(
                nx=w.nx, nz=w.nz, k=geo.k, num_probes=w.num_probes, probe_idx=np.array(PROBES[name]),
                exit=np.load(os.path.join(tmp, f"{name}_exit.npy")).astype(np.complex64),
                src=source(N), grad_s=grad_s, grad_slices=g[:, grad_s - 1].T.astype(np.complex64),
                grad_norms=np.linalg.norm(g, axis=0),
            )
            path = os.path.join(HERE, f"{name}_3d_full.npz")
            np.savez_compressed(path, **out)
            print(f"wrote {os.path.basename(path)} ({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main([a for a in sys.argv[1:] if a in PROBES] or list(PROBES))
