#!/usr/bin/env python
"""Throughput of the paraxial forward + adjoint hot path on B200.

Metric: probe·slice solves per second, forward + adjoint (one forward CN step
plus one adjoint CN step of one probe = one probe·slice), for the 2D batched
workload N = 2048 transverse × Nz = 1024 nodes × 512 probes (stride 3 px),
δn = 200 seeded Gaussian blobs + 1e-5 i, Gaussian probes (waist 8 px).
One step = factorise (forward and adjoint) + forward march storing the full
field (as the half pair sums (u_s + u_{s-1})/2 the gradient contracts with) +
amplitude-loss residual + exact-adjoint march with the fused probe gradient +
mapping onto the index nodes.  The full field (8.6 GB) is far larger than
L2, so no explicit flush is needed between steps.

The same line carries ``learned_vs_plain_3d``: forward + exact-adjoint
probe·slice solves/s of the 3D BiCGStab march (256 x 256 x 256 nodes, 64
probes) with the plain FFT preconditioner and with the learned correction,
after training the network on solver-generated pairs of another field.

``--impl reference`` times the CPU restatement of the reference's
IterativeLU path (per-slice sparse LU, per-probe march, reference adjoint)
on the host cores instead.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (weak scaling: 512 probes per rank, gradient all-reduced over NCCL):
  python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 bench.py --gpus N
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "probe·slice solves/s fwd+adj (2D CN, complex64, exact adjoint + fused gradient)"
REF_BUDGET_S = 120.0    # wall-time target of a whole `--impl reference` run
REF_DEADLINE_S = 200.0  # hard limit: the arm prints its line from the steps finished by then
REF_MAX_WORKERS = 32    # worker processes of the reference arm (one thread each)
# DRAM bytes (read + write) of one exact-adjoint march launch at N = 2048, nz = 1024, 512
# probes: an ncu capture of the same kernel at nz = 128 (127 slices, 512 probes) measured
# 1.0914 GB; the traffic grows in proportion to the slices, so it is scaled by 1023/127.
ADJ_TRAFFIC_BYTES_2048x1024_P512 = 1.09139e9 * 1023 / 127
UNIT = "probe·slice/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="2d-fwd-adj-2048x1024-p512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-3d", action="store_true", help="skip the 3D learned-vs-plain section")
    ap.add_argument("--ms-nz", type=int, default=0, help="3d-ms case: use the first N z nodes only")
    ap.add_argument("--pairs", choices=("mixed", "noise", "noise20k"), default="mixed",
                    help="training pairs of the learned preconditioner (3D cases)")
    ap.add_argument("--small", action="store_true",
                    help="kernels case: 64 probes for the NLCG pieces and 16 for the multislice (~1 GB on the "
                         "device; the size of the profiler captures)")
    ap.add_argument("--precond", choices=("learned", "fft"), default="learned",
                    help="3d-march-small: the learned correction of the FFT preconditioner, or the plain one")
    ap.add_argument("--step-by-step", action="store_true",
                    help="3D cases: launch the march's kernels step by step instead of as one CUDA graph with "
                         "conditional loops (the same kernels; profilers list the kernels of such graphs only "
                         "as one workload)")
    ap.add_argument("--case", choices=("headline", "3d-march-small", "3d-recon", "3d-ms", "pit", "kernels", "cnn"),
                    default="headline",
                    help="3d-march-small: a few learned 3D forward marches (256 x 256 x 5 nodes, 64 probes), "
                         "a small profiler target for the conv and FFT kernels; 3d-recon: `steps` gradient-descent "
                         "iterations of the 3D reconstruction (192 x 192 x 192, 256 probes), plain vs learned; "
                         "cnn: the learned preconditioner's network on `--cnn-batch` 256 x 256 slices")
    ap.add_argument("--cnn-batch", type=int, default=64, help="cnn case: slices per network launch")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (every 50 ms) of SM clock and throttle reasons.

    Started before the warm-up so that the sampler is running when the timed
    region begins; ``begin()``/``end()`` mark the timed region on the host
    clock and ``summary()`` keeps the rows whose nvidia-smi timestamp falls
    inside it (widened to the whole run, and said so, when the timed region
    is shorter than one sampling interval)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def wait_first(self, limit_s=5.0):
        """Block until the sampler has written one row (or `limit_s` passes)."""
        t = time.time()
        while self.proc is not None and time.time() - t < limit_s:
            if os.path.getsize(self.path) > 0:
                return
            time.sleep(0.02)

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    @staticmethod
    def _stamp(s):
        import datetime

        try:
            return datetime.datetime.strptime(s.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self):
        try:
            rows = [[x.strip() for x in r.split(",")] for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        rows = [r for r in rows if len(r) >= 10]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        window = "timed"
        sel = rows
        if self.t0 is not None and self.t1 is not None:
            sel = [r for r in rows if (ts := self._stamp(r[0])) is not None and self.t0 <= ts <= self.t1]
            if not sel:
                sel, window = rows, "whole run (timed region shorter than the 50 ms sampling interval)"

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [v for v in (num(r[2]) for r in sel) if v is not None]
        mx = [v for v in (num(r[3]) for r in sel) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in sel for i in range(4) if r[6 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sel), "window": window}


# --------------------------------------------------------------------------
# CPU legs (the oracle restatement of the reference's IterativeLU path)
# --------------------------------------------------------------------------
_CPU_CASE = {}


def _cpu_case(N, nz):
    """The 2D workload of size (N, nz) with its step matrices (cached per process)."""
    if (N, nz) not in _CPU_CASE:
        from oracle import pwe_oracle as po
        from thick_ptycho_b200.workloads import CONFIGS

        w = [c for c in CONFIGS.values() if c.nx == N and c.nz == nz and c.dimension == 2][0]
        geo = w.geometry()
        co = po.bc_coefficients(geo.k, 1.0, 1.0, bc_type="impedance")
        A, B = po.step_matrices_1d(N, co, "impedance", 1.0)
        _CPU_CASE[(N, nz)] = (geo, w.delta_n(), w.probes(geo), A, B)
    return _CPU_CASE[(N, nz)]


def _cpu_sample(args):
    """Factorisation + per-probe fwd/adj march time of the CPU restatement over
    the first `S` slices (the costs are linear in the slices).

    The same per-slice arithmetic as the reference's IterativeLU path
    (``build_lu_factors`` then ``march_with_lu``: one SuperLU of A − C_j and
    B + C_j per slice and mode, u_j = LU_j⁻¹(B_j u_{j−1}), the adjoint from
    the exit), but one slice's factor is held at a time: every SuperLU object
    keeps its work memory, and holding all 2 × 1023 of them takes ~7 GB per
    process.  Factorisation and march times are accumulated separately."""
    N, nz, probes_idx, seed, S = args
    from oracle import pwe_oracle as po

    geo, dn, probes, A, B = _cpu_case(N, nz)
    S = min(S, nz - 1)
    C = po.object_contribution(1 - dn[:, : S + 1], geo.k, 1.0)
    t_fact = 0.0
    t_march = 0.0
    exits = []
    for mode in ("forward", "adjoint"):
        states = [probes[p].astype(complex) for p in probes_idx] if mode == "forward" else \
            [np.zeros(N, dtype=complex) for _ in probes_idx]
        for j in range(1, S + 1):
            col = j - 1 if mode == "forward" else S - j  # the slice of step j (adjoint: C[:, -j])
            t0 = time.perf_counter()
            (lu,), (Bw,) = po.build_lu_factors(A, B, C[:, col:col + 1], mode)
            t1 = time.perf_counter()
            for i in range(len(states)):
                b = exits[i] if (mode == "adjoint" and j == 1) else 0.0  # rhs[:, -1] = the exit
                states[i] = lu.solve(Bw @ states[i] + b)
            t_fact += t1 - t0
            t_march += time.perf_counter() - t1
        if mode == "forward":
            exits = list(states)
    return t_fact, t_march / len(probes_idx)


def cpu_rate(N, nz, P, cores, probes_per_worker, slices=None, pool=None):
    """probe·slice/s of the CPU path extrapolated to P probes on `cores` workers
    (from `slices` of the L slices, default all of them, scaled linearly)."""
    L = nz - 1
    S = L if slices is None else max(1, min(int(slices), L))
    jobs = [(N, nz, [(c * 7 + i) % P for i in range(probes_per_worker)], c, S) for c in range(cores)]
    t0 = time.perf_counter()
    if cores == 1:
        res = [_cpu_sample(jobs[0])]
    elif pool is not None:
        res = pool.map(_cpu_sample, jobs)
    else:
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(cores) as p:
            res = p.map(_cpu_sample, jobs)
    wall = time.perf_counter() - t0
    t_fact = statistics.mean(r[0] for r in res) * L / S
    t_probe = statistics.mean(r[1] for r in res) * L / S
    per_worker = -(-P // cores)
    total = t_fact + per_worker * t_probe
    return P * L / total, t_fact, t_probe, wall


def _cpu_quota():
    """The cgroup CPU limit of this process ("quota period"), if readable."""
    for path in ("/sys/fs/cgroup/cpu.max", "/sys/fs/cgroup/cpu/cpu.cfs_quota_us"):
        try:
            with open(path) as f:
                return f.read().strip()
        except OSError:
            continue
    return None


def ref_workers():
    """Worker processes of the reference arm: the host threads this process may
    run on (its affinity mask, not the machine's core count), at most
    REF_MAX_WORKERS."""
    try:
        n = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        n = os.cpu_count() or 1
    return max(1, min(n, REF_MAX_WORKERS))


def run_reference(a):
    """The reference's CPU path (the oracle's restatement of its IterativeLU
    solver: per-slice SuperLU, serial per-probe march, its adjoint) on the host
    cores.  Each step times a sample of S of the L slices on every worker (the
    cost is linear in S; S is sized from a calibration sample so that the run
    takes about REF_BUDGET_S seconds), and the run stops at REF_DEADLINE_S
    whatever `--steps` asks, reporting the steps it finished."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    from thick_ptycho_b200.workloads import CONFIGS

    t_start = time.perf_counter()
    w = CONFIGS[a.config]
    cores = ref_workers()
    L = w.nz - 1
    # one thread per worker process: the reference's SuperLU and sparse products
    # are single-threaded, and BLAS/OpenMP pools in every worker oversubscribe
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS"):
        os.environ[v] = "1"
    budget = REF_BUDGET_S / max(1, a.warmup + a.steps)
    vals = []
    info = None
    S = probe_s = min(L, 16)
    with mp.get_context("spawn").Pool(cores) as pool:

        def rate(S, limit):
            jobs = [(w.nx, w.nz, [(c * 7) % w.num_probes], c, S) for c in range(cores)]
            t0 = time.perf_counter()
            res = pool.map_async(_cpu_sample, jobs).get(timeout=max(1.0, limit))
            wall = time.perf_counter() - t0
            t_fact = statistics.mean(r[0] for r in res) * L / S
            t_probe = statistics.mean(r[1] for r in res) * L / S
            total = t_fact + (-(-w.num_probes // cores)) * t_probe
            return w.num_probes * L / total, t_fact, t_probe, wall

        def left():
            return REF_DEADLINE_S - (time.perf_counter() - t_start)

        t_pool = time.perf_counter() - t_start
        calib0 = rate(probe_s, left())  # also starts the workers
        calib = rate(probe_s, left())
        S = max(8, min(L, int(probe_s * budget / max(calib[3], 1e-3))))
        done = 0
        walls = []
        for i in range(a.warmup + a.steps):
            # stop when the next step would not finish before the deadline
            if left() < 1.5 * (calib[3] * S / probe_s) + 5.0:
                break
            try:
                v, tf, tp, wall = rate(S, left())
            except mp.TimeoutError:
                break
            walls.append((round(time.perf_counter() - t_start - wall, 2), round(wall, 2)))
            if i >= a.warmup:
                vals.append(v)
                info = (tf, tp, wall)
                done += 1
        t_loop = time.perf_counter() - t_start
        pool.terminate()
    t_term = time.perf_counter() - t_start
    if not vals:  # deadline reached during the warm-up: report the calibration sample
        S, info, vals = probe_s, calib[1:], [calib[0]]
    value = statistics.median(vals)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": max(done, 1), "warmup": a.warmup,
        "steps_requested": a.steps, "ms_per_step": 1e3 * w.num_probes * L / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": w.name, "N": w.nx, "nz": w.nz, "probes": w.num_probes},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": (f"per step: {cores} spawn workers (one thread each) each factorise the first {S} "
                                    f"of {L} slices (forward + reference adjoint SuperLU) and march 1 probe fwd+adj "
                                    f"over them; rate scaled to {L} slices and {w.num_probes} probes split over "
                                    f"{cores} workers (last, scaled: factor {info[0]:.2f} s, probe {info[1]:.3f} s; "
                                    f"step wall {info[2]:.2f} s)")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t_start,
        "timing_s": {"pool_start": round(t_pool, 2), "calibration": [round(calib0[3], 2), round(calib[3], 2)],
                     "slices_per_step": S, "step_start_and_wall": walls, "loop_end": round(t_loop, 2),
                     "pool_closed": round(t_term, 2), "cpu_quota": _cpu_quota()},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# 3D: learned vs plain FFT-preconditioned BiCGStab (fwd + exact adjoint)
# --------------------------------------------------------------------------
PAIR_KINDS = {
    "mixed": "10 200 white-noise pairs (x, (I - P_s) x) and 10 200 step pairs (the step's right-hand side, its "
             "converged update), 40 probes x 255 slices each, of a different seeded field",
    "noise": "10 200 white-noise pairs (x, (I - P_s) x), 40 probes x 255 slices, of a different seeded field",
    "noise20k": "20 400 white-noise pairs (x, (I - P_s) x), 80 probe slots x 255 slices, of a different seeded "
                "field",
}


def train_learned(eng, geo, w, probes, kind, steps, dev):
    """The learned preconditioner trained on solver-generated pairs of another
    seeded field (`kind`, see PAIR_KINDS); returns the model and what it was
    trained on.  Not timed."""
    import torch

    from thick_ptycho_b200.cn3d import generate_pairs
    from thick_ptycho_b200.learned import LearnedPreconditioner, default_kappa
    from thick_ptycho_b200.workloads import ellipsoid_field_3d

    n, nz = w.nx, w.nz
    t0 = time.perf_counter()
    ftrain = torch.from_numpy((1 - ellipsoid_field_3d(n, n, nz, w.n_shapes, 1001)).reshape(n * n, nz)).to(dev)
    sets = []
    if kind in ("noise", "mixed"):
        sets.append(generate_pairs(eng, ftrain, probes[:40].contiguous(), every=1, kind="noise"))
    if kind == "mixed":
        sets.append(generate_pairs(eng, ftrain, probes[-40:].contiguous(), every=1, kind="rhs"))
    if kind == "noise20k":
        slots = torch.cat([probes, probes])[:80].contiguous()
        sets.append(generate_pairs(eng, ftrain, slots, every=1, kind="noise"))
    del ftrain
    model = LearnedPreconditioner(n, n, default_kappa(geo.k, 1.0, 5e-4), device=dev, seed=0)
    model.train(sets, steps=steps * len(sets), slices_per_batch=2, lr=1e-3)
    torch.cuda.synchronize(dev)
    info = {"pairs": sum(ps.count for ps in sets), "kind": PAIR_KINDS[kind], "steps": steps * len(sets),
            "seconds": time.perf_counter() - t0, "not_timed": True}
    del sets
    torch.cuda.empty_cache()
    return model, info


def fixture_exit_error(name, ex):
    """Relative L2 error of the exit waves `ex` (P, N) against the complex128
    oracle fixture of the geometry (its three checked probes)."""
    with np.load(os.path.join(ROOT, "tests", "golden", f"{name}_3d_full.npz")) as g:
        idx, ref = [int(i) for i in g["probe_idx"]], g["exit"].astype(np.complex128)
    got = ex[idx].cpu().numpy().astype(np.complex128)
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


def bench_learned_3d(dev, reps=2, train_steps=1500, pairs="mixed"):
    """fwd + adj probe·slice solves/s of the plain and the learned 3D forms.

    Workload: 256 x 256 transverse x 256 nodes, 64 probes (8 x 8 raster,
    stride 16, waist 12), δn = 400 seeded ellipsoids + 1e-6 i, impedance
    edges, BiCGStab to a 1e-6 relative residual per solve.  One step = a
    forward march storing the full field + an exact-adjoint march with the
    fused gradient, all 64 probes batched.  The network is trained first on
    solver-generated pairs of a different seeded field (`pairs`, see
    PAIR_KINDS); training time is reported, not timed.  Each form's exit
    waves are compared with the complex128 oracle fixture of the geometry.
    """
    import torch

    from thick_ptycho_b200.cn3d import CN3D
    from thick_ptycho_b200.workloads import CONFIG2

    w = CONFIG2
    geo = w.geometry()
    nz, P, n = w.nz, w.num_probes, w.nx
    N, L = n * n, nz - 1
    eng = CN3D(n, n, nz, geo.k, 1.0, 1.0, 1.0, "impedance", device=dev)
    field = torch.from_numpy((1 - w.delta_n()).reshape(N, nz)).to(dev)
    probes = torch.from_numpy(w.probes(geo).reshape(P, N).astype(np.complex64)).to(dev)
    stream = torch.cuda.current_stream(dev)

    model, training = train_learned(eng, geo, w, probes, pairs, train_steps, dev)

    store = eng.new_store(P)
    ex = torch.empty((P, N), dtype=torch.complex64, device=dev)
    grad = torch.zeros((L, N), dtype=torch.complex64, device=dev)
    out = {}
    exits = {}
    for name, pc in (("plain", True), ("learned", "learned")):
        ms = []
        eng.read_stats()
        for rep in range(reps + 1):
            if rep == 1:
                eng.read_stats()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            grad.zero_()
            e0.record(stream)
            eng.march(field, P, "forward", probes=probes, u_store=store, exit_out=ex, precond=pc, model=model)
            eng.march(field, P, "adjoint_exact", src_exit=ex, u_fwd=store, grad_c=grad, precond=pc, model=model,
                      reuse_filters=True)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if rep >= 1:
                ms.append(e0.elapsed_time(e1))
        st = eng.read_stats()
        t = statistics.median(ms)
        exits[name] = ex.clone()
        out[name] = {"value": P * L / (t / 1e3), "ms_per_step": t,
                     "krylov_iterations_per_solve": st["iterations"] / max(st["solves"], 1),
                     "failed_solves": st["failed"], "graph": st["graph"],
                     "exit_rel_error_vs_fp64_fixture": fixture_exit_error("config2", ex)}
    diff = float(torch.linalg.vector_norm(exits["learned"] - exits["plain"]) / torch.linalg.vector_norm(exits["plain"]))
    return {
        "workload": w.name, "metric": "probe·slice solves/s fwd+adj (3D BiCGStab, exact adjoint + gradient)",
        "unit": UNIT, "plain": out["plain"], "learned": out["learned"],
        "learned_over_plain": out["learned"]["value"] / out["plain"]["value"],
        "exit_rel_diff_learned_vs_plain": diff, "fallbacks": eng.fallbacks, "training": training,
    }


# --------------------------------------------------------------------------
# GPU leg
# --------------------------------------------------------------------------
def run_ours(a):
    import torch

    from thick_ptycho_b200.gradient import PWEGradient2D, amplitude_residual
    from thick_ptycho_b200.workloads import CONFIGS

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    w = CONFIGS[a.config]
    geo = w.geometry()
    N, nz, P, L = w.nx, w.nz, w.num_probes, w.nz - 1
    dn = w.delta_n()
    n_ref = 1 - dn                      # the reference PWE's index convention
    probes = w.probes(geo)
    # measured amplitudes: the same probes through a perturbed truth (host-side, seeded)
    amp = np.abs(np.fft.fft(probes, axis=-1)) * 1.01

    pg = PWEGradient2D(geo, "impedance", device=dev)
    eng = pg.engine
    field = torch.from_numpy(n_ref).to(dev)
    pr = torch.from_numpy(probes.astype(np.complex64)).to(dev)
    amp_d = torch.from_numpy(amp).to(dev)
    ex = torch.empty((P, N), dtype=torch.complex64, device=dev)
    store = eng.new_store(P)
    gc = eng.new_grad_buffer()
    ff_buf, fa_buf = eng.new_factor_buffer(), eng.new_factor_buffer()
    stream = torch.cuda.current_stream(dev)
    ev = {k: [] for k in ("fwd", "adj")}

    def step(record):
        ff = eng.factor(field, "forward", out=ff_buf)
        if record:
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        eng.march(ff, P, probes=pr, u_store=store, exit_out=ex, store_sums=True)
        if record:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(stream)
        _, ge = amplitude_residual(ex, amp_d)
        fa = eng.factor(field, "adjoint_exact", out=fa_buf)
        gc.zero_()
        if record:
            e2 = torch.cuda.Event(enable_timing=True)
            e2.record(stream)
        eng.march(fa, P, src_exit=ge, u_fwd=store, grad_c=gc, store_sums=True)
        if record:
            e3 = torch.cuda.Event(enable_timing=True)
            e3.record(stream)
            ev["fwd"].append((e0, e1))
            ev["adj"].append((e2, e3))
        g = eng.grad_to_n(gc)
        if dist is not None:
            dist.all_reduce(torch.view_as_real(g))
        return g

    with ClockSampler(local) as clk:
        clk.wait_first()
        for _ in range(a.warmup):
            step(False)
        eng.device_status()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        clk.begin()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(a.steps):
            step(True)
        t1.record(stream)
        torch.cuda.synchronize()
        clk.end()
        if dist is not None:
            dist.barrier()
    eng.device_status()
    ms = t0.elapsed_time(t1)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * P * L * a.steps / (ms_max / 1e3)
    fwd_ms = statistics.mean(s.elapsed_time(e) for s, e in ev["fwd"])
    adj_ms = statistics.mean(s.elapsed_time(e) for s, e in ev["adj"])

    # ---- e2e through the public API with pinned host buffers
    n_h = torch.from_numpy(n_ref).pin_memory()
    p_h = torch.from_numpy(probes.astype(np.complex64)).pin_memory()
    a_h = torch.from_numpy(amp).pin_memory()
    g_h = torch.empty((N, nz), dtype=torch.complex64).pin_memory()
    for _ in range(max(1, a.warmup)):
        pg.loss_and_grad(n_h, p_h, a_h, grad_out=g_h)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e_steps = max(3, a.steps // 2)
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(e_steps):
        pg.loss_and_grad(n_h, p_h, a_h, grad_out=g_h)  # loss.item() reads the result back each step
    s1.record(stream)
    torch.cuda.synchronize()
    e_ms = torch.tensor([s0.elapsed_time(s1)], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(e_ms, op=dist.ReduceOp.MAX)
    e2e = world * P * L * e_steps / (float(e_ms.item()) / 1e3)
    h2d = n_h.numel() * 16 + p_h.numel() * 8 + a_h.numel() * 8
    d2h = g_h.numel() * 8 + 8

    if rank == 0:
        hbm, kind = peaks()
        slice_fac = eng.factor_bytes / L
        fwd_bytes = P * L * 8 * eng.npad + L * slice_fac        # full-field write + factor stream
        adj_bytes = P * L * 8 * eng.npad + L * slice_fac + L * N * 8   # field read + factors + gradient
        dom = "adj" if adj_ms >= fwd_ms else "fwd"
        dom_bytes, dom_ms = (adj_bytes, adj_ms) if dom == "adj" else (fwd_bytes, fwd_ms)
        achieved = dom_bytes / (dom_ms / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64", "data": "synthetic (seeded Gaussian blobs and probes)",
            "config": {"workload": w.name, "N": N, "nz": nz, "probes_per_gpu": P, "bc": "impedance",
                       "l2": "working set 8.6 GB > L2 (no flush needed)", "parallelism": f"probe-shard x{world}"},
            "kernels_ms": {"cn2d_march_forward": fwd_ms, "cn2d_march_adjoint_exact_grad": adj_ms,
                           "step_total": ms_max / a.steps},
            "roofline": {"kernel": ("cn2d_team_kernel (" if eng.chunks == 128 else "cn2d_march_kernel (")
                         + ("adjoint_exact+grad" if dom == "adj" else "forward") + ")",
                         "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": kind,
                         "traffic": (ADJ_TRAFFIC_BYTES_2048x1024_P512
                                     if dom == "adj" and (N, nz, P) == (2048, 1024, 512) else None),
                         "algorithmic_bytes_per_launch": dom_bytes},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            # per step: 2 factorisations, 2 marches, the amplitude residual, the node mapping
            "gpu_launches": a.steps * 6,
            "clocks": clk.summary(),
        }
        if world == 1 and not a.no_3d:
            line["learned_vs_plain_3d"] = bench_learned_3d(dev, pairs=a.pairs)
        if world == 1 and not a.no_cpu_baseline:
            v, tf, tp, wall = cpu_rate(N, nz, P, 1, 2)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                    "sample": (f"CPU restatement of the reference IterativeLU path: factorise {L} "
                                               f"slices forward + adjoint ({tf:.2f} s) and march 2 probes fwd+adj "
                                               f"({tp:.3f} s/probe); extrapolated to {P} probes")}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_case_3d_small(a):
    """`steps` 3D forward marches on 256 x 256 x 5 nodes, 64 probes (config-2 probes and ellipsoid
    distribution), after `warmup` untimed ones; learned form with an untrained network (seeded), or the
    plain FFT preconditioner (`--precond fft`)."""
    import torch

    from thick_ptycho_b200.cn3d import CN3D
    from thick_ptycho_b200.learned import LearnedPreconditioner, default_kappa
    from thick_ptycho_b200.workloads import CONFIG2, ellipsoid_field_3d

    w = CONFIG2
    nz = 5
    geo = w.geometry()
    dev = torch.device("cuda", 0)
    eng = CN3D(w.nx, w.nx, nz, geo.k, 1.0, 1.0, 1.0, "impedance", device=dev)
    P = w.num_probes
    probes = torch.from_numpy(w.probes(geo).reshape(P, -1).astype(np.complex64)).to(dev)
    field = torch.from_numpy((1 - ellipsoid_field_3d(w.nx, w.nx, nz, 10, w.seed)).reshape(-1, nz)).to(dev)
    model = LearnedPreconditioner(w.nx, w.nx, default_kappa(geo.k, 1.0, 5e-4), device=dev, seed=0)
    ex = torch.empty((P, eng.N), dtype=torch.complex64, device=dev)
    eng.launch = 1 if a.step_by_step else 0
    ms = []
    for i in range(a.warmup + a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.march(field, P, "forward", probes=probes, exit_out=ex, precond=a.precond if a.precond == "learned" else True,
                  model=model)
        e1.record()
        torch.cuda.synchronize()
        if i >= a.warmup:
            ms.append(e0.elapsed_time(e1))
    print(json.dumps({"case": "3d-march-small", "precond": a.precond, "ms_per_march": statistics.median(ms) if ms else None,
                      "stats": eng.read_stats()}), flush=True)


def run_case_3d_ms(a):
    """3D multislice (the reference's multislice is 2D only) on the 256 x 256 x 256-node,
    64-probe geometry with n = 1 + δn (400 seeded ellipsoids): forward march to the exit
    plane, forward march keeping the field, adjoint march with the gradient; CUDA-event
    medians over `steps` after `warmup`, plus the complex128 numpy restatement timed on one
    probe for 8 slices."""
    import torch

    from oracle import pwe_oracle as po
    from thick_ptycho_b200.ms3d import MS3D
    from thick_ptycho_b200.workloads import CONFIG2

    w = CONFIG2
    geo = w.geometry()
    dev = torch.device("cuda", 0)
    nx, nz, P = w.nx, w.nz, w.num_probes
    n = 1 + w.delta_n()
    if a.ms_nz:  # fewer slices of the same field (small profiling captures)
        nz = int(a.ms_nz)
        n = np.ascontiguousarray(n[:, :, :nz])
    eng = MS3D(nx, nx, nz, geo.k, 1.0, 1.0, 1.0, device=dev)
    T = eng.transmission(torch.from_numpy(n.reshape(-1, nz)).to(dev))
    probes_np = w.probes(geo).reshape(P, -1).astype(np.complex64)
    probes = torch.from_numpy(probes_np).to(dev)
    ex = torch.empty((P, eng.N), dtype=torch.complex64, device=dev)
    st = torch.empty((P, nz, eng.N), dtype=torch.complex64, device=dev)
    gt = torch.zeros((eng.L, eng.N), dtype=torch.complex64, device=dev)
    rng = np.random.default_rng(3)
    src = torch.from_numpy((rng.standard_normal((P, eng.N)) + 1j * rng.standard_normal((P, eng.N))).astype(np.complex64)).to(dev)
    runs = {"forward_exit": lambda: eng.march(T, probes, exit_out=ex),
            "forward_store": lambda: eng.march(T, probes, u_store=st, exit_out=ex),
            "adjoint_grad": lambda: eng.backward(T, st, src, gt)}
    ms = {k: [] for k in runs}
    for i in range(a.warmup + a.steps):
        for key, fn in runs.items():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            if i >= a.warmup:
                ms[key].append(e0.elapsed_time(e1))
    med = {k: statistics.median(v) for k, v in ms.items()}
    ps = P * eng.L
    t0 = time.perf_counter()
    po.ms_forward_3d(n[:, :, :9], probes_np[0].reshape(nx, nx).astype(complex), geo.k, 1.0, 1.0, 1.0)
    cpu_s = (time.perf_counter() - t0) / 8
    print(json.dumps({"case": "3d-ms", "workload": f"3d-ms-{nx}x{nx}x{nz}-p{P}", "ms": med,
                      "probe_slices_per_s": {k: ps / (v * 1e-3) for k, v in med.items()},
                      "fwd_adj_probe_slices_per_s": ps / ((med["forward_store"] + med["adjoint_grad"]) * 1e-3),
                      "cpu_oracle_s_per_probe_slice": cpu_s,
                      "launches_per_march": 2 * eng.L + 1 + 3}), flush=True)


def run_case_pit(a):
    """PiT space-time GMRES (the reference's PWEFullPinTSolver) on the GPU: config 0
    (N = 256, nz = 128, 32 probes) and the config-1 geometry (N = 2048, nz = 1024) with
    8 probes; CUDA-event medians of `steps` solves after `warmup`, Arnoldi steps per
    probe, and the complex128 restatement of the reference's solver (scipy GMRES,
    splu blocks) timed on two config-0 probes on one host core."""
    import torch

    from oracle import pwe_oracle as po
    from thick_ptycho_b200.cn2d import CN2D
    from thick_ptycho_b200.pit import PiT2D
    from thick_ptycho_b200.workloads import CONFIG0, CONFIG1

    dev = torch.device("cuda", 0)
    out = {"case": "pit"}
    for w, P in ((CONFIG0, 32), (CONFIG1, 8)):
        geo = w.geometry()
        n = 1 - w.delta_n()
        probes = w.probes(geo)[:P]
        eng = CN2D(w.nx, w.nz, geo.k, 1.0, 1.0, "impedance", device=dev)
        pit = PiT2D(eng)
        field = torch.from_numpy(n).to(dev)
        pr = torch.from_numpy(probes.astype(np.complex64)).to(dev)
        ms = []
        for i in range(a.warmup + a.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            pit.solve(field, probes=pr)
            e1.record()
            torch.cuda.synchronize()
            if i >= a.warmup:
                ms.append(e0.elapsed_time(e1))
        med = statistics.median(ms)
        out[f"{w.nx}x{w.nz}-p{P}"] = {"ms_per_solve": med, "arnoldi_steps": sorted(set(pit.iters)),
                                       "max_resid": max(pit.resid),
                                       "probe_slices_per_s": P * (w.nz - 1) / (med * 1e-3)}
    w = CONFIG0
    geo = w.geometry()
    co = po.bc_coefficients(geo.k, 1.0, 1.0, bc_type="impedance")
    A, B = po.step_matrices_1d(w.nx, co, "impedance", 1.0)
    C = po.object_contribution(1 - w.delta_n(), geo.k, 1.0)
    t0 = time.perf_counter()
    _, its = po.pit_solve(A, B, C, w.probes(geo)[:2])
    cpu = (time.perf_counter() - t0) / 2
    out["cpu_reference_restatement"] = {"s_per_probe": cpu, "gmres_iterations": its, "cores": 1,
                                        "sample": "config 0, 2 probes (preconditioner set-up included)"}
    print(json.dumps(out), flush=True)


def run_case_3d_recon(a):
    """3D reconstruction, 192 x 192 transverse x 192 nodes, 256 probes (16 x 16 raster, stride 10,
    waist 12), ground truth δn = 600 seeded ellipsoids + 1e-6 i, data = |FFT2(exit)| of the truth;
    `steps` gradient-descent iterations from δn = 0 with the plain FFT preconditioner and with the
    learned one in the forward and adjoint marches (network trained on white-noise pairs of another
    seeded field, not timed).  Reports fwd+adj probe·slice/s of each run, Krylov iterations per
    solve, the loss histories, the final δn error against the truth and learned vs plain."""
    import torch

    from thick_ptycho_b200 import heads
    from thick_ptycho_b200.cn3d import CN3D, PWEGradient3D, generate_pairs
    from thick_ptycho_b200.learned import LearnedPreconditioner, default_kappa
    from thick_ptycho_b200.reconstruct import gradient_descent_3d
    from thick_ptycho_b200.workloads import CONFIG4, ellipsoid_field_3d

    w = CONFIG4
    geo = w.geometry()
    dev = torch.device("cuda", 0)
    n, nz, P = w.nx, w.nz, w.num_probes
    N, L = n * n, nz - 1
    dn_true = w.delta_n().reshape(N, nz)
    probes = torch.from_numpy(w.probes(geo).reshape(P, N).astype(np.complex64)).to(dev)
    truth = PWEGradient3D(geo, device=dev)
    ex = truth.forward(torch.from_numpy(1 - dn_true).to(dev), probes)
    amp = heads.fft2_last(ex.reshape(P, n, n).contiguous()).abs().to(torch.float64)
    fixture_err = {"plain": fixture_exit_error("config4", ex)}
    del truth, ex
    eng = CN3D(n, n, nz, geo.k, 1.0, 1.0, 1.0, "impedance", device=dev)
    model, training = train_learned(eng, geo, w, probes, a.pairs, 1500, dev)
    del eng
    # the learned form's exit waves of the ground truth against the same fixture
    lt = PWEGradient3D(geo, device=dev, precond="learned", model=model)
    fixture_err["learned"] = fixture_exit_error("config4", lt.forward(torch.from_numpy(1 - dn_true).to(dev), probes))
    del lt
    n0 = np.ones((N, nz), dtype=complex)
    res = {}
    for name, pc in (("plain", True), ("learned", "learned")):
        g3 = PWEGradient3D(geo, device=dev, precond=pc, model=model)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record()
        nk, losses, its = gradient_descent_3d(g3, n0, probes, amp, iters=a.steps)
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        dn = (1 - nk).cpu().numpy()  # the reference PWE index convention n = 1 − δn
        res[name] = {"value": a.steps * P * L / (ms / 1e3), "unit": UNIT, "ms_total": ms,
                     "krylov_iterations_per_solve": float(np.mean(its)), "loss_first": losses[0],
                     "loss_last": losses[-1],
                     "delta_n_rel_error_vs_truth": float(np.linalg.norm(dn - dn_true) / np.linalg.norm(dn_true)),
                     "fallbacks": g3.engine.fallbacks, "_n": nk}
    diff = float(torch.linalg.vector_norm(res["learned"]["_n"] - res["plain"]["_n"]) /
                 torch.linalg.vector_norm(res["plain"]["_n"] - torch.from_numpy(n0).to(dev)))
    for r in res.values():
        r.pop("_n")
    print(json.dumps({"case": "3d-recon", "workload": w.name, "iterations": a.steps,
                      "metric": "probe·slice solves/s fwd+adj (3D gradient descent)", "plain": res["plain"],
                      "learned": res["learned"], "learned_over_plain": res["learned"]["value"] / res["plain"]["value"],
                      "n_diff_learned_vs_plain_rel_update": diff,
                      "truth_exit_rel_error_vs_fp64_fixture": fixture_err, "training": training}),
          flush=True)


def run_case_cnn(a):
    """The learned preconditioner's network (features and four tcgen05 3x3
    convolutions) on `cnn_batch` seeded 256 x 256 object diagonals -- one chunk
    of the learned march's slices: CUDA-event median of `steps` forwards after
    `warmup`, with the FLOPs of the four layers."""
    import torch

    from thick_ptycho_b200.learned import LearnedPreconditioner

    B = a.cnn_batch
    m = LearnedPreconditioner(256, 256, 1.0, seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    d = (1e-3 * torch.randn((B, 65536), dtype=torch.complex64, device="cuda", generator=g)).contiguous()
    for _ in range(max(1, a.warmup)):
        m.filter(d)
    torch.cuda.synchronize()
    ms = []
    for _ in range(max(1, a.steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        m.filter(d)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = statistics.median(ms)
    flop = 2 * 65536 * 9 * 32 * (16 + 3 * 32) * B
    print(json.dumps({"case": "cnn", "batch": B, "ms": t, "tflops": flop / (t * 1e-3) / 1e12}), flush=True)


def run_case_kernels(a):
    """The kernels around the marches, each on a workload larger than L2 where
    its data allows, timed with CUDA events (median of `steps` launches after
    `warmup`) against its algorithmic bytes (or, for the network's weight
    gradients, FLOPs): the target workload of their profiler captures.

    * cn2d_factor_kernel: forward factor set of the 2048 x 1024 geometry
      (reads two index columns per slice, complex128; writes 1023 slices);
    * cn2d_grad_to_n_kernel: its gradient buffer mapped onto the index nodes;
    * cn2d_refgrad_kernel / cn2d_alpha_source_kernel: the reference NLCG's
      gradient contraction and step-size source on the 1024 x 512 geometry,
      256 probes (reading stored forward and adjoint fields of 1.07 GB each);
    * ms_march_kernel / ms_backward_kernel: 2D multislice, 2048 x 1024, 64
      probes, forward keeping the field (1.07 GB) and the adjoint with the
      gradient;
    * ms_3pie_kernel: one 3PIE epoch of the 256 x 128 geometry, 32 probes (one
      persistent CTA: sequential over probes, latency-bound);
    * conv3x3_wgrad_kernel: weight gradients of the learned preconditioner's
      four layers on 8 images of 256 x 256.

    ``--small``: 64 of the NLCG probes and 16 multislice probes (stored fields
    of 268 MB, still larger than L2).
    """
    import torch

    from thick_ptycho_b200.cn2d import CN2D
    from thick_ptycho_b200.learned import LearnedPreconditioner, default_kappa
    from thick_ptycho_b200.ms2d import MS2D, ReconstructorMSGpu
    from thick_ptycho_b200.reconstruct import ReconstructorPWEGpu
    from thick_ptycho_b200.workloads import CONFIG0, CONFIG1, CONFIG3

    dev = torch.device("cuda", 0)
    hbm, kind = peaks()
    out = {"case": "kernels", "peak_gbs": hbm, "peak_kind": kind}

    def timed(fn):
        for _ in range(max(1, a.warmup)):
            fn()
        ms = []
        for _ in range(max(1, a.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    def report(name, ms, nbytes, note):
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "algorithmic_bytes": nbytes, "achieved_gbs": gbs, "frac": gbs / hbm, "note": note}

    # 2D factorisation and node mapping, 2048 x 1024
    w = CONFIG1
    geo = w.geometry()
    eng = CN2D(w.nx, w.nz, geo.k, 1.0, 1.0, "impedance", device=dev)
    field = torch.from_numpy(1 - w.delta_n()).to(dev)
    fbuf = eng.new_factor_buffer()
    ms = timed(lambda: eng.factor(field, "forward", out=fbuf))
    report("cn2d_factor_kernel", ms, 2 * w.nx * (w.nz - 1) * 16 + eng.factor_bytes,
           "1023 slices of 2048 rows: fp64 elimination per chunk, PCR records; writes the factor set")
    gc = eng.new_grad_buffer()
    gc.copy_(torch.randn_like(gc))
    gn = torch.empty((w.nx, w.nz), dtype=torch.complex64, device=dev)
    ms = timed(lambda: eng.grad_to_n(gc))
    report("cn2d_grad_to_n_kernel", ms, gc.numel() * 8 + gn.numel() * 8, "reads grad_c (L, Npad), writes (N, nz)")
    del fbuf, gc, gn, field, eng
    # reference NLCG pieces, 1024 x 512, 256 probes
    w = CONFIG3
    geo = w.geometry()
    probes = w.probes(geo)[: 64 if a.small else w.num_probes]
    rec = ReconstructorPWEGpu(geo, np.abs(np.fft.fft(probes, axis=-1)) ** 2, probes, device=dev)
    nk = torch.from_numpy(1 - w.delta_n()).to(dev)
    ff = rec.forward_model(nk)
    err = rec.exit_error()
    rec.gradient(nk, err)
    e = rec.engine
    P = rec.P
    u_bytes = rec._u.numel() * 8
    ms = timed(lambda: e.lib.tp_cn2d_ref_gradient(e.op(), P, ctypes.c_void_p(rec._u.data_ptr()),
                                                  ctypes.c_void_p(rec._lam.data_ptr()),
                                                  ctypes.c_void_p(rec._gre.data_ptr()),
                                                  ctypes.c_void_p(rec._gim.data_ptr()),
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    report("cn2d_refgrad_kernel", ms, 2 * u_bytes + 2 * rec._gre.numel() * 4,
           f"reads the stored forward and adjoint fields ({P} probes), writes grad_re, grad_im")
    ms = timed(lambda: e.lib.tp_cn2d_alpha_source(e.op(), P, ctypes.c_void_p(rec._u.data_ptr()),
                                                  ctypes.c_void_p(rec._src.data_ptr()),
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    report("cn2d_alpha_source_kernel", ms, u_bytes + rec._src.numel() * 8,
           "reads the stored forward field, writes the per-probe source (P, L, N)")
    del rec, nk, ff, err
    torch.cuda.empty_cache()
    # 2D multislice, 2048 x 1024, 64 probes
    w = CONFIG1
    geo = w.geometry()
    P = 16 if a.small else 64
    ms2 = MS2D(w.nx, w.nz, geo.k, 1.0, 1.0, device=dev)
    T = ms2.transmission(torch.from_numpy(1 + w.delta_n()).to(dev))
    pr = torch.from_numpy(w.probes(geo)[:P].astype(np.complex64)).to(dev)
    st = torch.empty((P, w.nz, w.nx), dtype=torch.complex64, device=dev)
    ex = torch.empty((P, w.nx), dtype=torch.complex64, device=dev)
    ms = timed(lambda: ms2.march(T, pr, u_store=st, exit_out=ex))
    report("ms_march_kernel", ms, st.numel() * 8 + T.numel() * 8,
           f"{P} probes x 1023 slices: two shared-memory FFTs per slice, writes the field")
    gt = torch.zeros((w.nz - 1, w.nx), dtype=torch.complex64, device=dev)
    ms = timed(lambda: ms2.backward(T, st, ex, gt))
    report("ms_backward_kernel", ms, st.numel() * 8 + T.numel() * 8 + gt.numel() * 8,
           "reads the forward field, accumulates the transmission gradient")
    del st, gt, T, ms2
    torch.cuda.empty_cache()
    # 3PIE, 256 x 128, 32 probes (sequential)
    w = CONFIG0
    geo = w.geometry()
    probes = w.probes(geo)
    data = np.abs(np.fft.fft(probes, axis=-1)) ** 2
    pie = ReconstructorMSGpu(w.nx, w.nz, geo.k, 1.0, 1.0, data, probes, device=dev)
    ms = timed(lambda: pie.reconstruct(max_iters=1, alpha_obj=0.1))
    out["ms_3pie_kernel"] = {"ms": ms, "probe_slices_per_s": w.num_probes * (w.nz - 1) / (ms * 1e-3),
                             "note": "one CTA, 32 probes in sequence, forward + modulus + backward per probe"}
    # learned-preconditioner weight gradients, 8 images of 256 x 256
    nf = 256
    model = LearnedPreconditioner(nf, nf, default_kappa(4 * np.pi, 1.0, 5e-4), device=dev, seed=0)
    B = 8
    g = torch.Generator(device=dev).manual_seed(0)
    diag = (1e-3 * torch.randn((B, nf * nf), dtype=torch.complex64, device=dev, generator=g)).contiguous()
    z = torch.randn((B, nf * nf), dtype=torch.complex64, device=dev, generator=g)
    tgt = torch.randn((B, nf * nf), dtype=torch.complex64, device=dev, generator=g)
    scale = torch.ones(B, dtype=torch.float32, device=dev)
    ms = timed(lambda: model.loss_and_grads(diag, z, tgt, scale, 1))
    flops = 2 * B * nf * nf * 9 * (16 * 32 + 3 * 32 * 32)
    out["cnn_loss_and_grads"] = {"ms": ms, "wgrad_flops": flops,
                                 "note": "filter, filter gradient, 3 masked data-gradient convs, 4 weight gradients"}
    print(json.dumps(out), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.case == "3d-march-small":
        run_case_3d_small(a)
    elif a.case == "3d-recon":
        run_case_3d_recon(a)
    elif a.case == "3d-ms":
        run_case_3d_ms(a)
    elif a.case == "pit":
        run_case_pit(a)
    elif a.case == "kernels":
        run_case_kernels(a)
    elif a.case == "cnn":
        run_case_cnn(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
