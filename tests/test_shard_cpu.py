"""Probe sharding and the gradient all-reduce of the multi-GPU path, on two
gloo ranks on the CPU: each rank computes the exact-adjoint gradient of its
own probe block with the complex128 oracle, ``parallel.allreduce_gradient``
sums them, and the result must equal the single-process gradient over all
probes (to round-off, 1e-12 relative)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from thick_ptycho_b200.parallel import allreduce_gradient, probe_range


def test_probe_range_partitions():
    for P in (0, 1, 5, 7, 512):
        for W in (1, 2, 3, 8):
            blocks = [probe_range(P, W, r) for r in range(W)]
            assert blocks[0][0] == 0 and blocks[-1][1] == P
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        probe_range(4, 2, 2)


def _problem():
    from oracle import pwe_oracle as po

    rng = np.random.default_rng(7)
    N, nz, P, k = 24, 7, 5, 4 * np.pi
    n = 1 + 2e-3 * (rng.standard_normal((N, nz)) + 0.1j * rng.standard_normal((N, nz)))
    probes = np.exp(-((np.arange(N)[None] - rng.uniform(4, 20, (P, 1))) ** 2) / 9.0).astype(complex)
    target = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    co = po.bc_coefficients(k, 1.0, 1.0, bc_type="impedance")
    A, B = po.step_matrices_1d(N, co, "impedance", 1.0)
    C = po.object_contribution(n, k, 1.0)
    return po, A, B, C, probes, target


def _shard_grad(start, stop):
    """Σ_p gradient of ‖exit_p − target_p‖² w.r.t. the step coefficients, p in [start, stop)."""
    po, A, B, C, probes, target = _problem()
    g = np.zeros_like(C)
    loss = 0.0
    for p in range(start, stop):
        u = po.march(A, B, C, probes[p])
        r = u[:, -1] - target[p]
        loss += float(np.sum(np.abs(r) ** 2))
        src = np.zeros_like(C)
        src[:, -1] = 2 * r
        g += po.grad_c_from_adjoint(u, po.exact_adjoint(A, B, C, src))
    return g, loss


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = 5
        start, stop = probe_range(P, world, rank)
        g, loss = _shard_grad(start, stop)
        gt = torch.from_numpy(g)
        gt, loss = allreduce_gradient(gt, loss)
        if rank == 0:
            out.put((gt.numpy(), loss))
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_equals_full_gradient_two_gloo_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(2, port, q), nprocs=2, join=True, start_method="spawn")
    g_sh, loss_sh = q.get()
    g_full, loss_full = _shard_grad(0, 5)
    assert np.linalg.norm(g_sh - g_full) <= 1e-12 * np.linalg.norm(g_full)
    assert loss_sh == pytest.approx(loss_full, rel=1e-12)
