"""Probe sharding across ranks (one process per GPU).

The paraxial path shards by probe: given δn, every probe's forward march and
adjoint march are independent, so rank r of W takes a contiguous block of the
probes (the reference's scan order, ``simulation_space_2d.py:107-110``,
kept), replicates δn, and the only exchange is the sum of the per-rank
gradients and losses — one all-reduce per reconstruction step (NCCL on GPUs,
gloo on the CPU).  No kernel waits on another rank.
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch


def probe_range(num_probes: int, world: int, rank: int) -> Tuple[int, int]:
    """[start, stop) of rank `rank`'s probes: contiguous blocks whose sizes
    differ by at most one, the first ``num_probes % world`` ranks one larger."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    if num_probes < 0:
        raise ValueError("num_probes must be >= 0")
    base, extra = divmod(num_probes, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def allreduce_gradient(grad: torch.Tensor, loss: float, group=None) -> Tuple[torch.Tensor, float]:
    """Sum a complex gradient and a scalar loss over the ranks of `group` (in place for `grad`)."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return grad, float(loss)
    if grad.is_complex():
        dist.all_reduce(torch.view_as_real(grad), group=group)
    else:
        dist.all_reduce(grad, group=group)
    lt = torch.tensor([float(loss)], dtype=torch.float64, device=grad.device)
    dist.all_reduce(lt, group=group)
    return grad, float(lt.item())


class ShardedGradient2D:
    """``PWEGradient2D.loss_and_grad`` over this rank's probe block, summed over ranks."""

    def __init__(self, geometry, bc_type="impedance", device=None, group=None):
        import torch.distributed as dist

        from .gradient import PWEGradient2D

        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.inner = PWEGradient2D(geometry, bc_type, device=device)

    def loss_and_grad(self, n, probes, amplitude, grad_out: Optional[torch.Tensor] = None):
        start, stop = probe_range(probes.shape[0], self.world, self.rank)
        if stop > start:
            loss, grad = self.inner.loss_and_grad(n, probes[start:stop], amplitude[start:stop])
        else:  # more ranks than probes: this rank contributes nothing
            eng = self.inner.engine
            loss, grad = 0.0, torch.zeros((eng.n_obj, eng.nz), dtype=torch.complex64, device=self.inner.device)
        grad, loss = allreduce_gradient(grad, loss, self.group)
        if grad_out is not None:
            grad_out.copy_(grad)
            return loss, grad_out
        return loss, grad
