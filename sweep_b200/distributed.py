"""Shot-parallel gradients over ``torch.distributed`` -- the multi-GPU shape of
this path.

Shots are independent: each rank runs the forward and adjoint of its own shots
with a replicated model, then one ``all_reduce(SUM)`` per model gradient (and
of the loss) combines them, as the reference's shot-parallel FWI example does
(reference ``examples/multi-gpu/torch/fwi_marmousi_dist.py:338-360``).  There
is no halo exchange: nothing else crosses ranks.  On GPUs the backend is NCCL;
the same code runs on ``gloo`` for CPU tests.
"""
from __future__ import annotations

from typing import Callable, Sequence

import torch
import torch.distributed as dist

__all__ = ["shot_slice", "all_reduce_", "sharded_gradient"]


def shot_slice(n_shots: int, world_size: int, rank: int) -> slice:
    """The contiguous block of shots rank ``rank`` owns: sizes differ by at
    most one, lower ranks take the extra shots."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"bad rank {rank} of world size {world_size}")
    base, extra = divmod(int(n_shots), world_size)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def all_reduce_(tensors: Sequence[torch.Tensor], group=None) -> None:
    """In-place SUM over the ranks of ``group`` (no-op without a process group)."""
    if not (dist.is_available() and dist.is_initialized()):
        return
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def sharded_gradient(compute: Callable[[slice], tuple], n_shots: int, group=None):
    """Loss and model gradients of a survey of ``n_shots`` shots sharded over
    the ranks of ``group``.

    ``compute(shots)`` runs this rank's shots (a ``slice`` of the survey) and
    returns ``(loss, [grad, ...])`` as tensors; a rank with no shots must still
    return zero tensors of the right shapes.  Returns the all-reduced
    ``(loss, grads)``, identical on every rank."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    loss, grads = compute(shot_slice(n_shots, world, rank))
    grads = [g.contiguous() for g in grads]
    # the loss travels with the gradients (NCCL reduces device tensors only),
    # whatever compute() returned it as: a Python float, a CPU or GPU tensor
    dev = grads[0].device if grads else torch.device("cpu")
    loss = torch.as_tensor(loss, dtype=torch.float64).to(dev).reshape(1).clone()
    all_reduce_([loss, *grads], group)
    return loss[0], grads
