"""Data-parallel loss gradients: the frames of a batch split over the ranks of a process group.

The reference differentiates a batch chunk by chunk on one device
(src/nabladyn/training/_fit.py:33-70, ``_batch_gradient``). The batch loss is a mean over its
frames' elements, every frame holding the same elements, so it is the frame-weighted mean of
the chunks' losses: rank r of W takes a contiguous share of the batch's frames, computes its
share's loss and gradient, scales both by (its frames / the batch's frames), and one
all-reduce (a sum) of all of them, packed into one float64 vector, gives every rank the batch's
loss and gradient. One collective per update: 6 scalars for a two-type Lennard-Jones model,
about 50k values for the SchNet of the bead workload.
"""

from __future__ import annotations

import torch
import torch.distributed as dist
from torch import Tensor


def share(frames: Tensor, group=None) -> Tensor:
    """This rank's frames of a batch: a contiguous, balanced split (maybe empty)."""
    world = dist.get_world_size(group)
    return torch.tensor_split(frames, world)[dist.get_rank(group)]


def reduce(value: Tensor, gradient: dict[str, Tensor], weight: float,
           group=None) -> tuple[Tensor, dict[str, Tensor]]:
    """The batch's loss and gradient from every rank's share, scaled by ``weight``: one
    all-reduce of a float64 vector on the gradient's device (NCCL between GPUs, gloo on the
    host). Every rank gets the same result."""
    names = list(gradient)
    device = value.device
    flat = torch.cat([value.detach().reshape(1).to(torch.float64)]
                     + [gradient[name].detach().reshape(-1).to(torch.float64) for name in names])
    flat = flat * weight
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out, offset = {}, 1
    for name in names:
        size = gradient[name].numel()
        out[name] = flat[offset:offset + size].reshape(gradient[name].shape).to(
            gradient[name].dtype)
        offset += size
    return flat[0].to(device), out


__all__ = ("share", "reduce")
