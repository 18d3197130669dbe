"""Per-frame pair stacks for training, built by the GPU neighbor operator.

The rule of src/nabladyn/training/_fit.py:190-242: a zero-skin list counts each frame's pairs,
one sized for the densest frame builds every row, and rows are padded with self-pairs
(k mod N, k mod N) to a common width.
"""

import torch
from torch import Tensor

from .. import space
from .._native import OVERFLOW
from ..neighbors import NeighborList


def width(count: int) -> int:
    """``count`` rounded up to a multiple of 1/8 of its leading power of two."""
    step = 1 << max(0, count.bit_length() - 4)
    return -(-count // step) * step


def pair_stack(positions: Tensor, cells: Tensor, cutoff: float) -> Tensor:
    """The pairs within ``cutoff`` of frames [F, N, 3] in cells [F, 3], int32 [F, 2, C].

    Raises ``ValueError`` for a cell length that is not finite and above twice the cutoff, or
    a non-finite coordinate.
    """
    frames, atoms = positions.shape[:2]
    wrapped = space.wrap(positions.detach(), cells.detach()[:, None])[0].contiguous()
    cells = cells.detach().contiguous()
    totals = torch.empty(frames, dtype=torch.int32, device=positions.device)
    densest = 0
    while True:
        counter = NeighborList(cutoff, capacity_multiplier=2.0)
        counter.allocate(wrapped[densest], cells[densest])
        for frame in range(frames):
            counter._rebuild_wrapped(wrapped[frame], cells[frame])
            totals[frame:frame + 1].copy_(counter._buffers.pair_total)
        status = counter._buffers.status[0]
        flags, densest = torch.stack([status, totals.argmax().to(status.dtype)]).tolist()
        if flags & ~OVERFLOW:
            counter._check_status()
        if not flags & OVERFLOW:
            break
    neighbors = NeighborList(cutoff, capacity_multiplier=1.0)
    neighbors.allocate(wrapped[densest], cells[densest])
    capacity = neighbors.pair_capacity
    columns = width(capacity)
    fill = torch.arange(columns, dtype=torch.int32, device=positions.device) % atoms
    stack = fill.expand(frames, 2, columns).contiguous()
    pairs = neighbors.tensors().index
    for frame in range(frames):
        neighbors._rebuild_wrapped(wrapped[frame], cells[frame])
        stack[frame, :, :capacity].copy_(pairs)
    neighbors._check_status()
    return stack


__all__ = ("width", "pair_stack")
