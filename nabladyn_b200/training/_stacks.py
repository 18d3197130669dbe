"""Per-frame pair stacks for training, built by the GPU neighbor operator.

A stack is the reference's training input (src/nabladyn/training/_fit.py:190-242): int32
[F, 2, C] holding each frame's pairs within the cutoff (zero skin) in its first columns and
self-pairs (k mod N, k mod N) after them, C being the densest frame's pair capacity rounded up
by ``width``. Here one zero-skin list counts every frame on the device (its status cleared
between frames, so an overflow of one frame does not stop the count of the next) with a single
host read of all counts at the end; a second list, sized for the densest frame, then builds
each frame and its pairs are copied into the stack on the device.
"""

import torch
from torch import Tensor

from .. import space
from .._native import OVERFLOW
from ..neighbors import NeighborList
from ..neighbors._neighbor_list import status_causes


def width(count: int) -> int:
    """``count`` rounded up to a multiple of 2^(bits - 4), bits being its bit length: at most
    1/8 of padding, and few distinct widths across data sets."""
    shift = max(0, count.bit_length() - 4)
    return ((count + (1 << shift) - 1) >> shift) << shift


def pair_stack(positions: Tensor, cells: Tensor, cutoff: float) -> Tensor:
    """The pairs within ``cutoff`` of frames [F, N, 3] in cells [F, 3], int32 [F, 2, C].

    Raises ``ValueError`` for a cell length that is not finite and above twice the cutoff, or
    a non-finite coordinate.
    """
    frames, atoms = positions.shape[:2]
    device = positions.device
    wrapped = space.wrap(positions.detach(), cells.detach()[:, None])[0].contiguous()
    cells = cells.detach().contiguous()

    # Counting: every frame rebuilt into a list sized for frame 0; totals and error flags
    # gathered on the device.
    counter = NeighborList(cutoff, capacity_multiplier=1.0)
    counter.allocate(wrapped[0], cells[0])
    status = counter._device_tensors()["status"]
    totals = torch.empty(frames, dtype=torch.int32, device=device)
    errors = torch.zeros(1, dtype=torch.int32, device=device)
    for frame in range(frames):
        status.zero_()
        counter._rebuild_wrapped(wrapped[frame], cells[frame])
        totals[frame:frame + 1].copy_(counter._device_tensors()["pair_total"])
        errors.bitwise_or_(status[:1] & ~OVERFLOW)
    flags, densest = torch.cat([errors, totals.argmax().reshape(1).int()]).tolist()
    if flags:
        raise ValueError("; ".join(status_causes(flags, 0, 0, counter.radius)))

    # Building: a list sized for the densest frame, each frame's pairs copied into its row.
    builder = NeighborList(cutoff, capacity_multiplier=1.0)
    builder.allocate(wrapped[densest], cells[densest])
    capacity = builder.pair_capacity
    columns = width(capacity)
    stack = (torch.arange(columns, dtype=torch.int32, device=device) % atoms).expand(
        frames, 2, columns).contiguous()
    pairs = builder.tensors().index
    for frame in range(frames):
        builder._rebuild_wrapped(wrapped[frame], cells[frame])
        stack[frame, :, :capacity].copy_(pairs)
    builder._check_status()
    return stack


__all__ = ("width", "pair_stack")
