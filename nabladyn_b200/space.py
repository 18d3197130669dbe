"""Orthorhombic periodic geometry on [..., 3] tensors; ``cell`` [3] holds the edge lengths in nm.

The same functions and arithmetic as src/nabladyn/space.py:11-64. The MD engine does its own
wrapping inside its kernels; these serve the host-side API (allocation, checks, export).
"""

import torch
from torch import Tensor


def _displacement_wrapped(left: Tensor, right: Tensor, cell: Tensor) -> Tensor:
    """The minimum-image vector ``left - right`` for coordinates already in [0, L).

    The coordinate on the far side moves by L first, which is exact, so the vector is rounded
    once (src/nabladyn/space.py:11-19).
    """
    raw = left - right
    half = 0.5 * cell
    left_shift = torch.where(raw > half, cell, 0.0)
    right_shift = torch.where(raw < -half, cell, 0.0)
    return (left - left_shift) - (right - right_shift)


def wrap(positions: Tensor, cell: Tensor) -> tuple[Tensor, Tensor]:
    """Wrap positions [..., 3] into [0, L); return (wrapped, crossings int64).

    The floor of the quotient, then two fix-ups in this order keep every result in [0, L)
    (src/nabladyn/space.py:22-38).
    """
    crossings = torch.floor(positions / cell)
    wrapped = positions - crossings * cell
    below = wrapped < 0
    wrapped = torch.where(below, wrapped + cell, wrapped)
    crossings = torch.where(below, crossings - 1, crossings)
    above = wrapped >= cell
    wrapped = torch.where(above, wrapped - cell, wrapped)
    crossings = torch.where(above, crossings + 1, crossings)
    return wrapped, crossings.to(torch.int64)


def shift(positions: Tensor, delta: Tensor, cell: Tensor) -> tuple[Tensor, Tensor]:
    """``positions + delta`` wrapped into the cell, with ``wrap``'s crossings."""
    return wrap(positions + delta, cell)


def displacement(left: Tensor, right: Tensor, cell: Tensor) -> Tensor:
    """The minimum-image vector ``left - right`` [..., 3], for positions anywhere."""
    return _displacement_wrapped(wrap(left, cell)[0], wrap(right, cell)[0], cell)


def strained(vectors: Tensor, strain: Tensor | None) -> Tensor:
    """Deform ``vectors`` [..., 3] by (I + strain); None returns ``vectors`` itself."""
    if strain is None:
        return vectors
    return (
        vectors
        + vectors[..., 0:1] * strain[:, 0]
        + vectors[..., 1:2] * strain[:, 1]
        + vectors[..., 2:3] * strain[:, 2]
    )


__all__ = ("wrap", "shift", "displacement", "strained")
