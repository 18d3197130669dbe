"""The Potential contract: a model whose one scalar energy defines forces and virial.

Mirrors src/nabladyn/potential/_base.py:46-124: ``model(positions, cell, pairs, strain=None)``
checks its inputs, wraps the positions and returns the energy.
"""

from abc import ABC, abstractmethod

import torch
from torch import Tensor, nn

from .. import space
from ..neighbors import NeighborPairs


def _check_tensor(name: str, value, shape, dtype, device) -> None:
    if not isinstance(value, Tensor) or value.shape != shape:
        raise ValueError(f"{name} must be a tensor of shape {list(shape)}")
    if value.dtype != dtype or value.device != device:
        raise ValueError(f"{name} must be {dtype} on {device} to match the model")


def _check_pairs(pairs: NeighborPairs, num_atoms: int, cutoff: float, device) -> None:
    for listed in (pairs, *pairs.inner):
        index = listed.index
        if index.ndim != 2 or index.shape[0] != 2 or index.device != device:
            raise ValueError(f"pairs.index must be a [2, C] tensor on {device}")
        if listed.num_atoms != num_atoms:
            raise ValueError(
                f"the pairs are for {listed.num_atoms} atoms, the model for {num_atoms}",
            )
    if pairs.cutoff < cutoff:
        raise ValueError(
            f"the neighbor list's cutoff {pairs.cutoff} nm is below the model's {cutoff} nm",
        )


class Potential(nn.Module, ABC):
    """A model of a fixed set of atoms with one scalar energy in kJ/mol."""

    @property
    @abstractmethod
    def cutoff(self) -> float:
        """The interaction cutoff in nm."""

    @property
    @abstractmethod
    def num_atoms(self) -> int:
        """The number of atoms in the model's topology."""

    @property
    @abstractmethod
    def dtype(self) -> torch.dtype:
        """The floating dtype the model computes in."""

    @property
    @abstractmethod
    def device(self) -> torch.device:
        """The device the model computes on."""

    @property
    def _list_cutoffs(self) -> tuple[float, ...]:
        return (self.cutoff,)

    def forward(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs,
                strain: Tensor | None = None) -> Tensor:
        """The energy in kJ/mol of positions [N, 3] in nm, which may lie outside the cell.

        Raises ``ValueError`` for inputs of another shape, dtype or device, or for pairs of
        another system or a shorter cutoff. No host sync.
        """
        _check_tensor("positions", positions, (self.num_atoms, 3), self.dtype, self.device)
        _check_tensor("cell", cell, (3,), self.dtype, self.device)
        if strain is not None:
            _check_tensor("strain", strain, (3, 3), self.dtype, self.device)
        _check_pairs(pairs, self.num_atoms, self.cutoff, self.device)
        wrapped, _ = space.wrap(positions, cell)
        return self._energy_wrapped(wrapped, cell, pairs, strain)

    @abstractmethod
    def _energy_wrapped(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs,
                        strain: Tensor | None = None) -> Tensor:
        """``forward``'s energy for positions already in [0, L), without checks."""

    def _trained_masks(self) -> dict[str, Tensor]:
        return {}


__all__ = ("Potential",)
