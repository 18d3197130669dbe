"""The sum of models: one energy, the sum of the parts' energies.

Mirrors src/nabladyn/potential/_sum/_potential.py (Sum :45-118) and the constructor
src/nabladyn/potential/_api.py:273-293: parts of one topology, dtype and device; the cutoff is
the largest part's; each part reads the shortest given list that reaches its own cutoff (the
neighbor list's inner lists), so a list per cutoff changes the cost, never the energy. When
every part has fused kernels (Lennard-Jones, float32 SchNet), E, F and W are the sums of the
parts' fused results, each on its own list.
"""

from __future__ import annotations

import torch
from torch import Tensor, nn

from ..neighbors import NeighborPairs
from ._base import Potential


def _check_matching(models) -> None:
    first = models[0]
    shared = (first.num_atoms, first.dtype, first.device)
    for model in models[1:]:
        if (model.num_atoms, model.dtype, model.device) != shared:
            raise ValueError(
                f"the models of a sum must match: {first.num_atoms} atoms in {first.dtype} on "
                f"{first.device}, against {model.num_atoms} in {model.dtype} on "
                f"{model.device}; convert a sum as a whole, not one of its models")


def own_pairs(pairs: NeighborPairs, cutoff: float) -> NeighborPairs:
    """The first list, ascending through ``pairs.inner`` then ``pairs``, that reaches
    ``cutoff``, with the shorter lists as its inner lists."""
    lists = (*pairs.inner, pairs)
    own = [listed for listed in lists if listed.cutoff >= cutoff][0]
    shorter = tuple(listed for listed in lists if listed.cutoff < own.cutoff)
    return NeighborPairs(own.index, own.num_atoms, own.cutoff, shorter)


class Sum(Potential):
    """Models whose energies add, E = sum_k E_k; built by ``potential.sum``."""

    def __init__(self, *models: Potential):
        super().__init__()
        if not all(isinstance(model, Potential) for model in models):
            raise TypeError("every model of a sum must be a Potential")
        if len(models) < 2:
            raise ValueError(f"a sum needs at least two models, not {len(models)}")
        _check_matching(models)
        self._cutoff = max(model.cutoff for model in models)
        self.parts = nn.ModuleList(models)

    @property
    def cutoff(self) -> float:
        return self._cutoff

    @property
    def num_atoms(self) -> int:
        return self.parts[0].num_atoms

    @property
    def dtype(self) -> torch.dtype:
        _check_matching(self.parts)
        return self.parts[0].dtype

    @property
    def device(self) -> torch.device:
        _check_matching(self.parts)
        return self.parts[0].device

    @property
    def _list_cutoffs(self) -> tuple[float, ...]:
        return tuple(sorted({value for part in self.parts for value in part._list_cutoffs}))

    def _trained_masks(self) -> dict[str, Tensor]:
        return {f"parts.{index}.{name}": mask for index, part in enumerate(self.parts)
                for name, mask in part._trained_masks().items()}

    def _energy_wrapped(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs,
                        strain: Tensor | None = None) -> Tensor:
        energies = [part._energy_wrapped(positions, cell, own_pairs(pairs, part.cutoff), strain)
                    for part in self.parts]
        return torch.stack(energies).sum()

    @property
    def _fused_kernel(self) -> bool:
        return all(getattr(part, "_fused_kernel", False) for part in self.parts)

    def _energy_force_virial(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs):
        total = None
        for part in self.parts:
            e, f, w = part._energy_force_virial(positions, cell, own_pairs(pairs, part.cutoff))
            total = (e, f, w) if total is None else (total[0] + e, total[1] + f, total[2] + w)
        return total


def sum(*models: Potential) -> Potential:  # noqa: A001 - the reference's name
    """A model whose energy is the sum of the models' energies (two or more, of the same
    atoms, dtype and device); its cutoff is the largest. It holds the models themselves: its
    parameters are theirs, named ``parts.<k>.<name>``. Raises ``TypeError`` for a model that
    is not a Potential and ``ValueError`` for fewer than two models or mismatched ones."""
    return Sum(*models)


__all__ = ("Sum", "sum", "own_pairs")
