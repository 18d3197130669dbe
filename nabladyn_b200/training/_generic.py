"""Predictions and parameter gradients of any Potential by the reference's algorithm.

A float32 SchNet on a GPU takes its loss gradient from the fused kernels and their written-out
second-order pass (``_schnet_gradient``). For other models (and float64 SchNet) the channels of
a batch of frames and their gradient in the trained parameters come from the reference's own
algorithm
(src/nabladyn/training/_loss.py:49-102, _fit.py:245-271): the model's definition under
``torch.func.functional_call``, E/F/W by ``torch.func`` (so a force or virial loss
differentiates twice), vmapped over frames. ``loss_and_gradient`` runs the frames in chunks,
so the double backward of a large model stays within device memory, and sums the chunks'
gradients (the loss is a sum over frames).
"""

from __future__ import annotations

from collections.abc import Mapping

import torch
from torch import Tensor

from .. import quantity
from ..neighbors import NeighborPairs
from . import _schnet_gradient
from ._loss import loss as batch_loss

_QUANTITIES = {
    ("forces",): quantity.force,
    ("virial",): quantity.virial,
    ("energy", "forces"): quantity.energy_and_force,
    ("energy", "virial"): quantity.energy_virial,
    ("forces", "virial"): quantity.force_virial,
    ("energy", "forces", "virial"): quantity.energy_force_virial,
}


def predict(model, parameters: Mapping[str, Tensor], positions: Tensor, cells: Tensor,
            stacks: tuple[Tensor, ...], channels: tuple[str, ...]) -> dict[str, Tensor]:
    """The channels of B frames by name, differentiable in ``parameters`` (any Potential).

    positions [B, N, 3], cells [B, 3], one [B, 2, C] pair stack (int64 columns are used as
    given; int32 ones are widened, since scatter_add takes int64 indices).
    """
    def energy(positions, cell, pairs, strain=None):
        return torch.func.functional_call(model, dict(parameters), (positions, cell, pairs),
                                          {"strain": strain})

    evaluate = energy if tuple(channels) == ("energy",) else _QUANTITIES[tuple(channels)](energy)
    cutoff, atoms = model.cutoff, model.num_atoms

    def one(x, cell, index):
        values = evaluate(x, cell, NeighborPairs(index, atoms, cutoff))
        return values if isinstance(values, tuple) else (values,)

    stack = stacks[-1].long()
    return dict(zip(channels, torch.func.vmap(one)(positions, cells, stack)))


def loss_and_gradient(model, parameters: Mapping[str, Tensor], positions: Tensor, cells: Tensor,
                      stacks: tuple[Tensor, ...], labels: Mapping[str, Tensor],
                      weights: Mapping[str, float], scales: Mapping[str, float],
                      chunk: int = 4) -> tuple[Tensor, dict[str, Tensor]]:
    """The batch loss (frames weighted 1/B) and its gradient in ``parameters``, ``chunk``
    frames at a time (a fused SchNet runs frame by frame on its kernels instead)."""
    if _schnet_gradient.supported(model):
        return _schnet_gradient.loss_and_gradient(model, parameters, positions, cells, stacks,
                                                  labels, weights, scales)
    return torch_func_loss_and_gradient(model, parameters, positions, cells, stacks, labels,
                                        weights, scales, chunk)


def torch_func_loss_and_gradient(model, parameters: Mapping[str, Tensor], positions: Tensor,
                                 cells: Tensor, stacks: tuple[Tensor, ...],
                                 labels: Mapping[str, Tensor], weights: Mapping[str, float],
                                 scales: Mapping[str, float],
                                 chunk: int = 4) -> tuple[Tensor, dict[str, Tensor]]:
    """``loss_and_gradient`` by the reference's torch.func algorithm, for any model."""
    frames = positions.shape[0]
    channels = tuple(name for name in ("energy", "forces", "virial") if name in labels)
    trained = {name: value.detach() for name, value in parameters.items()}
    total = torch.zeros((), dtype=torch.float64, device=positions.device)
    gradient = {name: torch.zeros_like(value) for name, value in trained.items()}
    for begin in range(0, frames, chunk):
        end = min(frames, begin + chunk)
        coefficients = torch.full((end - begin,), 1.0 / frames, dtype=positions.dtype,
                                  device=positions.device)

        def chunk_loss(values):
            predicted = predict(model, values, positions[begin:end], cells[begin:end],
                                tuple(s[begin:end] for s in stacks), channels)
            part = {name: labels[name][begin:end] for name in channels}
            return batch_loss(predicted, part, weights, scales, coefficients)[0]

        grads, value = torch.func.grad_and_value(chunk_loss)(trained)
        total = total + value.double()
        for name in gradient:
            gradient[name] = gradient[name] + grads[name]
    return total, gradient


__all__ = ("predict", "loss_and_gradient", "torch_func_loss_and_gradient")
