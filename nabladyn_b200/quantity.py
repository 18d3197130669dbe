"""Energy, forces and virial from one scalar energy.

The API of src/nabladyn/quantity.py:88-184: each function binds an energy, any callable
``energy(positions, cell, pairs, strain=None)`` such as a Potential, and returns a function of
``(positions, cell, pairs)``. E is in kJ/mol, F = -dE/dpositions [N, 3] in kJ/mol/nm and
W = -dE/dstrain at zero strain [3, 3] in kJ/mol.

For the Lennard-Jones model and float32 SchNet models of 64 features (the model itself, or its
``_energy_wrapped``) every binding runs the fused CUDA kernels once: E, F and W come out of the
same pass, with E and W reduced in float64. Any other energy is differentiated by
``torch.func`` exactly as the reference does.
"""

from collections.abc import Callable

import torch
from torch import Tensor

from .neighbors import NeighborPairs
from .potential._base import Potential, _check_pairs, _check_tensor
from . import space


def _fused(energy_fn):
    """(model, wraps) when ``energy_fn`` is a model with fused kernels (Lennard-Jones, or a
    SchNet the kernels cover) or its wrapped energy."""
    if isinstance(energy_fn, Potential) and getattr(energy_fn, "_fused_kernel", False):
        return energy_fn, True
    owner = getattr(energy_fn, "__self__", None)
    if (
        isinstance(owner, Potential)
        and getattr(owner, "_fused_kernel", False)
        and getattr(energy_fn, "__func__", None) is type(owner)._energy_wrapped
    ):
        return owner, False
    return None, False


def _fused_evaluate(model: Potential, wraps: bool):
    def evaluate(positions: Tensor, cell: Tensor, pairs: NeighborPairs):
        if wraps:
            # The model's own call checks its inputs and wraps the positions.
            _check_tensor("positions", positions, (model.num_atoms, 3), model.dtype, model.device)
            _check_tensor("cell", cell, (3,), model.dtype, model.device)
            _check_pairs(pairs, model.num_atoms, model.cutoff, model.device)
            positions = space.wrap(positions, cell)[0]
        return model._energy_force_virial(positions, cell, pairs)

    return evaluate


def _with_strain(energy_fn: Callable[..., Tensor]):
    def strained_energy(positions, strain, cell, pairs):
        return energy_fn(positions, cell, pairs, strain=strain)

    return strained_energy


def energy_force_virial(energy_fn: Callable[..., Tensor]):
    """Bind (E, F, W): the energy and virial [3, 3] in kJ/mol, forces [N, 3] in kJ/mol/nm."""
    model, wraps = _fused(energy_fn)
    if model is not None:
        return _fused_evaluate(model, wraps)
    gradient_and_value = torch.func.grad_and_value(_with_strain(energy_fn), argnums=(0, 1))

    def evaluate(positions, cell, pairs):
        (position_grad, strain_grad), energy = gradient_and_value(
            positions, positions.new_zeros((3, 3)), cell, pairs,
        )
        return energy, -position_grad, -strain_grad

    return evaluate


def energy_and_force(energy_fn: Callable[..., Tensor]):
    """Bind (E, F)."""
    model, wraps = _fused(energy_fn)
    if model is not None:
        fused = _fused_evaluate(model, wraps)
        return lambda positions, cell, pairs: fused(positions, cell, pairs)[:2]
    gradient_and_value = torch.func.grad_and_value(energy_fn, argnums=0)

    def evaluate(positions, cell, pairs):
        gradient, energy = gradient_and_value(positions, cell, pairs)
        return energy, -gradient

    return evaluate


def force(energy_fn: Callable[..., Tensor]):
    """Bind F."""
    model, wraps = _fused(energy_fn)
    if model is not None:
        fused = _fused_evaluate(model, wraps)
        return lambda positions, cell, pairs: fused(positions, cell, pairs)[1]
    gradient = torch.func.grad(energy_fn, argnums=0)
    return lambda positions, cell, pairs: -gradient(positions, cell, pairs)


def force_virial(energy_fn: Callable[..., Tensor]):
    """Bind (F, W)."""
    model, wraps = _fused(energy_fn)
    if model is not None:
        fused = _fused_evaluate(model, wraps)
        return lambda positions, cell, pairs: fused(positions, cell, pairs)[1:]
    gradient = torch.func.grad(_with_strain(energy_fn), argnums=(0, 1))

    def evaluate(positions, cell, pairs):
        position_grad, strain_grad = gradient(positions, positions.new_zeros((3, 3)), cell, pairs)
        return -position_grad, -strain_grad

    return evaluate


def virial(energy_fn: Callable[..., Tensor]):
    """Bind W."""
    model, wraps = _fused(energy_fn)
    if model is not None:
        fused = _fused_evaluate(model, wraps)
        return lambda positions, cell, pairs: fused(positions, cell, pairs)[2]
    gradient = torch.func.grad(_with_strain(energy_fn), argnums=1)
    return lambda positions, cell, pairs: -gradient(
        positions, positions.new_zeros((3, 3)), cell, pairs,
    )


def energy_virial(energy_fn: Callable[..., Tensor]):
    """Bind (E, W)."""
    model, wraps = _fused(energy_fn)
    if model is not None:
        fused = _fused_evaluate(model, wraps)

        def evaluate_fused(positions, cell, pairs):
            energy, _, w = fused(positions, cell, pairs)
            return energy, w

        return evaluate_fused
    gradient_and_value = torch.func.grad_and_value(_with_strain(energy_fn), argnums=1)

    def evaluate(positions, cell, pairs):
        strain_grad, energy = gradient_and_value(
            positions, positions.new_zeros((3, 3)), cell, pairs,
        )
        return energy, -strain_grad

    return evaluate


__all__ = (
    "force",
    "energy_and_force",
    "force_virial",
    "virial",
    "energy_virial",
    "energy_force_virial",
)
