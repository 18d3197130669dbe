"""12-6 Lennard-Jones shifted to zero at the cutoff, one sigma and epsilon per type pair.

Mirrors src/nabladyn/potential/_lennard_jones/_potential.py (LennardJones :113-237,
pair_index :143-151) and the constructor src/nabladyn/potential/_api.py:18-57. The energy and
all its first derivatives (forces, virial, parameter gradients) come from one pass of the
CUDA pair kernel (nd_lj_energy_force_virial); ``_LJEnergy`` exposes them to autograd and
torch.func, so ``quantity``'s generic path and plain ``.backward()`` work on the model.
"""

from __future__ import annotations

import math
from collections.abc import Mapping, Sequence
from numbers import Integral, Real

import torch
from torch import Tensor, nn

from .. import _native
from .._native import LJPairsArgs, call, dtype_code, ptr, stream_handle
from ..neighbors import NeighborPairs
from ._base import Potential


def _check_trainable_names(trainable) -> None:
    if isinstance(trainable, str) or not set(trainable) <= {"sigma", "epsilon"}:
        raise ValueError('trainable must name parameters among "sigma" and "epsilon"')


def _check_cutoff(cutoff: Real) -> None:
    if isinstance(cutoff, bool) or not isinstance(cutoff, Real) or not math.isfinite(cutoff) or cutoff <= 0:
        raise ValueError("cutoff must be a finite positive number")


def _check_parameter_vectors(sigma: Tensor, epsilon: Tensor) -> None:
    for name, value in (("sigma", sigma), ("epsilon", epsilon)):
        if (
            not isinstance(value, Tensor)
            or value.ndim != 1
            or value.dtype not in (torch.float32, torch.float64)
        ):
            raise ValueError(f"{name} must be a float32 or float64 vector")
    if (epsilon.shape, epsilon.dtype, epsilon.device) != (sigma.shape, sigma.dtype, sigma.device):
        raise ValueError("sigma and epsilon must share shape, dtype and device")


def _num_types(sigma: Tensor) -> int:
    """T from sigma's T(T+1)/2 rows; ``ValueError`` unless the count is triangular."""
    num_types = math.isqrt(2 * sigma.numel())
    if num_types == 0 or num_types * (num_types + 1) // 2 != sigma.numel():
        raise ValueError("sigma and epsilon need T(T+1)/2 values, one per type pair")
    return num_types


def _check_parameter_values(sigma: Tensor, epsilon: Tensor) -> None:
    values = torch.cat([sigma, epsilon])
    if not bool((values.isfinite() & (values > 0)).all()):
        raise ValueError("sigma and epsilon must be finite and positive")


def _check_atom_types(atom_types: Tensor, num_types: int) -> None:
    if (
        not isinstance(atom_types, Tensor)
        or atom_types.ndim != 1
        or atom_types.dtype != torch.int64
        or atom_types.numel() == 0
    ):
        raise ValueError("atom_types must be a nonempty int64 vector")
    if not bool(((atom_types >= 0) & (atom_types < num_types)).all()):
        raise ValueError(f"atom_types must lie in [0, {num_types})")


def _row_mask(trainable, name: str, count: int, device) -> Tensor | None:
    """A bool mask of the trained rows of ``name``, or None when all or none train."""
    if not isinstance(trainable, Mapping) or name not in trainable:
        return None
    rows = trainable[name]
    if (
        isinstance(rows, (str, bytes))
        or not isinstance(rows, Sequence)
        or not rows
        or any(
            isinstance(row, bool) or not isinstance(row, Integral) or not 0 <= row < count
            for row in rows
        )
    ):
        raise ValueError(f"trainable[{name!r}] must list rows in [0, {count})")
    if len(set(rows)) == count:
        return None
    mask = torch.zeros(count, dtype=torch.bool, device=device)
    mask[[int(row) for row in rows]] = True
    return mask


def pair_index(first: Tensor, second: Tensor, num_types: int) -> Tensor:
    """The parameter row of each unordered type pair: row-major upper triangle.

    For a <= b the row is a (2T - a - 1) / 2 + b (src/nabladyn/potential/_lennard_jones/
    _potential.py:143-151).
    """
    low, high = torch.minimum(first, second), torch.maximum(first, second)
    return low * (2 * num_types - low - 1) // 2 + high


def evaluate_pairs(
    positions: Tensor,
    cell: Tensor,
    index: Tensor,
    kernel_types: Tensor | None,
    num_types: int,
    sigma: Tensor,
    epsilon: Tensor,
    cutoff: float,
    strain: Tensor | None = None,
    parameter_grads: bool = False,
):
    """One pass of the pair kernel over wrapped positions.

    Returns (E float64 [], F [N, 3] in the positions' dtype, W float64 [3, 3], dE/dsigma,
    dE/depsilon float64 or None). No host sync.
    """
    device, dtype = positions.device, positions.dtype
    positions = positions.detach().contiguous()
    cell = cell.detach().contiguous()
    index = index.detach()
    if index.dtype != torch.int32:
        index = index.to(torch.int32)
    index = index.contiguous()
    sigma = sigma.detach().to(dtype).contiguous()
    epsilon = epsilon.detach().to(dtype).contiguous()
    rows = sigma.numel()
    energy = torch.empty(1, dtype=torch.float64, device=device)
    virial = torch.empty((3, 3), dtype=torch.float64, device=device)
    forces = torch.empty_like(positions)
    grads = (
        torch.empty((2, rows), dtype=torch.float64, device=device) if parameter_grads else None
    )
    if strain is not None:
        strain = strain.detach().to(dtype).contiguous()
    args = LJPairsArgs(
        dtype=dtype_code(dtype),
        positions=ptr(positions),
        cell=ptr(cell),
        num_atoms=positions.shape[0],
        pairs=ptr(index),
        capacity=index.shape[1],
        atom_types=ptr(kernel_types) if num_types > 1 else None,
        num_types=num_types,
        sigma=ptr(sigma),
        epsilon=ptr(epsilon),
        cutoff=float(cutoff),
        strain=ptr(strain),
        energy=ptr(energy),
        forces=ptr(forces),
        virial=ptr(virial),
        sigma_grad=grads[0].data_ptr() if grads is not None else None,
        epsilon_grad=grads[1].data_ptr() if grads is not None else None,
    )
    with torch.cuda.device(device):
        call("nd_lj_energy_force_virial", args, stream_handle(device))
    return (
        energy[0],
        forces,
        virial,
        grads[0] if grads is not None else None,
        grads[1] if grads is not None else None,
    )


class _LJEnergy(torch.autograd.Function):
    """E of the pair kernel, with its saved first derivatives as the backward.

    Inputs (positions, strain, sigma, epsilon) may require gradients; the kernel computes all
    of them in the forward pass, so the backward only scales. The parameter gradients are
    computed only when sigma or epsilon requires one.
    """

    @staticmethod
    def forward(positions, strain, sigma, epsilon, cell, index, kernel_types, num_types, cutoff,
                want_parameters):
        energy, forces, virial, dsigma, depsilon = evaluate_pairs(
            positions, cell, index, kernel_types, num_types, sigma, epsilon, cutoff,
            strain=strain, parameter_grads=want_parameters,
        )
        dtype = positions.dtype
        if dsigma is None:
            dsigma = torch.zeros_like(sigma)
            depsilon = torch.zeros_like(epsilon)
        return (
            energy.to(dtype),
            -forces,
            (-virial).to(dtype),
            dsigma.to(sigma.dtype),
            depsilon.to(epsilon.dtype),
        )

    @staticmethod
    def setup_context(ctx, inputs, output):
        _, dpositions, dstrain, dsigma, depsilon = output
        ctx.mark_non_differentiable(dpositions, dstrain, dsigma, depsilon)
        ctx.save_for_backward(dpositions, dstrain, dsigma, depsilon)
        ctx.has_strain = inputs[1] is not None

    @staticmethod
    def backward(ctx, grad_energy, *_):
        dpositions, dstrain, dsigma, depsilon = ctx.saved_tensors
        return (
            grad_energy * dpositions,
            grad_energy * dstrain if ctx.has_strain else None,
            grad_energy * dsigma,
            grad_energy * depsilon,
            None, None, None, None, None, None,
        )


class LennardJones(Potential):
    """12-6 Lennard-Jones shifted to zero at the cutoff; built by ``lennard_jones``."""

    # E, F and W always come from the fused pair kernel (float32 and float64).
    _fused_kernel = True

    def __init__(self, *, atom_types: Tensor, sigma: Tensor, epsilon: Tensor, cutoff: Real,
                 trainable=()):
        super().__init__()
        _check_trainable_names(trainable)
        _check_cutoff(cutoff)
        _check_parameter_vectors(sigma, epsilon)
        num_types = _num_types(sigma)
        _check_parameter_values(sigma, epsilon)
        _check_atom_types(atom_types, num_types)
        self._cutoff = float(cutoff)
        self._num_types = num_types
        self.sigma = nn.Parameter(sigma.detach().clone(), requires_grad="sigma" in trainable)
        self.epsilon = nn.Parameter(
            epsilon.detach().clone(), requires_grad="epsilon" in trainable,
        )
        self.register_buffer("atom_types", atom_types.detach().to(sigma.device, copy=True))
        # The kernels read types as int32.
        self.register_buffer(
            "_kernel_types", self.atom_types.to(torch.int32).contiguous(), persistent=False,
        )
        for name in ("sigma", "epsilon"):
            mask = _row_mask(trainable, name, sigma.numel(), sigma.device)
            self.register_buffer(f"_{name}_rows", mask, persistent=False)

    @property
    def cutoff(self) -> float:
        return self._cutoff

    @property
    def num_atoms(self) -> int:
        return self.atom_types.numel()

    @property
    def num_types(self) -> int:
        return self._num_types

    @property
    def dtype(self) -> torch.dtype:
        return self.sigma.dtype

    @property
    def device(self) -> torch.device:
        return self.sigma.device

    def _trained_masks(self) -> dict[str, Tensor]:
        masks = {"sigma": self._sigma_rows, "epsilon": self._epsilon_rows}
        return {name: mask for name, mask in masks.items() if mask is not None}

    def _energy_wrapped(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs,
                        strain: Tensor | None = None) -> Tensor:
        want = bool(self.sigma.requires_grad or self.epsilon.requires_grad) and torch.is_grad_enabled()
        energy, *_ = _LJEnergy.apply(
            positions, strain, self.sigma, self.epsilon, cell, pairs.index, self._kernel_types,
            self._num_types, self._cutoff, want,
        )
        return energy

    def _energy_force_virial(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs):
        """(E, F, W) of wrapped positions in one kernel pass, in the model's dtype."""
        energy, forces, virial, _, _ = evaluate_pairs(
            positions, cell, pairs.index, self._kernel_types, self._num_types, self.sigma,
            self.epsilon, self._cutoff,
        )
        dtype = positions.dtype
        return energy.to(dtype), forces, virial.to(dtype)


def lennard_jones(*, atom_types: Tensor, sigma: Tensor, epsilon: Tensor, cutoff: Real,
                  trainable=()) -> Potential:
    r"""Build a 12-6 Lennard-Jones model shifted to zero at the cutoff.

    E sums u(r) = 4 eps [(sigma/r)^12 - (sigma/r)^6] - u_c over pairs closer than the cutoff,
    u_c the unshifted value at r_c, each pair with its own row of sigma and epsilon.
    ``atom_types`` [N] int64 in [0, T); ``sigma`` (nm) and ``epsilon`` (kJ/mol) hold T(T+1)/2
    rows in the order (0, 0), (0, 1), ..., (1, 1), ...; ``trainable`` names what a fit trains
    ("sigma", "epsilon", or a mapping to rows). Raises ``ValueError`` as the reference does.
    """
    return LennardJones(
        atom_types=atom_types, sigma=sigma, epsilon=epsilon, cutoff=cutoff, trainable=trainable,
    )


__all__ = ("LennardJones", "lennard_jones", "pair_index")
