"""SchNet: continuous-filter convolutions over the pairs of a neighbor list.

Mirrors src/nabladyn/potential/_schnet/_potential.py (SchNet :123-208, _Interaction :55-87,
_pair_geometry :90-120) and the constructor src/nabladyn/potential/_api.py:133-184: the same
parameters under the same state-dict names, drawn from the same seed in the same order, and
``_energy_wrapped`` as the model's definition (the path torch.func differentiates, and the one
float64 models take).

Float32 models with 64 features and at most 64 Gaussians have a fused path: E, F and W from
the hand-written CUDA kernels of ``csrc/schnet.cu`` (``nd_schnet_energy_force_virial``),
which run the per-pair filter network and the atom-wise layers on BF16 tcgen05 tensor cores
with FP32 accumulation, and the reverse pass for forces and virial by hand. ``quantity`` and
the MD engine pick it.
"""

from __future__ import annotations

import math
from numbers import Integral, Real

import torch
from torch import Tensor, nn

from .. import space
from ..neighbors import NeighborPairs
from ._base import Potential
from ._lennard_jones import _check_atom_types, _check_cutoff


def _check_sizes(num_types: int, features: int, interactions: int, gaussians: int) -> None:
    sizes = (("num_types", num_types, 1), ("features", features, 2),
             ("interactions", interactions, 1), ("gaussians", gaussians, 2))
    for name, value, least in sizes:
        if isinstance(value, bool) or not isinstance(value, Integral) or value < least:
            raise ValueError(f"{name} must be an integer of at least {least}")
    if features % 2:
        raise ValueError("features must be even: the readout halves it")


def _check_flag_and_seed(trainable: bool, seed: int) -> None:
    if not isinstance(trainable, bool):
        raise ValueError("trainable must be True or False")
    if isinstance(seed, bool) or not isinstance(seed, Integral):
        raise ValueError("seed must be an integer")


def shifted_softplus(x: Tensor) -> Tensor:
    """ln(1 + e^x) - ln 2, zero at x = 0."""
    return nn.functional.softplus(x) - math.log(2.0)


def _dense(inputs: int, outputs: int, bias: bool = True) -> nn.Linear:
    """An uninitialised float64 ``nn.Linear`` (weight, then bias); the model's seed sets it."""
    layer = nn.Linear.__new__(nn.Linear)
    nn.Module.__init__(layer)
    layer.in_features, layer.out_features = inputs, outputs
    layer.weight = nn.Parameter(torch.empty((outputs, inputs), dtype=torch.float64))
    if bias:
        layer.bias = nn.Parameter(torch.empty(outputs, dtype=torch.float64))
    else:
        layer.register_parameter("bias", None)
    return layer


class _Interaction(nn.Module):
    """One block: x + ssp(m D1^T + d1) D2^T + d2 with m_i = sum_j f_ij * (x_j A^T)."""

    def __init__(self, features: int, gaussians: int):
        super().__init__()
        self.atoms = _dense(features, features, bias=False)
        self.filter1 = _dense(gaussians, features)
        self.filter2 = _dense(features, features)
        self.update1 = _dense(features, features)
        self.update2 = _dense(features, features)

    def forward(self, x: Tensor, basis: Tensor, envelope: Tensor, first: Tensor,
                second: Tensor) -> Tensor:
        values = self.atoms(x)
        filters = self.filter2(shifted_softplus(self.filter1(basis))) * envelope[:, None]
        width = x.shape[1]
        # Each listed pair sends to both its atoms; out of place, so vmap over frames works.
        messages = (
            x.new_zeros(x.shape)
            .scatter_add(0, first[:, None].expand(-1, width), filters * values[second])
            .scatter_add(0, second[:, None].expand(-1, width), filters * values[first])
        )
        return x + self.update2(shifted_softplus(self.update1(messages)))


def pair_geometry(positions: Tensor, cell: Tensor, pairs: NeighborPairs, strain: Tensor | None,
                  cutoff: float, centres: Tensor):
    """(first, second, d, r, envelope, Gaussians) of the list's columns; masked columns
    (padding self-pairs, pairs beyond the cutoff) get r = 1 and a zero envelope."""
    first, second = pairs.index[0].long(), pairs.index[1].long()
    vectors = space.strained(space._displacement_wrapped(positions[first], positions[second],
                                                         cell), strain)
    squared = vectors.square().sum(dim=-1)
    valid = (first != second) & (squared < cutoff**2)
    distance = torch.where(valid, squared, 1.0).sqrt()
    envelope = torch.where(valid, 0.5 * (torch.cos(distance * (math.pi / cutoff)) + 1.0), 0.0)
    width = cutoff / (centres.numel() - 1)
    basis = torch.exp(-0.5 * ((distance[:, None] - centres) / width).square())
    return first, second, vectors, distance, envelope, basis


class SchNet(Potential):
    """SchNet with fixed Gaussians, a cosine envelope and the shifted softplus."""

    def __init__(self, *, atom_types: Tensor, num_types: int, cutoff: Real, features: int,
                 interactions: int, gaussians: int, trainable: bool, seed: int,
                 dtype: torch.dtype):
        super().__init__()
        _check_sizes(num_types, features, interactions, gaussians)
        _check_cutoff(cutoff)
        _check_flag_and_seed(trainable, seed)
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be torch.float32 or torch.float64")
        _check_atom_types(atom_types, num_types)
        self._cutoff = float(cutoff)
        self._num_types = int(num_types)
        self.embedding = nn.Parameter(torch.empty(num_types, features, dtype=torch.float64))
        self.blocks = nn.ModuleList(_Interaction(features, gaussians) for _ in range(interactions))
        self.readout1 = _dense(features, features // 2)
        self.readout2 = _dense(features // 2, 1)
        # One float64 stream from the seed, parameters in registration order: the table
        # standard normal, matrices Xavier-uniform, biases zero; so a seed gives the same
        # network in both dtypes and in the reference.
        generator = torch.Generator().manual_seed(int(seed))
        with torch.no_grad():
            for name, parameter in self.named_parameters():
                if name == "embedding":
                    values = torch.randn(parameter.shape, generator=generator, dtype=torch.float64)
                elif name.endswith("weight"):
                    bound = math.sqrt(6.0 / sum(parameter.shape))
                    uniform = torch.rand(parameter.shape, generator=generator, dtype=torch.float64)
                    values = (2.0 * uniform - 1.0) * bound
                else:
                    values = torch.zeros_like(parameter)
                parameter.copy_(values)
        self.to(device=atom_types.device, dtype=dtype)
        self.requires_grad_(trainable)
        self.register_buffer("atom_types", atom_types.detach().clone(), persistent=False)
        centres = torch.linspace(0.0, self._cutoff, gaussians, dtype=dtype, device=self.device)
        self.register_buffer("_centres", centres, persistent=False)
        self._packed = None

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
    def features(self) -> int:
        return self.embedding.shape[1]

    @property
    def gaussians(self) -> int:
        return self._centres.numel()

    @property
    def interactions(self) -> int:
        return len(self.blocks)

    @property
    def dtype(self) -> torch.dtype:
        return self.embedding.dtype

    @property
    def device(self) -> torch.device:
        return self.embedding.device

    def _energy_wrapped(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs,
                        strain: Tensor | None = None) -> Tensor:
        first, second, _, _, envelope, basis = pair_geometry(
            positions, cell, pairs, strain, self._cutoff, self._centres)
        x = self.embedding[self.atom_types]
        for block in self.blocks:
            x = block(x, basis, envelope, first, second)
        return self.readout2(shifted_softplus(self.readout1(x))).sum()

    @property
    def _fused_kernel(self) -> bool:
        """Whether E/F/W come from the CUDA kernels: float32 on a GPU, 64 features, at most
        64 Gaussians. Other sizes and float64 run ``_energy_wrapped`` under torch.func."""
        return (self.dtype == torch.float32 and self.device.type == "cuda"
                and self.features == 64 and self.gaussians <= 64)

    def _energy_force_virial(self, positions: Tensor, cell: Tensor, pairs: NeighborPairs):
        from ._schnet_kernels import energy_force_virial

        return energy_force_virial(self, positions, cell, pairs)


def schnet(*, atom_types: Tensor, num_types: int, cutoff: Real, features: int = 64,
           interactions: int = 3, gaussians: int = 50, trainable: bool = False, seed: int = 0,
           dtype: torch.dtype = torch.float32) -> Potential:
    r"""A SchNet network (Schütt et al., J. Chem. Phys. 148, 241722, 2018).

    Each atom starts from its type's row of a table [T, F]. Each of the ``interactions``
    blocks adds ssp(m_i D1 + d1) D2 + d2, where m_i sums f_ij * (x_j A) over the pairs within
    the cutoff, each pair sending to both atoms, with the filter
    f_ij = (ssp(g(r_ij) B1 + b1) B2 + b2) C(r_ij): K = ``gaussians`` fixed Gaussians
    g_k(r) = exp(-(r - kD)^2 / (2 D^2)), D = r_c / (K - 1), and C(r) = (1 + cos(pi r / r_c)) / 2.
    E = sum_i ssp(x_i R1 + e1) R2 + e2 in kJ/mol, ssp(x) = ln(1 + e^x) - ln 2.

    ``atom_types`` [N] int64 in [0, ``num_types``) fixes the atoms and the device; ``cutoff``
    in nm; ``features`` F even (the readout's hidden layer is F / 2). Weights are drawn in
    float64 from ``seed`` and cast to ``dtype``. Raises ``ValueError`` for sizes out of
    range, an odd F, a bad cutoff or dtype, or atom types out of range.
    """
    return SchNet(atom_types=atom_types, num_types=num_types, cutoff=cutoff, features=features,
                  interactions=interactions, gaussians=gaussians, trainable=trainable,
                  seed=seed, dtype=dtype)


__all__ = ("SchNet", "schnet", "shifted_softplus", "pair_geometry")
