"""Host side of the fused SchNet kernels (nd_schnet_energy_force_virial).

Packs a model's parameters into the kernels' parameter block: per block ten 64 x 64 BF16
operand images in the tensor cores' core-matrix order (filter1, filter2, filter2^T,
filter1^T, atoms, atoms^T, update1, update1^T, update2, update2^T; filter1 zero-padded from K
to 64 Gaussians), then the float32 biases (filter1, filter2, update1, update2 per block), the
readout (R1 [32, 64], e1 [32], R2 [32], e2 padded to 32) and the tables (embedding [T, 64] and
embedding A0^T [T, 64]). The block is rebuilt only when a parameter changed.
"""

from __future__ import annotations

import ctypes

import torch
from torch import Tensor

from .._native import SchNetArgs, call, lib, ptr, stream_handle
from ..neighbors import NeighborPairs

FEATURES = 64


def _image(weight: Tensor) -> Tensor:
    """A [64, 64] matrix (row = output feature, column = reduction index) as a BF16 operand
    image: element (row, k) at (row // 8) * 512 + (k // 8) * 64 + (row % 8) * 8 + k % 8."""
    return weight.to(torch.bfloat16).reshape(8, 8, 8, 8).permute(0, 2, 1, 3).reshape(-1)


def _padded(weight: Tensor, rows: int, cols: int) -> Tensor:
    out = weight.new_zeros((rows, cols))
    out[: weight.shape[0], : weight.shape[1]] = weight
    return out


def weight_bytes(interactions: int, num_types: int) -> int:
    return int(lib().nd_schnet_weight_bytes(interactions, num_types))


def workspace_bytes(num_atoms: int, num_columns: int, interactions: int) -> int:
    return int(lib().nd_schnet_workspace_bytes(num_atoms, num_columns, interactions))


@torch.no_grad()
def pack(model, values=None) -> Tensor:
    """The model's parameter block, uint8 on the model's device; ``values`` (name -> tensor)
    stand in for the model's own parameters of those names."""
    given = dict(model.named_parameters())
    if values is not None:
        given.update(values)

    def get(name: str) -> Tensor:
        return given[name].detach().float()

    images, vectors = [], []
    for b in range(len(model.blocks)):
        b1 = get(f"blocks.{b}.filter1.weight")
        b2 = get(f"blocks.{b}.filter2.weight")
        a = get(f"blocks.{b}.atoms.weight")
        d1 = get(f"blocks.{b}.update1.weight")
        d2 = get(f"blocks.{b}.update2.weight")
        for matrix in (_padded(b1, 64, 64), b2, b2.T, _padded(b1.T, 64, 64), a, a.T, d1, d1.T,
                       d2, d2.T):
            images.append(_image(matrix.contiguous()))
        vectors += [get(f"blocks.{b}.{name}.bias")
                    for name in ("filter1", "filter2", "update1", "update2")]
    e2 = torch.zeros(32, dtype=torch.float32, device=model.device)
    e2[0] = get("readout2.bias")[0]
    floats = torch.cat([
        *vectors,
        get("readout1.weight").reshape(-1),
        get("readout1.bias"),
        get("readout2.weight").reshape(-1),
        e2,
        get("embedding").reshape(-1),
        (get("embedding") @ get("blocks.0.atoms.weight").T).reshape(-1),
    ])
    blob = torch.cat([torch.cat(images).view(torch.uint8), floats.view(torch.uint8)])
    expected = weight_bytes(len(model.blocks), model.num_types)
    if blob.numel() != expected:
        raise RuntimeError(f"packed {blob.numel()} bytes, the kernels expect {expected}")
    return blob


def packed(model) -> Tensor:
    key = tuple((p.data_ptr(), p._version) for p in model.parameters())
    cache = getattr(model, "_packed", None)
    if cache is None or cache[0] != key:
        model._packed = (key, pack(model))
    return model._packed[1]


def launch(model, positions: Tensor, cell: Tensor, index: Tensor, *, energy: Tensor,
           forces: Tensor | None, virial: Tensor | None, status: Tensor,
           workspace: Tensor, weights: Tensor | None = None) -> None:
    """Launch the kernels into given buffers: energy [1] float64, forces [N, 3] float32 or
    None, virial [9] float64 or None, status [4] int32, and a workspace of at least
    ``workspace_bytes`` for the index's columns; ``weights`` a parameter block from ``pack``
    in place of the model's own. No allocation, no host sync: capturable."""
    args = SchNetArgs(
        num_atoms=model.num_atoms, num_columns=index.shape[1], interactions=len(model.blocks),
        num_types=model.num_types, gaussians=model.gaussians, reserved=0,
        cutoff=model.cutoff, positions=ptr(positions), cell=ptr(cell), pairs=ptr(index),
        atom_types=ptr(model.atom_types),
        weights=ptr(packed(model) if weights is None else weights), workspace=ptr(workspace),
        energy=ptr(energy), forces=ptr(forces), virial=ptr(virial), status=ptr(status),
    )
    call("nd_schnet_energy_force_virial", ctypes.byref(args), stream_handle(positions.device))


def energy_force_virial(model, positions: Tensor, cell: Tensor, pairs: NeighborPairs,
                        forces: bool = True, virial: bool = True):
    """(E, F [N, 3], W [3, 3]) in the model's dtype from the fused kernels; positions wrapped.

    The count of pairs within the cutoff, the status bits and the diagnostics of a tensor-core
    product that did not complete land in ``model._status`` [4] (int32, on the device; read
    without a sync only when wanted).
    """
    device = positions.device
    n = model.num_atoms
    index = pairs.index
    if index.dtype != torch.int32:
        index = index.to(torch.int32)
    index = index.contiguous()
    workspace = torch.empty(workspace_bytes(n, index.shape[1], len(model.blocks)),
                            dtype=torch.uint8, device=device)
    energy = torch.empty(1, dtype=torch.float64, device=device)
    out_forces = torch.empty((n, 3), dtype=torch.float32, device=device) if forces else None
    out_virial = torch.empty(9, dtype=torch.float64, device=device) if virial else None
    status = torch.empty(4, dtype=torch.int32, device=device)
    launch(model, positions.contiguous(), cell.contiguous(), index, energy=energy,
           forces=out_forces, virial=out_virial, status=status, workspace=workspace)
    model._status = status
    e = energy[0].to(model.dtype)
    w = out_virial.view(3, 3).to(model.dtype) if virial else None
    return e, out_forces, w


__all__ = ("pack", "packed", "launch", "energy_force_virial", "weight_bytes", "workspace_bytes")
