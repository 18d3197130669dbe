"""Batched Lennard-Jones predictions with a hand-written parameter backward.

``predict`` gives the energy, forces and virial of F frames in one kernel launch
(nd_lj_batch_forward); its autograd backward is nd_lj_batch_parameter_backward, which turns the
loss's gradients with respect to E, F and W into dLoss/dsigma and dLoss/depsilon in one pass
over the pairs. The reference gets the same numbers by a torch.func double backward through
vmapped forces (src/nabladyn/training/_loss.py:71-102, _fit.py:245-271).
"""

from __future__ import annotations

from collections.abc import Mapping

import torch
from torch import Tensor

from .. import space
from .._native import LJBatchArgs, call, dtype_code, ptr, stream_handle
from ..potential._lennard_jones import LennardJones

CHANNELS = ("energy", "forces", "virial")


def _args(positions, cells, stacks, kernel_types, num_types, sigma, epsilon, cutoff):
    frames, atoms = positions.shape[:2]
    return LJBatchArgs(
        dtype=dtype_code(positions.dtype),
        frames=frames,
        positions=ptr(positions),
        cells=ptr(cells),
        num_atoms=atoms,
        pairs=ptr(stacks),
        capacity=stacks.shape[2],
        atom_types=ptr(kernel_types) if num_types > 1 else None,
        num_types=num_types,
        sigma=ptr(sigma),
        epsilon=ptr(epsilon),
        cutoff=float(cutoff),
    )


class _BatchLJ(torch.autograd.Function):
    """(sigma, epsilon) -> (E [F], F [F, N, 3], W [F, 3, 3]) of fixed wrapped frames."""

    @staticmethod
    def forward(ctx, sigma, epsilon, positions, cells, stacks, kernel_types, num_types, cutoff):
        dtype, device = positions.dtype, positions.device
        frames, atoms = positions.shape[:2]
        sigma_c = sigma.detach().to(dtype).contiguous()
        epsilon_c = epsilon.detach().to(dtype).contiguous()
        energy = torch.empty(frames, dtype=torch.float64, device=device)
        forces = torch.empty((frames, atoms, 3), dtype=dtype, device=device)
        virial = torch.empty((frames, 3, 3), dtype=torch.float64, device=device)
        args = _args(positions, cells, stacks, kernel_types, num_types, sigma_c, epsilon_c, cutoff)
        args.energy, args.forces, args.virial = ptr(energy), ptr(forces), ptr(virial)
        with torch.cuda.device(device):
            call("nd_lj_batch_forward", args, stream_handle(device))
        ctx.save_for_backward(sigma_c, epsilon_c, positions, cells, stacks, kernel_types)
        ctx.num_types, ctx.cutoff = num_types, cutoff
        ctx.parameter_dtype = sigma.dtype
        return energy.to(dtype), forces, virial.to(dtype)

    @staticmethod
    def backward(ctx, grad_energy, grad_forces, grad_virial):
        sigma, epsilon, positions, cells, stacks, kernel_types = ctx.saved_tensors
        dtype, device = positions.dtype, positions.device
        frames, atoms = positions.shape[:2]
        ge = (grad_energy if grad_energy is not None
              else torch.zeros(frames, device=device)).to(torch.float64).contiguous()
        gf = (grad_forces if grad_forces is not None
              else torch.zeros((frames, atoms, 3), device=device)).to(dtype).contiguous()
        gw = (grad_virial if grad_virial is not None
              else torch.zeros((frames, 3, 3), device=device)).to(torch.float64).contiguous()
        rows = sigma.numel()
        grads = torch.empty((2, rows), dtype=torch.float64, device=device)
        args = _args(positions, cells, stacks, kernel_types, ctx.num_types, sigma, epsilon,
                     ctx.cutoff)
        args.energy_grad, args.forces_grad, args.virial_grad = ptr(ge), ptr(gf), ptr(gw)
        args.sigma_grad, args.epsilon_grad = grads[0].data_ptr(), grads[1].data_ptr()
        with torch.cuda.device(device):
            call("nd_lj_batch_parameter_backward", args, stream_handle(device))
        out_dtype = ctx.parameter_dtype
        return grads[0].to(out_dtype), grads[1].to(out_dtype), None, None, None, None, None, None


def predict(model: LennardJones, parameters: Mapping[str, Tensor], positions: Tensor,
            cells: Tensor, stacks: tuple[Tensor, ...], channels: tuple[str, ...]) -> dict[str, Tensor]:
    """The channels of F frames by name, differentiable in ``parameters``.

    Lennard-Jones runs the batched kernels and the hand-written backward; any other model the
    reference's torch.func algorithm (``_generic.predict``).

    positions [F, N, 3] (anywhere), cells [F, 3], ``stacks`` one [F, 2, C] pair stack per
    cutoff of the model (one for Lennard-Jones); ``parameters`` replaces the model's "sigma"
    and/or "epsilon". Gives energy [F], forces [F, N, 3], virial [F, 3, 3]. Gradients flow to
    the parameters only.
    """
    if not isinstance(model, LennardJones):
        from ._generic import predict as generic_predict

        return generic_predict(model, parameters, positions, cells, stacks, channels)
    unknown = set(channels) - set(CHANNELS)
    if not channels or unknown:
        raise ValueError(f"channels must be a nonempty subsequence of {CHANNELS}")
    sigma = parameters.get("sigma", model.sigma)
    epsilon = parameters.get("epsilon", model.epsilon)
    wrapped = space.wrap(positions.detach(), cells.detach()[:, None])[0].contiguous()
    stack = stacks[-1]
    if stack.dtype != torch.int32:
        stack = stack.to(torch.int32)
    energy, forces, virial = _BatchLJ.apply(
        sigma, epsilon, wrapped, cells.detach().contiguous(), stack.contiguous(),
        model._kernel_types, model.num_types, model.cutoff,
    )
    values = {"energy": energy, "forces": forces, "virial": virial}
    return {name: values[name] for name in channels}


__all__ = ("predict", "CHANNELS")
