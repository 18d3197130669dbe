"""The parameter gradient of a SchNet training loss, on the fused kernels.

The loss of src/nabladyn/training/_loss.py:105-125 over E, F and W, and its gradient in the
parameters, which the reference takes with torch.func through a double backward
(src/nabladyn/training/_fit.py:245-271). Here it is forward-over-reverse, frame by frame:

1. E, F and W from the fused kernels (nd_schnet_energy_force_virial);
2. the frame's loss term and its adjoints e_bar = dL/dE, f_bar = dL/dF, w_bar = dL/dW;
3. a forward pass that carries beside every value its derivative along the direction in which
   pair p's distance moves at rdot_p = (d . (f_bar_a - f_bar_b) + d^T w_bar d) / r, since
   f_bar . F + w_bar : W is minus the derivative of E along it;
4. one reverse pass over both streams of Phi = e_bar E - Edot, whose parameter gradient is
   the loss's.

The per-pair work of steps 3 and 4 (the filter network with its tangent, the messages and their
reverse) runs in the tcgen05 tangent kernels (nd_schnet_tangent); the atom-wise layers, the
readout and their weights' gradients in the FP32 atom kernels (nd_schnet_atoms); the sums over
pairs of the filter weights' gradients are GEMMs with FP32 results. Operands of the per-pair
products are BF16, as in the E/F/W kernels, so the gradient agrees with the float64 definition
to the BF16 level, not bitwise. One frame's work is one CUDA graph over static buffers,
replayed frame after frame.
"""

from __future__ import annotations

import ctypes
import weakref
from collections.abc import Mapping

import torch
from torch import Tensor

from .._native import SchNetAtomArgs, SchNetTangentArgs, call, lib, ptr, stream_handle
from ..potential import _schnet_kernels as kernels

_ROWS = 8
# Each model's plan (buffers and graph), beside the model rather than on it, so the module
# still deep-copies and pickles; dropped with the model.
_PLANS: "weakref.WeakKeyDictionary" = weakref.WeakKeyDictionary()
# The atom kernels' per-atom arrays the host hands on (nd_schnet_atom_offset kinds): per block
# m, m_dot, v_bar, v_dot_bar (FP32) and v, v_dot (BF16); x_bar (FP32); m_bar, m_dot_bar (BF16).
_M, _M_DOT, _V_BAR, _V_DOT_BAR = 4, 5, 6, 7
_X_BAR, _V, _V_DOT, _M_BAR, _M_DOT_BAR = 10, 12, 13, 14, 15
# Offsets (floats) of the atom-side parameter block: per block A, D1, d1, D2, d2; readout.
_BLOCK_FLOATS = 3 * 4096 + 2 * 64
_BLOCK_PARTS = (("atoms.weight", 0, (64, 64)), ("update1.weight", 4096, (64, 64)),
                ("update1.bias", 8192, (64,)), ("update2.weight", 8256, (64, 64)),
                ("update2.bias", 12352, (64,)))
_READOUT_PARTS = (("readout1.weight", 0, (32, 64)), ("readout1.bias", 2048, (32,)),
                  ("readout2.weight", 2080, (1, 32)), ("readout2.bias", 2112, (1,)))
_READOUT_FLOATS = 2048 + 3 * 32


def supported(model) -> bool:
    """Whether the model's gradient runs here: a SchNet whose E/F/W use the fused kernels."""
    from ..potential._schnet import SchNet

    return isinstance(model, SchNet) and model._fused_kernel


class _Buffers:
    """Device buffers of one model size and pair-list width, reused frame after frame."""

    def __init__(self, model, columns: int):
        device = model.device
        n = model.num_atoms
        blocks = len(model.blocks)
        self.columns = columns
        self.workspace = torch.empty(kernels.workspace_bytes(n, columns, blocks),
                                     dtype=torch.uint8, device=device)
        self.energy = torch.empty(1, dtype=torch.float64, device=device)
        self.forces = torch.empty((n, 3), dtype=torch.float32, device=device)
        self.virial = torch.empty(9, dtype=torch.float64, device=device)
        self.status = torch.empty(4, dtype=torch.int32, device=device)
        self.rows = torch.empty((_ROWS, max(columns, 1), 64), dtype=torch.bfloat16, device=device)
        self.ones = torch.ones((1, max(columns, 1)), dtype=torch.bfloat16, device=device)
        self.atoms = torch.empty(int(lib().nd_schnet_atom_workspace_bytes(n, blocks)),
                                 dtype=torch.uint8, device=device)
        self.n, self.blocks = n, blocks

    def view(self, kind: int, block: int = 0) -> Tensor:
        """Array `kind` (of `block`) of the atom kernels' workspace, [N, 64]."""
        offset = int(lib().nd_schnet_atom_offset(self.n, self.blocks, kind, block))
        bf16 = kind >= _V
        size = self.n * 64 * (2 if bf16 else 4)
        return self.atoms[offset:offset + size].view(
            torch.bfloat16 if bf16 else torch.float32).view(self.n, 64)


def _tangent(model, buffers: _Buffers, weights: Tensor, block: int, direction: int,
             force_adjoint: Tensor, virial_adjoint: Tensor) -> None:
    reverse = direction == 1
    view = buffers.view
    args = SchNetTangentArgs(
        num_atoms=model.num_atoms, num_columns=buffers.columns,
        interactions=len(model.blocks), num_types=model.num_types, gaussians=model.gaussians,
        block=block, cutoff=model.cutoff, weights=ptr(weights), workspace=ptr(buffers.workspace),
        force_adjoint=ptr(force_adjoint), virial_adjoint=ptr(virial_adjoint),
        v=ptr(view(_V, block)), v_dot=ptr(view(_V_DOT, block)),
        m=None if reverse else ptr(view(_M, block)),
        m_dot=None if reverse else ptr(view(_M_DOT, block)),
        m_bar=ptr(view(_M_BAR)) if reverse else None,
        m_dot_bar=ptr(view(_M_DOT_BAR)) if reverse else None,
        v_bar=ptr(view(_V_BAR, block)) if reverse else None,
        v_dot_bar=ptr(view(_V_DOT_BAR, block)) if reverse else None,
        pair_rows=ptr(buffers.rows) if reverse else None, capacity=buffers.rows.shape[1],
        status=ptr(buffers.status),
    )
    call("nd_schnet_tangent", ctypes.byref(args), direction, stream_handle(force_adjoint.device))


def _atoms(model, buffers: _Buffers, parameters: Tensor, gradient: Tensor, e_bar: Tensor,
           stage: int, block: int) -> None:
    args = SchNetAtomArgs(
        num_atoms=model.num_atoms, interactions=len(model.blocks), num_types=model.num_types,
        atom_types=ptr(model.atom_types), parameters=ptr(parameters), gradient=ptr(gradient),
        energy_adjoint=ptr(e_bar), workspace=ptr(buffers.atoms),
    )
    call("nd_schnet_atoms", ctypes.byref(args), stage, block, stream_handle(gradient.device))


def atom_parameters(values: Mapping[str, Tensor], blocks: int) -> Tensor:
    """The FP32 atom-side parameter block of nd_schnet_atoms from parameters by name."""
    parts = []
    for b in range(blocks):
        parts += [values[f"blocks.{b}.{name}"].reshape(-1) for name, _, _ in _BLOCK_PARTS]
    parts += [values[name].reshape(-1) for name, _, _ in _READOUT_PARTS]
    e2 = parts.pop()
    parts += [e2, e2.new_zeros(31), values["embedding"].reshape(-1)]
    return torch.cat([part.float() for part in parts])


def atom_gradient_views(block: Tensor, blocks: int) -> dict[str, Tensor]:
    """The parameters' views into a gradient block laid out as atom_parameters."""
    views = {}
    for b in range(blocks):
        for name, offset, shape in _BLOCK_PARTS:
            start = b * _BLOCK_FLOATS + offset
            views[f"blocks.{b}.{name}"] = block[start:start + _numel(shape)].view(shape)
    base = blocks * _BLOCK_FLOATS
    for name, offset, shape in _READOUT_PARTS:
        views[name] = block[base + offset:base + offset + _numel(shape)].view(shape)
    views["embedding"] = block[base + _READOUT_FLOATS:].view(-1, 64)
    return views


def _numel(shape: tuple[int, ...]) -> int:
    total = 1
    for size in shape:
        total *= size
    return total


def _frame_loss(energy: Tensor, forces: Tensor, virial: Tensor, labels: Mapping[str, Tensor],
                weights: Mapping[str, Tensor], scales: Mapping[str, Tensor], coefficient: Tensor):
    """The frame's loss term (float64, on the device) and its adjoints: e_bar (0-d), f_bar
    [N, 3] float32, w_bar [9] float64 (zeros for channels without a weight). Weights, scales
    and the frame's coefficient are 0-d float64 device tensors."""
    predicted = {"energy": energy.double().reshape(()), "forces": forces.double(),
                 "virial": virial.double().reshape(3, 3)}
    value = torch.zeros((), dtype=torch.float64, device=forces.device)
    adjoints = {}
    for name, x in predicted.items():
        if name not in weights:
            adjoints[name] = torch.zeros_like(x)
            continue
        error = (x - labels[name]) / scales[name]
        value = value + coefficient * weights[name] * error.square().mean()
        adjoints[name] = coefficient * weights[name] * 2.0 * error / scales[name] / error.numel()
    return (value, adjoints["energy"], adjoints["forces"].float().contiguous(),
            adjoints["virial"].reshape(9).contiguous())


def _frame_gradient(model, plan, e_bar: Tensor, f_bar: Tensor, w_bar: Tensor) -> None:
    """Adds one frame's d(e_bar E - Edot)/dtheta to the plan's gradient (steps 3 and 4)."""
    buffers, blob = plan.buffers, plan.blob
    blocks = len(model.blocks)
    k = model.gaussians

    def atoms(stage: int, block: int = 0) -> None:
        _atoms(model, buffers, plan.atom_parameters, plan.atom_gradient, e_bar, stage, block)

    atoms(0)
    for b in range(blocks):
        _tangent(model, buffers, blob, b, 0, f_bar, w_bar)
        atoms(1, b)
    atoms(2)
    f32 = torch.float32
    for b in reversed(range(blocks)):
        atoms(3, b)
        _tangent(model, buffers, blob, b, 1, f_bar, w_bar)
        # rows past the pair count are zero, so the sums run over every row
        g, g_dot, s, s_dot, z_bar, z_dot_bar, u_bar, u_dot_bar = buffers.rows.unbind(0)
        name = f"blocks.{b}."
        gradient = plan.gradient
        gradient[name + "filter2.weight"] += (torch.mm(u_bar.T, s, out_dtype=f32)
                                             + torch.mm(u_dot_bar.T, s_dot, out_dtype=f32))
        gradient[name + "filter2.bias"] += torch.mm(buffers.ones, u_bar, out_dtype=f32)[0]
        filter1 = (torch.mm(z_bar.T, g, out_dtype=f32)
                   + torch.mm(z_dot_bar.T, g_dot, out_dtype=f32))
        gradient[name + "filter1.weight"] += filter1[:, :k]
        # with K < 64 the kernel's g rows carry 1 in column 63: the sum of z_bar
        gradient[name + "filter1.bias"] += (filter1[:, 63] if k < 64
                                            else z_bar.sum(dim=0, dtype=f32))
        atoms(4, b)
    plan.gradient["embedding"].index_add_(0, model.atom_types, buffers.view(_X_BAR))


def _plan_key(model, columns: int, channels: tuple[str, ...]) -> tuple:
    """What a plan's buffers and captured graph depend on besides the parameter values (copied
    in at every call): the stack width, the channels, the device, the sizes (atoms, types,
    blocks) and the atom-type buffer (a new buffer at a freed address has other sizes or a
    new version)."""
    types = model.atom_types
    return (columns, channels, str(model.device), model.num_atoms, model.num_types,
            len(model.blocks), tuple(types.shape), types.data_ptr(), types._version)


class _Plan:
    """Static buffers for one pair-stack width and set of loss channels (parameters, the frame's
    inputs and labels, the loss weights, the accumulated loss, gradient and status bits) and
    the CUDA graph of one frame's work over them: the first frame ever runs eagerly (it
    configures the kernels and the GEMM library), the second is captured, every later one is
    a replay. Kept beside the model for its next call."""

    def __init__(self, model, columns: int, channels: tuple[str, ...]):
        device = model.device
        n = model.num_atoms
        f64 = torch.float64
        self.key = _plan_key(model, columns, channels)
        self.device = device
        self.buffers = _Buffers(model, columns)
        self.values = {name: torch.empty(value.shape, dtype=torch.float32, device=device)
                       for name, value in model.named_parameters()}
        self.blob = torch.empty(kernels.weight_bytes(len(model.blocks), model.num_types),
                                dtype=torch.uint8, device=device)
        self.positions = torch.empty((n, 3), dtype=torch.float32, device=device)
        self.cell = torch.empty(3, dtype=torch.float32, device=device)
        self.index = torch.empty((2, columns), dtype=torch.int32, device=device)
        shapes = {"energy": (), "forces": (n, 3), "virial": (3, 3)}
        self.labels = {name: torch.empty(shapes[name], dtype=f64, device=device)
                       for name in channels}
        self.weights = {name: torch.empty((), dtype=f64, device=device) for name in channels}
        self.scales = {name: torch.empty((), dtype=f64, device=device) for name in channels}
        self.coefficient = torch.empty((), dtype=f64, device=device)
        blocks = len(model.blocks)
        self.atom_parameters = torch.empty(
            int(lib().nd_schnet_atom_parameter_floats(blocks, model.num_types)),
            dtype=torch.float32, device=device)
        self.atom_gradient = torch.zeros_like(self.atom_parameters)
        self.gradient = {name: torch.zeros_like(value) for name, value in self.values.items()}
        # the atom-side parameters' gradients are views into the atom kernels' gradient block
        self.gradient.update(atom_gradient_views(self.atom_gradient, blocks))
        self.total = torch.zeros((), dtype=f64, device=device)
        self.bits = torch.zeros((), dtype=torch.int32, device=device)
        self.warm = False
        self.graph = None

    def frame(self, model) -> None:
        """One frame's loss and gradient from the static inputs, added to the accumulators."""
        b = self.buffers
        x = torch.remainder(self.positions, self.cell)
        kernels.launch(model, x, self.cell, self.index, energy=b.energy, forces=b.forces,
                       virial=b.virial, status=b.status, workspace=b.workspace,
                       weights=self.blob)
        value, e_bar, f_bar, w_bar = _frame_loss(b.energy[0], b.forces, b.virial, self.labels,
                                                 self.weights, self.scales, self.coefficient)
        self.total += value
        _frame_gradient(model, self, e_bar, f_bar, w_bar)
        # the counters hold the frame's E/F/W and tangent bits; the last copy has them all
        self.bits.bitwise_or_(b.status[1])

    def run(self, model) -> None:
        if self.graph is not None:
            self.graph.replay()
            return
        if not self.warm:
            side = torch.cuda.Stream(self.device)
            side.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(side):
                self.frame(model)
            torch.cuda.current_stream(self.device).wait_stream(side)
            self.warm = True
            return
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.frame(model)
        self.graph = graph
        graph.replay()


def loss_and_gradient(model, parameters: Mapping[str, Tensor], positions: Tensor, cells: Tensor,
                      stacks: tuple[Tensor, ...], labels: Mapping[str, Tensor],
                      weights: Mapping[str, float], scales: Mapping[str, float]
                      ) -> tuple[Tensor, dict[str, Tensor]]:
    """The batch loss (frames weighted 1/B) and its gradient in ``parameters`` (by name; the
    model's own values for the names not given), for a model with ``supported(model)``.

    positions [B, N, 3], cells [B, 3], one [B, 2, C] pair stack; labels of the weighted
    channels. Each frame is a few input copies and one CUDA-graph replay; the call syncs with
    the host once, at its end. The buffers (about 1 KB per stack column) and the graph stay
    beside the model (until it is freed) for its next call with the same stack width and
    channels. Raises
    ``RuntimeError`` when a kernel reports a pair index out of range or a tensor-core product
    that did not complete.
    """
    if not supported(model):
        raise ValueError("the fused SchNet gradient needs a float32 SchNet on a GPU with 64 "
                         "features and at most 64 Gaussians")
    stack = stacks[-1]
    frames, columns = positions.shape[0], stack.shape[-1]
    channels = tuple(name for name in ("energy", "forces", "virial") if name in weights)
    plan = _PLANS.get(model)
    if plan is None or plan.key != _plan_key(model, columns, channels):
        _PLANS.pop(model, None)
        plan = _Plan(model, columns, channels)
        _PLANS[model] = plan
    values = {name: value.detach().float() for name, value in model.named_parameters()}
    values.update({name: value.detach().float() for name, value in parameters.items()})
    with torch.no_grad():
        for name, value in values.items():
            plan.values[name].copy_(value)
        plan.blob.copy_(kernels.pack(model, values))
        plan.atom_parameters.copy_(atom_parameters(values, len(model.blocks)))
        for name in channels:
            plan.weights[name].fill_(float(weights[name]))
            plan.scales[name].fill_(float(scales[name]))
        plan.coefficient.fill_(1.0 / frames)
        plan.total.zero_()
        plan.bits.zero_()
        for value in plan.gradient.values():
            value.zero_()
        plan.atom_gradient.zero_()
        for f in range(frames):
            plan.positions.copy_(positions[f])
            plan.cell.copy_(cells[f])
            plan.index.copy_(stack[f])
            for name in channels:
                plan.labels[name].copy_(labels[name][f])
            plan.run(model)
    bits = int(plan.bits)
    if bits:
        raise RuntimeError(f"SchNet kernels reported status {bits} (1: a pair index out of "
                           "range; 16: a tensor-core product did not complete)")
    return plan.total.clone(), {name: plan.gradient[name].to(value.dtype, copy=True)
                                for name, value in parameters.items()}


__all__ = ("supported", "loss_and_gradient")
