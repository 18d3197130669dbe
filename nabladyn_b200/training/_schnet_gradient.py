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
reverse) runs in the tcgen05 tangent kernels (nd_schnet_tangent); the atom-wise 64 x 64 layers,
the readout and the sums over pairs of the filter weights' gradients are GEMMs with FP32
results. Operands of the per-pair products are BF16, as in the E/F/W kernels, so the gradient
agrees with the float64 definition to the BF16 level, not bitwise. One frame's work is one CUDA
graph over static buffers, replayed frame after frame.
"""

from __future__ import annotations

import ctypes
import weakref
from collections.abc import Mapping

import torch
import torch.nn.functional as functional
from torch import Tensor

from .._native import SchNetTangentArgs, call, ptr, stream_handle
from ..potential import _schnet_kernels as kernels

_ROWS = 8
# Each model's plan (buffers and graph), beside the model rather than on it, so the module
# still deep-copies and pickles; dropped with the model.
_PLANS: "weakref.WeakKeyDictionary" = weakref.WeakKeyDictionary()
_LN2 = 0.6931471805599453
_CHUNK_ROWS = 1024


def supported(model) -> bool:
    """Whether the model's gradient runs here: a SchNet whose E/F/W use the fused kernels."""
    from ..potential._schnet import SchNet

    return isinstance(model, SchNet) and model._fused_kernel


def _ssp(x: Tensor) -> Tensor:
    return functional.softplus(x) - _LN2


def _gram(*terms: tuple[Tensor, Tensor]) -> Tensor:
    """sum_i a_i^T b_i over [N, p] and [N, q] float32 pairs: one batched GEMM over chunks of
    1,024 rows and a sum of the chunks (a p x q product with a long reduction would otherwise
    run on a single CTA)."""
    a = torch.cat([x for x, _ in terms])
    b = torch.cat([y for _, y in terms])
    pad = -a.shape[0] % _CHUNK_ROWS
    if pad:
        a = functional.pad(a, (0, 0, 0, pad))
        b = functional.pad(b, (0, 0, 0, pad))
    a = a.view(-1, _CHUNK_ROWS, a.shape[1])
    b = b.view(-1, _CHUNK_ROWS, b.shape[1])
    return torch.bmm(a.transpose(1, 2), b).sum(dim=0)


class _Buffers:
    """Device buffers of one model size and pair-list width, reused frame after frame."""

    def __init__(self, model, columns: int):
        device = model.device
        n = model.num_atoms
        self.columns = columns
        self.workspace = torch.empty(kernels.workspace_bytes(n, columns, len(model.blocks)),
                                     dtype=torch.uint8, device=device)
        self.energy = torch.empty(1, dtype=torch.float64, device=device)
        self.forces = torch.empty((n, 3), dtype=torch.float32, device=device)
        self.virial = torch.empty(9, dtype=torch.float64, device=device)
        self.status = torch.empty(4, dtype=torch.int32, device=device)
        self.m = torch.empty((n, 64), dtype=torch.float32, device=device)
        self.m_dot = torch.empty_like(self.m)
        self.v_bar = torch.empty_like(self.m)
        self.v_dot_bar = torch.empty_like(self.m)
        self.rows = torch.empty((_ROWS, max(columns, 1), 64), dtype=torch.bfloat16, device=device)
        self.ones = torch.ones((1, max(columns, 1)), dtype=torch.bfloat16, device=device)


def _tangent(model, buffers: _Buffers, weights: Tensor, block: int, direction: int,
             force_adjoint: Tensor, virial_adjoint: Tensor, v: Tensor, v_dot: Tensor,
             m_bar: Tensor | None = None, m_dot_bar: Tensor | None = None) -> None:
    reverse = direction == 1
    args = SchNetTangentArgs(
        num_atoms=model.num_atoms, num_columns=buffers.columns,
        interactions=len(model.blocks), num_types=model.num_types, gaussians=model.gaussians,
        block=block, cutoff=model.cutoff, weights=ptr(weights), workspace=ptr(buffers.workspace),
        force_adjoint=ptr(force_adjoint), virial_adjoint=ptr(virial_adjoint), v=ptr(v),
        v_dot=ptr(v_dot), m=None if reverse else ptr(buffers.m),
        m_dot=None if reverse else ptr(buffers.m_dot),
        m_bar=ptr(m_bar) if reverse else None, m_dot_bar=ptr(m_dot_bar) if reverse else None,
        v_bar=ptr(buffers.v_bar) if reverse else None,
        v_dot_bar=ptr(buffers.v_dot_bar) if reverse else None,
        pair_rows=ptr(buffers.rows) if reverse else None, capacity=buffers.rows.shape[1],
        status=ptr(buffers.status),
    )
    call("nd_schnet_tangent", ctypes.byref(args), direction, stream_handle(v.device))


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


def _frame_gradient(model, values: Mapping[str, Tensor], weights_blob: Tensor,
                    buffers: _Buffers, e_bar: Tensor, f_bar: Tensor, w_bar: Tensor,
                    gradient: dict[str, Tensor]) -> None:
    """Adds one frame's d(e_bar E - Edot)/dtheta to ``gradient`` (steps 3 and 4)."""
    def w(name: str) -> Tensor:
        return values[name]

    blocks = len(model.blocks)
    x = w("embedding")[model.atom_types]
    x_dot = torch.zeros_like(x)
    saved = []
    for b in range(blocks):
        a = w(f"blocks.{b}.atoms.weight")
        v = (x @ a.T).to(torch.bfloat16)
        v_dot = (x_dot @ a.T).to(torch.bfloat16)
        buffers.m.zero_()
        buffers.m_dot.zero_()
        _tangent(model, buffers, weights_blob, b, 0, f_bar, w_bar, v, v_dot)
        m, m_dot = buffers.m.clone(), buffers.m_dot.clone()
        d1 = w(f"blocks.{b}.update1.weight")
        h = torch.addmm(w(f"blocks.{b}.update1.bias"), m, d1.T)
        h_dot = m_dot @ d1.T
        saved.append((x, x_dot, v, v_dot, m, m_dot, h, h_dot))
        d2 = w(f"blocks.{b}.update2.weight")
        x = x + torch.addmm(w(f"blocks.{b}.update2.bias"), _ssp(h), d2.T)
        x_dot = x_dot + (torch.sigmoid(h) * h_dot) @ d2.T
    r1, r2 = w("readout1.weight"), w("readout2.weight")[0]
    y = torch.addmm(w("readout1.bias"), x, r1.T)
    y_dot = x_dot @ r1.T
    sy = torch.sigmoid(y)
    e = e_bar.float()
    y_bar = (e * sy - sy * (1.0 - sy) * y_dot) * r2
    y_dot_bar = -sy * r2
    gradient["readout2.weight"][0] += (e * _ssp(y) - sy * y_dot).sum(dim=0)
    gradient["readout2.bias"][0] += e * model.num_atoms
    gradient["readout1.weight"] += _gram((y_bar, x), (y_dot_bar, x_dot))
    gradient["readout1.bias"] += y_bar.sum(dim=0)
    x_bar, x_dot_bar = y_bar @ r1, y_dot_bar @ r1
    k = model.gaussians
    for b in reversed(range(blocks)):
        x, x_dot, v, v_dot, m, m_dot, h, h_dot = saved[b]
        name = f"blocks.{b}."
        d2, d1 = w(name + "update2.weight"), w(name + "update1.weight")
        sg = torch.sigmoid(h)
        gradient[name + "update2.weight"] += _gram((x_bar, _ssp(h)), (x_dot_bar, sg * h_dot))
        gradient[name + "update2.bias"] += x_bar.sum(dim=0)
        ssp_bar, q_bar = x_bar @ d2, x_dot_bar @ d2
        h_bar = ssp_bar * sg + q_bar * h_dot * sg * (1.0 - sg)
        h_dot_bar = q_bar * sg
        gradient[name + "update1.weight"] += _gram((h_bar, m), (h_dot_bar, m_dot))
        gradient[name + "update1.bias"] += h_bar.sum(dim=0)
        m_bar = (h_bar @ d1).to(torch.bfloat16)
        m_dot_bar = (h_dot_bar @ d1).to(torch.bfloat16)
        buffers.v_bar.zero_()
        buffers.v_dot_bar.zero_()
        _tangent(model, buffers, weights_blob, b, 1, f_bar, w_bar, v, v_dot, m_bar, m_dot_bar)
        # rows past the pair count are zero, so the sums run over every row
        g, g_dot, s, s_dot, z_bar, z_dot_bar, u_bar, u_dot_bar = buffers.rows.unbind(0)
        f32 = torch.float32
        gradient[name + "filter2.weight"] += (torch.mm(u_bar.T, s, out_dtype=f32)
                                             + torch.mm(u_dot_bar.T, s_dot, out_dtype=f32))
        gradient[name + "filter2.bias"] += torch.mm(buffers.ones, u_bar, out_dtype=f32)[0]
        filter1 = (torch.mm(z_bar.T, g, out_dtype=f32)
                   + torch.mm(z_dot_bar.T, g_dot, out_dtype=f32))
        gradient[name + "filter1.weight"] += filter1[:, :k]
        # with K < 64 the kernel's g rows carry 1 in column 63: the sum of z_bar
        gradient[name + "filter1.bias"] += (filter1[:, 63] if k < 64
                                            else z_bar.sum(dim=0, dtype=f32))
        a = w(name + "atoms.weight")
        v_bar, v_dot_bar = buffers.v_bar, buffers.v_dot_bar
        gradient[name + "atoms.weight"] += _gram((v_bar, x), (v_dot_bar, x_dot))
        x_bar = x_bar + v_bar @ a
        x_dot_bar = x_dot_bar + v_dot_bar @ a
    gradient["embedding"].index_add_(0, model.atom_types, x_bar)


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
        self.key = (columns, channels)
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
        self.gradient = {name: torch.zeros_like(value) for name, value in self.values.items()}
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
        _frame_gradient(model, self.values, self.blob, b, e_bar, f_bar, w_bar, self.gradient)
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
    if plan is None or plan.key != (columns, channels):
        _PLANS.pop(model, None)
        plan = _Plan(model, columns, channels)
        _PLANS[model] = plan
    values = {name: value.detach().float() for name, value in model.named_parameters()}
    values.update({name: value.detach().float() for name, value in parameters.items()})
    with torch.no_grad():
        for name, value in values.items():
            plan.values[name].copy_(value)
        plan.blob.copy_(kernels.pack(model, values))
        for name in channels:
            plan.weights[name].fill_(float(weights[name]))
            plan.scales[name].fill_(float(scales[name]))
        plan.coefficient.fill_(1.0 / frames)
        plan.total.zero_()
        plan.bits.zero_()
        for value in plan.gradient.values():
            value.zero_()
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
