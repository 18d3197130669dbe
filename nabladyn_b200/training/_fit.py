"""Fitting a potential's parameters to labeled frames: ``Dataset``, ``fit`` and its ``Report``.

The interface and update rule of src/nabladyn/training/_fit.py:332-439 and _dataset.py:44-102:
frames prepared once with their pair stacks, batches from one seeded shuffle per epoch, the
batch's loss gradient written into ``.grad`` and ``optimizer.step()``, rows the model does not
train held, RMS errors before and after. The gradient of a Lennard-Jones model comes from the
batched kernels and their hand-written parameter backward in one pass over the batch; any
other model's from the reference's torch.func algorithm in chunks of frames. Given a process
group, the frames of each batch are split over its ranks (``_parallel``).
"""

from __future__ import annotations

import dataclasses
import math
from numbers import Integral, Real

import numpy as np
import torch
from torch import Tensor

from ..potential import Potential
from ..potential._lennard_jones import LennardJones
from . import _parallel
from ._generic import loss_and_gradient
from ._loss import CHANNELS, loss as batch_loss, scales as label_scales
from ._predict import predict
from ._stacks import pair_stack


def _host(value) -> Tensor:
    tensor = value if isinstance(value, Tensor) else torch.from_numpy(np.asarray(value))
    return tensor.detach().to("cpu", copy=True)


class Dataset:
    """Labeled frames of one topology, kept on the host.

    ``positions`` [F, N, 3] and ``cells`` [F, 3] in nm; optional ``energy`` [F] (kJ/mol),
    ``forces`` [F, N, 3] (kJ/mol/nm), ``virial`` [F, 3, 3] (kJ/mol); NumPy arrays or tensors of
    one dtype, float32 or float64. Indexing (int, slice, index array) selects frames. Raises
    ``ValueError`` for a wrong shape or dtype, a non-finite value or a nonpositive cell.
    """

    def __init__(self, positions, cells, *, energy=None, forces=None, virial=None):
        given = {"positions": positions, "cells": cells, "energy": energy, "forces": forces,
                 "virial": virial}
        fields = {name: _host(value) for name, value in given.items() if value is not None}
        x = fields["positions"]
        if x.ndim != 3 or x.shape[0] == 0 or x.shape[2] != 3:
            raise ValueError("positions must be [F, N, 3] with at least one frame")
        frames, atoms = x.shape[:2]
        shapes = {"positions": (frames, atoms, 3), "cells": (frames, 3), "energy": (frames,),
                  "forces": (frames, atoms, 3), "virial": (frames, 3, 3)}
        for name, value in fields.items():
            if tuple(value.shape) != shapes[name]:
                raise ValueError(f"{name} must be {list(shapes[name])}, not {list(value.shape)}")
            if value.dtype != x.dtype or value.dtype not in (torch.float32, torch.float64):
                raise ValueError("every field must share one dtype, float32 or float64")
            if not bool(torch.isfinite(value).all()):
                raise ValueError(f"{name} must be finite")
        if not bool((fields["cells"] > 0).all()):
            raise ValueError("cells must be positive")
        self._fields = fields

    def __len__(self) -> int:
        return self._fields["positions"].shape[0]

    def __getitem__(self, key) -> Dataset:
        index = torch.arange(len(self))[key] if isinstance(key, slice) else torch.as_tensor(key)
        index = index.cpu().reshape(-1)
        out = Dataset.__new__(Dataset)
        out._fields = {name: value[index] for name, value in self._fields.items()}
        return out

    @property
    def positions(self) -> Tensor:
        return self._fields["positions"]

    @property
    def cells(self) -> Tensor:
        return self._fields["cells"]

    @property
    def labels(self) -> dict[str, Tensor]:
        return {name: self._fields[name] for name in CHANNELS if name in self._fields}


@dataclasses.dataclass(frozen=True)
class Report:
    """``loss`` [updates] (each batch's loss before its step), ``scales``, and per weighted
    channel the RMS error (before, after) on ``training`` and ``validation`` (or None)."""

    loss: np.ndarray
    scales: dict[str, float]
    training: dict[str, tuple[float, float]]
    validation: dict[str, tuple[float, float]] | None


def batches(frames: int, batch_size: int, updates: int, seed: int) -> list[Tensor]:
    """Frame indices per update: each epoch a new shuffle from ``seed`` (a CPU generator, as
    the reference draws it), cut into batches, the last one the remainder."""
    generator = torch.Generator().manual_seed(seed)
    result = []
    while len(result) < updates:
        result.extend(torch.randperm(frames, generator=generator).split(batch_size))
    return result[:updates]


def _prepared(model, data: Dataset, channels):
    def move(value):
        return value.to(device=model.device, dtype=model.dtype)

    positions, cells = move(data.positions), move(data.cells)
    labels = {name: move(data.labels[name]) for name in channels}
    stack = pair_stack(positions, cells, model.cutoff)
    return positions, cells, stack, labels


def _errors(model, prepared, channels, size: int) -> dict[str, float]:
    positions, cells, stack, labels = prepared
    squares = dict.fromkeys(channels, 0.0)
    with torch.no_grad():
        for index in torch.arange(len(positions), device=positions.device).split(size):
            values = predict(model, {}, positions[index], cells[index], (stack[index],),
                             channels)
            for name in channels:
                squares[name] += float((values[name] - labels[name][index]).square().sum())
    return {name: math.sqrt(squares[name] / labels[name].numel()) for name in channels}


def _gradient(model, trained, prepared, frames, weights, scales, channels, chunk,
              process_group=None):
    """The batch's loss and gradient; with a process group, each rank differentiates its share
    of the frames and one all-reduce sums the frame-weighted shares."""
    if process_group is None:
        return _share_gradient(model, trained, prepared, frames, weights, scales, channels,
                               chunk)
    mine = _parallel.share(frames, process_group)
    if len(mine) > 0:
        value, grads = _share_gradient(model, trained, prepared, mine, weights, scales,
                                       channels, chunk)
    else:
        value = torch.zeros((), dtype=torch.float64, device=prepared[0].device)
        grads = {name: torch.zeros_like(tensor) for name, tensor in trained.items()}
    return _parallel.reduce(value, grads, len(mine) / len(frames), process_group)


def _share_gradient(model, trained, prepared, frames, weights, scales, channels, chunk):
    positions, cells, stack, labels = prepared
    index = frames.to(positions.device)
    part = {name: labels[name][index] for name in channels}
    if isinstance(model, LennardJones):
        params = {name: value.detach().clone().requires_grad_(True)
                  for name, value in trained.items()}
        predicted = predict(model, params, positions[index], cells[index], (stack[index],),
                            channels)
        value, _ = batch_loss(predicted, part, weights, scales)
        grads = torch.autograd.grad(value, list(params.values()))
        return value.detach(), dict(zip(params, grads))
    value, grads = loss_and_gradient(model, {k: v.detach() for k, v in trained.items()},
                                     positions[index], cells[index], (stack[index],), part,
                                     weights, scales, chunk=chunk)
    return value, grads


def fit(model: Potential, train: Dataset, optimizer: torch.optim.Optimizer, *, updates: Integral,
        batch_size: Integral, energy: Real | None = None, forces: Real | None = None,
        virial: Real | None = None, validation: Dataset | None = None, seed: Integral = 0,
        scheduler=None, echo_every: Integral | None = None, chunk: Integral = 4,
        process_group=None) -> Report:
    """Fit the model's trainable parameters to the training labels; return a ``Report``.

    A channel enters the loss when its weight is given: w mean(((X - X*) / s)^2), s from the
    training labels. Each of the ``updates`` takes the next batch of ``batch_size`` frames,
    writes the gradient of the batch's loss into ``.grad`` and steps the optimizer (and the
    ``scheduler`` after it); rows the model does not train keep their values. ``chunk`` bounds
    the frames a non-LJ model differentiates at once. With ``echo_every`` = k, prints the
    mean loss and terms every k updates. With ``process_group`` (torch.distributed, one rank
    per GPU, every rank calling ``fit`` with the same arguments), each update's frames are
    split over the ranks and their gradients summed by one all-reduce, so every rank takes
    the same step. Syncs with the host.

    Raises ``TypeError`` for a model that is not a Potential and ``ValueError`` for weights
    or counts out of range, no trainable parameter, or sets with another atom count or
    without the weighted labels.
    """
    if not isinstance(model, Potential):
        raise TypeError("model must be a Potential")
    weights = {name: value for name, value in (("energy", energy), ("forces", forces),
                                               ("virial", virial)) if value is not None}
    if not weights:
        raise ValueError("give at least one channel's weight: energy, forces or virial")
    for name, value in weights.items():
        if isinstance(value, bool) or not isinstance(value, Real) or not math.isfinite(value) \
                or value <= 0:
            raise ValueError(f"the {name} weight must be a finite positive number")
    for name, value in (("updates", updates), ("batch_size", batch_size), ("seed", seed),
                        ("echo_every", 1 if echo_every is None else echo_every)):
        if isinstance(value, bool) or not isinstance(value, Integral) or value < 0:
            raise ValueError(f"{name} must be a nonnegative integer")
    if updates == 0 or echo_every == 0 or not 0 < batch_size <= len(train):
        raise ValueError("updates and echo_every must be positive, and batch_size between 1 "
                         "and the training set's size")
    trained = {name: value for name, value in model.named_parameters() if value.requires_grad}
    if not trained:
        raise ValueError("the model has no trainable parameter; set trainable when building "
                         "the potential")
    masks = model._trained_masks()
    held = [(value, ~masks[name], value.detach().clone()) for name, value in trained.items()
            if name in masks]
    channels = tuple(name for name in CHANNELS if name in weights)
    sets = {"training": train} | ({"validation": validation} if validation is not None else {})
    for label, data in sets.items():
        if data.positions.shape[1] != model.num_atoms:
            raise ValueError(f"the {label} frames hold {data.positions.shape[1]} atoms, the "
                             f"model {model.num_atoms}")
        for name in channels:
            if name not in data.labels:
                raise ValueError(f"the {label} frames have no {name} labels")
    prepared = {label: _prepared(model, data, channels) for label, data in sets.items()}
    scales = label_scales(**prepared["training"][3])
    before = {label: _errors(model, data, channels, batch_size)
              for label, data in prepared.items()}
    losses = np.empty(updates)
    if echo_every is not None:
        print("update loss", flush=True)
    for update, frames in enumerate(batches(len(train), batch_size, updates, seed)):
        value, gradient = _gradient(model, trained, prepared["training"], frames, weights,
                                    scales, channels, int(chunk), process_group)
        optimizer.zero_grad()
        for name, parameter in trained.items():
            parameter.grad = gradient[name].to(parameter.dtype)
        for parameter, mask, _ in held:
            parameter.grad = parameter.grad.masked_fill(mask, 0)
        optimizer.step()
        with torch.no_grad():
            for parameter, mask, values in held:
                parameter.copy_(torch.where(mask, values, parameter))
        if scheduler is not None:
            scheduler.step()
        losses[update] = float(value)
        if echo_every is not None and (update + 1) % echo_every == 0:
            print(f"{update + 1} {losses[update + 1 - echo_every:update + 1].mean():.6g}",
                  flush=True)
    after = {label: _errors(model, data, channels, batch_size)
             for label, data in prepared.items()}
    errors = {label: {name: (before[label][name], after[label][name]) for name in channels}
              for label in prepared}
    return Report(loss=losses, scales=scales, training=errors["training"],
                  validation=errors.get("validation"))


__all__ = ("Dataset", "Report", "batches", "fit")
