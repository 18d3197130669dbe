"""Fitting model parameters to labeled frames: batched predictions, the scaled loss, and
parameter gradients (hand-written kernels for Lennard-Jones; the reference's torch.func
algorithm, in frame chunks, for other models such as SchNet)."""

from ._fit import Dataset, Report, batches, fit
from ._generic import loss_and_gradient
from ._loss import CHANNELS, loss, scales
from ._predict import predict
from ._stacks import pair_stack, width

__all__ = ("CHANNELS", "Dataset", "Report", "batches", "fit", "loss", "scales", "predict",
           "loss_and_gradient", "pair_stack", "width")
