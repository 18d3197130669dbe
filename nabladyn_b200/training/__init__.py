"""Fitting Lennard-Jones parameters to labeled frames: batched predictions, the scaled loss and
its hand-written parameter backward."""

from ._loss import CHANNELS, loss, scales
from ._predict import predict
from ._stacks import pair_stack, width

__all__ = ("CHANNELS", "loss", "scales", "predict", "pair_stack", "width")
