"""The supervised loss: scaled errors of predicted energies, forces and virials.

The same scales and loss as src/nabladyn/training/_loss.py:26-46 and :105-125.
"""

from collections.abc import Mapping

import torch
from torch import Tensor

CHANNELS = ("energy", "forces", "virial")


def scales(energy: Tensor | None = None, forces: Tensor | None = None,
           virial: Tensor | None = None) -> dict[str, float]:
    """Each given channel's scale from its labels: energy [F] and virial [F, 3, 3] by the RMS
    about the mean over frames, forces [F, N, 3] by the plain RMS; constant labels fall back to
    the plain RMS and all-zero labels to 1. Syncs with the host."""
    result = {}
    for name, labels, about_mean in (("energy", energy, True), ("forces", forces, False),
                                     ("virial", virial, True)):
        if labels is not None:
            rms = float(labels.square().mean().sqrt())
            spread = rms
            if about_mean:
                spread = float((labels - labels.mean(dim=0)).square().mean().sqrt())
            result[name] = spread or rms or 1.0
    return result


def loss(predicted: Mapping[str, Tensor], labels: Mapping[str, Tensor],
         weights: Mapping[str, float | Tensor], scales: Mapping[str, float | Tensor],
         coefficients: Tensor | None = None) -> tuple[Tensor, dict[str, Tensor]]:
    """The batch loss, the weighted sum of its channel terms, and the terms by name.

    A channel's term is each frame's mean of ((X - X*) / s_X)^2 over its components, times the
    frame's coefficient [B] (1/B when ``coefficients`` is None), summed over the frames.
    """
    terms = {}
    for name, value in predicted.items():
        squares = ((value - labels[name]) / scales[name]).square()
        per_frame = squares.reshape(squares.shape[0], -1).mean(dim=1)
        terms[name] = per_frame.mean() if coefficients is None else (coefficients * per_frame).sum()
    return sum(weights[name] * term for name, term in terms.items()), terms


__all__ = ("CHANNELS", "scales", "loss")
