"""The state of a simulation: one frame, detached from the simulation that made it.

The same records as src/nabladyn/md/_state.py:23-57, so a state from either build resumes in
the other.
"""

from typing import NamedTuple

from torch import Tensor


class ChainState(NamedTuple):
    """A Nose-Hoover chain: positions [3], dimensionless, and momenta [3] in kJ ps/mol."""

    positions: Tensor
    momenta: Tensor


class BarostatState(NamedTuple):
    """An isotropic barostat: the box momentum [] float64 and its chain."""

    momentum: Tensor
    chain: ChainState


class State(NamedTuple):
    """A copy of a simulation's frame, in nm, nm/ps and kJ/mol/nm.

    ``positions`` [N, 3] lie in [0, L); ``images`` [N, 3] int64 count lattice crossings, so
    the unwrapped positions are ``positions + images * cell``. ``forces`` act at
    ``positions``; ``step`` counts steps since the first frame; ``thermostat`` is the chain of
    an NVT run.
    """

    positions: Tensor
    velocities: Tensor
    forces: Tensor
    cell: Tensor
    images: Tensor
    step: int
    thermostat: ChainState | None = None
    barostat: BarostatState | None = None


__all__ = ("BarostatState", "ChainState", "State")
