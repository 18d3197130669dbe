"""Molecular dynamics on the GPU: each step is a few engine kernels replayed from CUDA Graphs."""

from ._output import read_sample_file
from ._simulation import FIELDS, Simulation, npt, nve, nvt
from ._state import BarostatState, ChainState, State
from ._velocities import maxwell_boltzmann

__all__ = (
    "nve",
    "nvt",
    "npt",
    "maxwell_boltzmann",
    "Simulation",
    "FIELDS",
    "State",
    "ChainState",
    "BarostatState",
    "read_sample_file",
)
