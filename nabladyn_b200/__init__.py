"""nabladyn_b200: the MD step hot path of NablaDyn, B200-native.

The cell-list neighbor operator (binning, pair build and the on-GPU skin-reuse check),
Lennard-Jones energy/force/virial and the velocity-Verlet / Nose-Hoover update, as hand-written
sm_100a CUDA behind the C-ABI of include/nabladyn_b200.h, with the reference's Python interface
on top: ``neighbors.NeighborList``, ``quantity.energy_force_virial``, ``potential.lennard_jones``
and ``md.nve`` / ``md.nvt``.
"""

from . import md, neighbors, observables, potential, quantity, space, training, units

__version__ = "0.1.0"

__all__ = ("md", "neighbors", "observables", "potential", "quantity", "space", "training", "units")
