"""Potentials: models whose one scalar energy defines forces and virial."""

from ._base import Potential
from ._lennard_jones import LennardJones, lennard_jones, pair_index

__all__ = ("Potential", "LennardJones", "lennard_jones", "pair_index")
