"""Potentials: models whose one scalar energy defines forces and virial."""

from ._base import Potential
from ._lennard_jones import LennardJones, lennard_jones, pair_index
from ._schnet import SchNet, schnet
from ._sum import Sum, sum

__all__ = ("Potential", "LennardJones", "lennard_jones", "pair_index", "SchNet", "schnet",
           "Sum", "sum")
