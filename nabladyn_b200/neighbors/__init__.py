"""The CUDA neighbor list."""

from ._neighbor_list import NeighborList
from ._pairs import NeighborPairs

__all__ = ("NeighborList", "NeighborPairs")
