"""Seeded synthetic systems: jittered lattices in cubic boxes, for the benchmark and the tests.

The inputs of the benchmark workloads: argon-like fluids started from a simple-cubic or
face-centered cubic lattice with Gaussian jitter, all seeded.
"""

from __future__ import annotations

import math

import numpy as np


def simple_cubic(n_side: int, length: float, jitter: float, seed: int, count: int | None = None):
    """The first ``count`` sites of an n^3 simple-cubic lattice in a cubic box, jittered."""
    a = length / n_side
    grid = np.stack(np.meshgrid(*(np.arange(n_side),) * 3, indexing="ij"), axis=-1).reshape(-1, 3)
    sites = (grid + 0.5) * a
    if count is not None:
        sites = sites[:count]
    rng = np.random.default_rng(seed)
    positions = sites + rng.normal(0.0, jitter, sites.shape)
    return positions, np.full(3, length)


def fcc(cells_per_side: int, length: float, jitter: float, seed: int):
    """A face-centered cubic lattice of 4 n^3 sites, jittered by a Gaussian of ``jitter`` nm."""
    a = length / cells_per_side
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    grid = np.stack(np.meshgrid(*(np.arange(cells_per_side),) * 3, indexing="ij"), axis=-1)
    sites = (grid.reshape(-1, 1, 3) + base[None] + 0.25).reshape(-1, 3) * a
    rng = np.random.default_rng(seed)
    positions = sites + rng.normal(0.0, jitter, sites.shape)
    return positions, np.full(3, length)


def argon_box(num_atoms: int, density: float = 21.09):
    """The cubic box length of ``num_atoms`` at ``density`` per nm^3."""
    return (num_atoms / density) ** (1.0 / 3.0)


def random_box(num_atoms: int, lengths, seed: int):
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, dtype=np.float64)
    return rng.uniform(0.0, 1.0, (num_atoms, 3)) * lengths, lengths


def large_lj(jitter: float = 0.02, seed: int = 2024):
    """1,048,576 atoms: a 64^3-cell FCC lattice in L = 36.77 nm (rho = 21.1 per nm^3)."""
    return fcc(64, 36.77, jitter, seed)


__all__ = ("simple_cubic", "fcc", "argon_box", "random_box", "large_lj")
