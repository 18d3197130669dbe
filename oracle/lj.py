"""ORACLE (test infrastructure): Lennard-Jones E/F/W and parameter gradients in float64 numpy.

Restates src/nabladyn/potential/_lennard_jones/_potential.py:209-234 (shifted 12-6 per
type-pair row, pairs with r^2 < r_c^2 and i != j) and src/nabladyn/quantity.py:160-184
(F = -dE/dx, W = -dE/dstrain at zero strain) with the derivatives written out.
"""

from __future__ import annotations

import numpy as np


def displacement(left: np.ndarray, right: np.ndarray, cell: np.ndarray) -> np.ndarray:
    """Minimum-image left - right for wrapped coordinates (src/nabladyn/space.py:11-19)."""
    raw = left - right
    half = 0.5 * cell
    return (left - np.where(raw > half, cell, 0.0)) - (right - np.where(raw < -half, cell, 0.0))


def pair_rows(types_a: np.ndarray, types_b: np.ndarray, num_types: int) -> np.ndarray:
    low, high = np.minimum(types_a, types_b), np.maximum(types_a, types_b)
    return low * (2 * num_types - low - 1) // 2 + high


def all_pairs(n: int) -> tuple[np.ndarray, np.ndarray]:
    i, j = np.triu_indices(n, k=1)
    return i.astype(np.int64), j.astype(np.int64)


def energy_force_virial(positions, cell, first, second, sigma, epsilon, cutoff, atom_types=None,
                        parameter_grads=False):
    """E, F [N, 3], W [3, 3] (and dE/dsigma, dE/depsilon per row) in float64.

    ``first``/``second`` list each pair once; self-pairs and pairs beyond the cutoff drop out.
    """
    x = np.asarray(positions, dtype=np.float64)
    cell = np.asarray(cell, dtype=np.float64)
    sigma = np.asarray(sigma, dtype=np.float64)
    epsilon = np.asarray(epsilon, dtype=np.float64)
    first = np.asarray(first, dtype=np.int64)
    second = np.asarray(second, dtype=np.int64)
    keep = first != second
    first, second = first[keep], second[keep]
    d = displacement(x[first], x[second], cell)
    r2 = (d * d).sum(axis=1)
    valid = r2 < cutoff * cutoff
    first, second, d, r2 = first[valid], second[valid], d[valid], r2[valid]
    num_types = int(round((np.sqrt(8 * sigma.size + 1) - 1) / 2))
    if num_types == 1 or atom_types is None:
        rows = np.zeros(first.shape, dtype=np.int64)
    else:
        types = np.asarray(atom_types, dtype=np.int64)
        rows = pair_rows(types[first], types[second], num_types)
    s, e = sigma[rows], epsilon[rows]
    p6 = (s * s / r2) ** 3
    pc6 = (s * s / (cutoff * cutoff)) ** 3
    energy = float((4 * e * (p6 * p6 - p6) - 4 * e * (pc6 * pc6 - pc6)).sum())
    fs = 24 * e * (2 * p6 * p6 - p6) / r2
    fvec = fs[:, None] * d
    forces = np.zeros_like(x)
    np.add.at(forces, first, fvec)
    np.add.at(forces, second, -fvec)
    virial = (fs[:, None, None] * d[:, :, None] * d[:, None, :]).sum(axis=0)
    if not parameter_grads:
        return energy, forces, virial
    dsigma = np.zeros_like(sigma)
    depsilon = np.zeros_like(epsilon)
    np.add.at(dsigma, rows, 24 * e / s * (2 * p6 * p6 - p6 - 2 * pc6 * pc6 + pc6))
    np.add.at(depsilon, rows, 4 * (p6 * p6 - p6) - 4 * (pc6 * pc6 - pc6))
    return energy, forces, virial, dsigma, depsilon


def sample_forces(positions, cell, centers, sigma, epsilon, cutoff):
    """float64 forces on the atoms ``centers`` only, each with its complete neighbor set.

    For boxes too large for an all-atom evaluation here: positions [N, 3] anywhere (wrapped in
    float64 first), neighbors within the cutoff found by a periodic k-d tree, each unordered
    pair listed once, then ``energy_force_virial`` over those pairs (one atom type).
    """
    from scipy.spatial import cKDTree

    cell = np.asarray(cell, dtype=np.float64)
    x = np.asarray(positions, dtype=np.float64)
    x = x - np.floor(x / cell) * cell
    x = np.where(x >= cell, x - cell, x)
    centers = np.asarray(centers, dtype=np.int64)
    tree = cKDTree(x, boxsize=cell)
    found = tree.query_ball_point(x[centers], cutoff)
    sampled = np.zeros(len(x), dtype=bool)
    sampled[centers] = True
    first, second = [], []
    for center, neighbors in zip(centers, found):
        neighbors = np.asarray(neighbors, dtype=np.int64)
        # A pair of two sampled atoms is listed from its lower index only.
        keep = (neighbors != center) & ~(sampled[neighbors] & (neighbors < center))
        second.append(neighbors[keep])
        first.append(np.full(int(keep.sum()), center, dtype=np.int64))
    first, second = np.concatenate(first), np.concatenate(second)
    _, forces, _ = energy_force_virial(x, cell, first, second, sigma, epsilon, cutoff)
    return forces[centers]
