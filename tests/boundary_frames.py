"""Frames whose pair sets are decided by the rounding of r^2 = dx^2 + dy^2 + dz^2.

Each designed pair's exact squared distance (from its stored coordinates) lies within about
half an ulp of the squared list radius, so whether it is listed depends on the order of the
roundings in the sum. The reference's kernels write ``dx * dx + dy * dy + dz * dz``
(src/nabladyn/neighbors/csrc/common/traversal.cuh:103,140, pairs/all_pairs.cuh:61), which nvcc
contracts into fused multiply-adds; these frames let a test tell the possible contractions
apart by their pair sets. Used by tests/test_reference_op_gpu.py and
tests/test_neighbors_gpu.py.
"""

from __future__ import annotations

from fractions import Fraction

import numpy as np

# The candidate roundings of dx*dx + dy*dy + dz*dz: fma(a, b, c) rounds a*b + c once.
ORDERS = {
    "fma(dz,dz,fma(dx,dx,dy*dy))": lambda dx, dy, dz, r: r(dz * dz + r(dx * dx + r(dy * dy))),
    "fma(dz,dz,fma(dy,dy,dx*dx))": lambda dx, dy, dz, r: r(dz * dz + r(dy * dy + r(dx * dx))),
    "(dx*dx+dy*dy)+dz*dz": lambda dx, dy, dz, r: r(r(r(dx * dx) + r(dy * dy)) + r(dz * dz)),
}
PINNED = "fma(dz,dz,fma(dx,dx,dy*dy))"


def _rounder(dtype):
    if np.dtype(dtype) == np.float64:
        return lambda value: Fraction(float(value))
    return lambda value: Fraction(float(np.float32(float(value))))


def designed_frame(length: float, pairs: int, radius: float, dtype, seed: int):
    """Positions [2 * pairs, 3] of ``dtype`` in a cubic box of ``length``: pairs at the list
    radius whose exact r^2 is within 0.6 ulp of the radius^2 the kernels compare against,
    away from the faces (one image), plus the (first, second) indices of the designed pairs."""
    dtype = np.dtype(dtype)
    rng = np.random.default_rng(seed)
    r = dtype.type(radius)
    r2 = Fraction(float(r * r))  # the threshold as the kernels hold it: radius^2 rounded
    ulp = Fraction(float(np.spacing(r * r)))
    kept_a, kept_b = [], []
    while len(kept_a) < pairs:
        centers = rng.uniform(radius + 0.05, length - radius - 0.05, (20000, 3)).astype(dtype)
        directions = rng.normal(size=(20000, 3))
        directions /= np.linalg.norm(directions, axis=1, keepdims=True)
        partners = (centers.astype(np.float64) + directions * float(r)).astype(dtype)
        d = centers.astype(np.longdouble) - partners.astype(np.longdouble)
        close = np.abs((d * d).sum(axis=1) - np.longdouble(float(r2))) < 2 * float(ulp)
        for a, b in zip(centers[close], partners[close]):
            exact = sum((Fraction(float(p)) - Fraction(float(q))) ** 2 for p, q in zip(a, b))
            if abs(exact - r2) <= ulp * Fraction(6, 10):
                kept_a.append(a)
                kept_b.append(b)
    a, b = np.array(kept_a[:pairs]), np.array(kept_b[:pairs])
    positions = np.concatenate([a, b]).astype(dtype)
    first = np.arange(pairs, dtype=np.int64)
    return positions, np.full(3, length, dtype=dtype), first, first + pairs


def listed_under(order: str, positions, first, second, radius: float) -> np.ndarray:
    """Which designed pairs ``order`` lists: r^2 < radius^2 with r^2 rounded that way."""
    dtype = positions.dtype
    rnd = _rounder(dtype)
    r = dtype.type(radius)
    r2 = Fraction(float(r * r))
    out = np.zeros(len(first), dtype=bool)
    for k, (i, j) in enumerate(zip(first, second)):
        # Sign and image do not matter: the pairs sit one image apart and d is exact.
        dx, dy, dz = (rnd(Fraction(float(p)) - Fraction(float(q)))
                      for p, q in zip(positions[i], positions[j]))
        out[k] = ORDERS[order](dx, dy, dz, rnd) < r2
    return out


def designed_listed(pair_keys: np.ndarray, first, second) -> np.ndarray:
    """Which designed pairs a set of pair keys (oracle.neighbors.pair_set) holds."""
    wanted = np.minimum(first, second) * (1 << 32) + np.maximum(first, second)
    return np.isin(wanted, pair_keys)


def matching_orders(listed: np.ndarray, positions, first, second, radius: float) -> list[str]:
    """The candidate orders whose decisions equal ``listed`` on the designed pairs."""
    return [name for name in ORDERS
            if np.array_equal(listed_under(name, positions, first, second, radius), listed)]
