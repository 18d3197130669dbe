"""ORACLE (test infrastructure): ctypes wrapper of neighbors.c, the CPU restatement of the
reference's neighbor operator, plus the host rules of src/nabladyn/neighbors/_neighbor_list.py
(_grid :115-122, the all-pairs choice :131-140, the capacity :259)."""

from __future__ import annotations

import ctypes
import math

import numpy as np

from .build import LIB, build

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = ctypes.CDLL(str(LIB))
        for suffix in ("f32", "f64"):
            grid = getattr(_lib, f"oracle_grid_pairs_{suffix}")
            grid.restype = ctypes.c_int64
            grid.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_int64, ctypes.c_void_p]
            every = getattr(_lib, f"oracle_all_pairs_{suffix}")
            every.restype = ctypes.c_int64
            every.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
            reuse = getattr(_lib, f"oracle_reuse_{suffix}")
            reuse.restype = ctypes.c_int
            reuse.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int64, ctypes.c_double,
                                                      ctypes.c_double] + [ctypes.c_void_p] * 3
    return _lib


def _suffix(dtype) -> str:
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def grid_dims(lengths, radius: float, dtype) -> list[int]:
    """Bins per axis: max(1, floor(L / (R + 4 eps L))), in float64 (the allocate rule)."""
    eps = float(np.finfo(dtype).eps)
    return [max(1, math.floor(float(length) / (radius + 4 * eps * float(length))))
            for length in lengths]


def wrap(positions: np.ndarray, cell: np.ndarray) -> np.ndarray:
    """src/nabladyn/space.py:22-38 in the array's dtype."""
    crossings = np.floor(positions / cell)
    wrapped = positions - crossings * cell
    wrapped = np.where(wrapped < 0, wrapped + cell, wrapped)
    wrapped = np.where(wrapped >= cell, wrapped - cell, wrapped)
    return wrapped.astype(positions.dtype)


def pairs(positions: np.ndarray, cell: np.ndarray, radius: float, dims=None):
    """The reference's pair list of wrapped positions: (first, second, path), in its order.

    ``dims`` defaults to the allocate rule; the all-pairs path runs when every axis has at
    most three bins.
    """
    lib = _load()
    positions = np.ascontiguousarray(positions)
    dtype = positions.dtype
    cell = np.ascontiguousarray(cell, dtype=dtype)
    n = positions.shape[0]
    if dims is None:
        dims = grid_dims(cell, radius, dtype)
    suffix = _suffix(dtype)
    if max(dims) <= 3:
        function, path = getattr(lib, f"oracle_all_pairs_{suffix}"), "all"
        count = function(positions.ctypes.data, cell.ctypes.data, n, radius, None, None, 0)
        first = np.empty(max(count, 1), dtype=np.int32)
        second = np.empty(max(count, 1), dtype=np.int32)
        function(positions.ctypes.data, cell.ctypes.data, n, radius, first.ctypes.data,
                 second.ctypes.data, count)
        return first[:count], second[:count], path
    dims_array = np.asarray(dims, dtype=np.int32)
    widths = np.asarray([float(cell[a]) / dims[a] for a in range(3)], dtype=dtype)
    function = getattr(lib, f"oracle_grid_pairs_{suffix}")
    count = function(positions.ctypes.data, cell.ctypes.data, n, dims_array.ctypes.data,
                     widths.ctypes.data, radius, None, None, 0, None)
    first = np.empty(max(count, 1), dtype=np.int32)
    second = np.empty(max(count, 1), dtype=np.int32)
    function(positions.ctypes.data, cell.ctypes.data, n, dims_array.ctypes.data,
             widths.ctypes.data, radius, first.ctypes.data, second.ctypes.data, count, None)
    return first[:count], second[:count], "grid"


def pair_set(first: np.ndarray, second: np.ndarray) -> np.ndarray:
    """Pairs as sorted unique int64 keys min * 2^32 + max, for set comparison."""
    low = np.minimum(first, second).astype(np.int64)
    high = np.maximum(first, second).astype(np.int64)
    return np.sort(low * (1 << 32) + high)


def capacity(count: int, multiplier: float = 1.25) -> int:
    """max(8, ceil(multiplier * count)), src/nabladyn/neighbors/_neighbor_list.py:259."""
    return max(8, math.ceil(multiplier * count))


def reuse(positions, reference_positions, cell, reference_cell, cutoff, radius, limits):
    """The update's decision: 1 rebuild, 0 reuse, -1 bad cell, -2 non-finite; and dims."""
    lib = _load()
    dtype = positions.dtype
    arrays = [np.ascontiguousarray(a, dtype=dtype)
              for a in (positions, reference_positions, cell, reference_cell)]
    limits = np.ascontiguousarray(limits, dtype=np.int32)
    dims = np.zeros(3, dtype=np.int32)
    widths = np.zeros(3, dtype=dtype)
    decision = getattr(lib, f"oracle_reuse_{_suffix(dtype)}")(
        *(a.ctypes.data for a in arrays), arrays[0].shape[0], cutoff, radius,
        limits.ctypes.data, dims.ctypes.data, widths.ctypes.data)
    return decision, dims
