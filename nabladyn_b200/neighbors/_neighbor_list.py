"""The neighbor list: pairs of atoms closer than cutoff + skin, kept on the GPU.

The public contract is the reference's ``NeighborList`` (src/nabladyn/neighbors/
_neighbor_list.py:162-405): the constructor and its checks, ``allocate`` / ``update`` /
``tensors`` / ``pair_capacity`` / ``num_pairs``, the capacity rule max(8, ceil(m * count)), the
grid rule, inner lists, and the exceptions with their messages. The device work runs through
``torch.ops.nabladyn_neighbors`` (the reference's four schemas, registered over this package's
kernels in libnabladyn_b200.so), so the same buffers in the same order cross that boundary.

How this class keeps them is its own: one ``_DeviceList`` owns every tensor of a list (the 15
schema buffers and the update's 6), built from a size plan; the pair count of a first frame is
read as one (offset, count) pair of the last atom instead of a sum over all atoms; the status
word is decoded by one function shared with the MD engines.
"""

from __future__ import annotations

import math
from numbers import Real

import torch
from torch import Tensor

from .. import space
from .._native import INVALID_CELL, NON_FINITE, OVERFLOW, neighbor_ops
from ._pairs import NeighborPairs

_INT32_MAX = 2**31 - 1

# The schema's buffer order (src/nabladyn/neighbors/csrc/ops.cpp:13-18), then the update's.
_BUILD_ORDER = ("dims", "widths", "atom_bin", "bin_counts", "bin_offsets", "unordered_ids",
                "sorted_ids", "sorted_positions", "scan_temp", "pair_counts", "pair_offsets",
                "pair_total", "status", "pairs", "bits")
_UPDATE_ORDER = ("reference_positions", "reference_cell", "limits", "reuse", "rebuild",
                 "rebuild_count")


def grid(lengths: list[float], radius: float, dtype: torch.dtype) -> list[int]:
    """Bins per axis: floor(L / (R + 4 eps L)), at least one, in float64 arithmetic.

    Each bin is wider than the list radius by a few roundings of L, so binning in the list's
    dtype never puts two atoms closer than R more than one bin apart (the rule of
    src/nabladyn/neighbors/_neighbor_list.py:115-122).
    """
    eps = torch.finfo(dtype).eps
    return [max(1, math.floor(length / (radius + 4 * eps * length))) for length in lengths]


def check_cell_lengths(lengths: list[float], cutoff: float) -> None:
    """Raise ``ValueError`` unless every cell length is finite and above twice the cutoff."""
    if not all(math.isfinite(length) and length > 2 * cutoff for length in lengths):
        raise ValueError("every cell length must be finite and above twice the cutoff")


def status_causes(flags: int, needed: int, capacity: int, radius: float) -> list[str]:
    """The messages of a list's status word [flags, pairs needed], in the reference's words."""
    causes = []
    if flags & INVALID_CELL:
        causes.append("every cell length must be finite and above twice the cutoff")
    if flags & NON_FINITE:
        causes.append("positions must be finite")
    if flags & OVERFLOW:
        causes.append(
            f"the pair capacity {capacity} is too small: the frame has {needed} pairs within "
            f"{radius} nm; raise capacity_multiplier",
        )
    return causes


def _is_number(value) -> bool:
    return isinstance(value, Real) and not isinstance(value, bool) and math.isfinite(value)


def _validate_settings(cutoff, skin, capacity_multiplier, inner_cutoffs) -> None:
    if not all(_is_number(v) for v in (cutoff, skin, capacity_multiplier)):
        bad = next(name for name, v in (("cutoff", cutoff), ("skin", skin),
                                        ("capacity_multiplier", capacity_multiplier))
                   if not _is_number(v))
        raise ValueError(f"{bad} must be a finite number")
    if not (cutoff > 0 and skin >= 0 and capacity_multiplier >= 1):
        raise ValueError(
            "cutoff must be positive, skin nonnegative and capacity_multiplier at least 1",
        )
    if not isinstance(inner_cutoffs, (tuple, list)):
        raise ValueError("inner_cutoffs must be a tuple of cutoffs in nm")
    if not all(_is_number(v) and 0 < v < cutoff for v in inner_cutoffs):
        raise ValueError("every inner cutoff must be a number between 0 and the cutoff")
    if len(set(inner_cutoffs)) != len(inner_cutoffs):
        raise ValueError("the inner cutoffs must be distinct")


def _validate_frame(positions: Tensor, cell: Tensor) -> None:
    if not (isinstance(positions, Tensor) and positions.layout is torch.strided):
        raise TypeError("positions must be a dense tensor")
    if not (isinstance(cell, Tensor) and cell.layout is torch.strided):
        raise TypeError("cell must be a dense tensor")
    if positions.ndim != 2 or positions.shape[1] != 3 or not 1 <= positions.shape[0] <= _INT32_MAX:
        raise ValueError("positions must have shape [N, 3] with 1 <= N < 2**31")
    if positions.dtype not in (torch.float32, torch.float64) or not positions.is_cuda:
        raise TypeError("positions must be a CUDA float32 or float64 tensor")
    if cell.shape != (3,) or cell.dtype != positions.dtype or cell.device != positions.device:
        raise ValueError("cell must be a [3] tensor with the positions' dtype and device")


class _DeviceList:
    """Every device tensor of one list, created from its size plan.

    ``build_args()`` and ``update_args()`` give them in the schemas' orders. The pairs start as
    [2, 1] and are replaced once the first frame is counted; all-pairs lists (a first grid of
    at most three bins per axis) carry an N x ceil(N / 32) word matrix, others an empty one.
    """

    def __init__(self, num_atoms: int, dims: list[int], lengths: list[float], scan_bytes: int,
                 dtype: torch.dtype, device: torch.device):
        ints = {"dtype": torch.int32, "device": device}
        bins = math.prod(dims)
        words = num_atoms * ((num_atoms + 31) // 32) if max(dims) <= 3 else 0
        self.tensors: dict[str, Tensor] = {
            "dims": torch.tensor(dims, **ints),
            "widths": torch.tensor([length / count for length, count in zip(lengths, dims)],
                                   dtype=dtype, device=device),
            "atom_bin": torch.empty(num_atoms, **ints),
            "bin_counts": torch.zeros(bins + 1, **ints),
            "bin_offsets": torch.empty(bins + 1, **ints),
            "unordered_ids": torch.empty(num_atoms, **ints),
            "sorted_ids": torch.empty(num_atoms, **ints),
            "sorted_positions": torch.empty((num_atoms, 3), dtype=dtype, device=device),
            "scan_temp": torch.empty(scan_bytes, dtype=torch.uint8, device=device),
            "pair_counts": torch.empty(num_atoms, **ints),
            "pair_offsets": torch.empty(num_atoms, **ints),
            "pair_total": torch.zeros(1, **ints),
            "status": torch.zeros(2, **ints),
            "pairs": torch.empty((2, 1), **ints),
            "bits": torch.zeros(words, **ints),
            "limits": torch.tensor(dims, **ints),
            "reuse": torch.zeros(4, dtype=dtype, device=device),
            "rebuild": torch.zeros(1, **ints),
            "rebuild_count": torch.ones(1, **ints),
        }

    def __getitem__(self, name: str) -> Tensor:
        return self.tensors[name]

    def build_args(self) -> tuple[Tensor, ...]:
        return tuple(self.tensors[name] for name in _BUILD_ORDER)

    def update_args(self) -> tuple[Tensor, ...]:
        return tuple(self.tensors[name] for name in _UPDATE_ORDER)


class NeighborList:
    """Pairs of atoms closer than the list radius, cutoff + skin, in nm.

    ``allocate`` sizes the list to ``capacity_multiplier`` times a first frame's pair count and
    builds it; ``update`` reuses the pairs until an atom has moved far enough that a pair
    within the cutoff could be missing, then rebuilds; ``tensors()`` returns the pairs. Cells
    are orthorhombic and periodic; positions may lie outside the cell. ``inner_cutoffs`` keeps
    an inner list per smaller cutoff, with the same skin and capacity rule, handed to a sum of
    models in ``NeighborPairs.inner``.

    Raises ``ValueError`` unless ``cutoff`` is positive, ``skin`` nonnegative and
    ``capacity_multiplier`` at least 1, all finite, and the inner cutoffs distinct numbers
    between 0 and ``cutoff``.
    """

    def __init__(self, cutoff: Real, *, skin: Real = 0.0, capacity_multiplier: Real = 1.25,
                 inner_cutoffs: tuple[Real, ...] = ()):
        _validate_settings(cutoff, skin, capacity_multiplier, inner_cutoffs)
        self._cutoff, self._skin = float(cutoff), float(skin)
        self._capacity_multiplier = float(capacity_multiplier)
        self._inner = tuple(NeighborList(value, skin=skin, capacity_multiplier=capacity_multiplier)
                            for value in sorted(inner_cutoffs))
        self._device: _DeviceList | None = None
        self._failure: str | None = None

    @property
    def cutoff(self) -> float:
        """The cutoff in nm."""
        return self._cutoff

    @property
    def radius(self) -> float:
        """The list radius, cutoff + skin, in nm."""
        return self._cutoff + self._skin

    # -- building ----------------------------------------------------------------------

    def allocate(self, positions: Tensor, cell: Tensor) -> None:
        """Count the pairs of positions [N, 3] in the cell [3], size the list and build it.

        Syncs with the host. Raises ``TypeError`` or ``ValueError`` for invalid positions or
        cell, and ``ValueError`` when the grid or the pairs do not fit int32.
        """
        _validate_frame(positions, cell)
        lengths = [float(length) for length in cell.tolist()]
        check_cell_lengths(lengths, self._cutoff)
        if not bool(torch.isfinite(positions).all()):
            raise ValueError("positions must be finite")
        dims = grid(lengths, self.radius, positions.dtype)
        if math.prod(dims) >= _INT32_MAX:
            raise ValueError("the grid must have fewer than 2**31 - 1 bins")
        ops = neighbor_ops()
        n = positions.shape[0]
        scan_bytes = max(ops.scan_temp_bytes(positions, math.prod(dims) + 1),
                         ops.scan_temp_bytes(positions, n))
        device = _DeviceList(n, dims, lengths, scan_bytes, positions.dtype, positions.device)
        frame, _ = space.wrap(positions.detach(), cell.detach())
        box = cell.detach().contiguous()
        ops.count_first_frame(frame, box, self.radius, *device.build_args())
        # The pairs of the frame: the last atom's offset plus its count.
        offset, last = torch.stack([device["pair_offsets"][-1], device["pair_counts"][-1]]).tolist()
        count = offset + last
        capacity = max(8, math.ceil(self._capacity_multiplier * count))
        if capacity > _INT32_MAX:
            raise ValueError(
                f"the pair capacity {capacity}, capacity_multiplier times {count} pairs, "
                "exceeds the int32 range",
            )
        device.tensors["pairs"] = torch.empty((2, capacity), dtype=torch.int32,
                                              device=positions.device)
        ops.fill_first_frame(frame, box, self.radius, *device.build_args())
        device.tensors["reference_positions"] = frame.clone()
        device.tensors["reference_cell"] = box.clone()
        self._device = device
        # The list stays failed until its inner lists are built from the same frame.
        self._failure = "an inner list was not allocated"
        for inner in self._inner:
            inner.allocate(positions, cell)
        self._failure = None

    def update(self, positions: Tensor, cell: Tensor) -> None:
        """Reuse the pairs for positions [N, 3] in the cell [3], or rebuild them.

        The pairs are reused while no atom has moved more than (R s_min - r_c) / 2 from its
        position at the last rebuild, scaled with the cell. Syncs with the host. Raises
        ``TypeError``/``ValueError`` for positions or a cell of the wrong kind; ``ValueError``,
        failing the list until ``allocate``, for a bad cell length, a non-finite coordinate or
        too many pairs; ``RuntimeError`` before ``allocate`` or after a failure.
        """
        device = self._live()
        _validate_frame(positions, cell)
        like = device["sorted_positions"]
        if (positions.shape, positions.dtype, positions.device) != (like.shape, like.dtype,
                                                                    like.device):
            raise ValueError("positions must match the allocated shape, dtype and device")
        frame, _ = space.wrap(positions.detach(), cell.detach())
        self._update_wrapped(frame, cell.detach().contiguous())
        self._check_status()

    def _update_wrapped(self, positions: Tensor, cell: Tensor) -> None:
        """The device update of positions already in [0, L): no checks, no host sync, so it can
        be captured in a CUDA graph (the MD step calls it)."""
        device = self._device
        neighbor_ops().update(positions, cell, self._cutoff, self.radius, *device.update_args(),
                              *device.build_args())
        for inner in self._inner:
            inner._update_wrapped(positions, cell)

    def _rebuild_wrapped(self, positions: Tensor, cell: Tensor) -> None:
        """A device update that always rebuilds: an infinite reference cell makes every scale
        zero, so the reuse allowance is negative."""
        for listed in (self, *self._inner):
            listed._device["reference_cell"].fill_(math.inf)
        self._update_wrapped(positions, cell)

    # -- status --------------------------------------------------------------------------

    def _check_status(self) -> None:
        """Raise ``ValueError`` and fail the list if an update of it or an inner list failed."""
        flags, needed = self._live()["status"].tolist()
        causes = status_causes(flags, needed, self.pair_capacity, self.radius)
        if causes:
            self._failure = "; ".join(causes)
            raise ValueError(self._failure)
        for inner in self._inner:
            try:
                inner._check_status()
            except ValueError as error:
                self._failure = str(error)
                raise

    def _live(self) -> _DeviceList:
        if self._device is None:
            raise RuntimeError("call allocate() first")
        if self._failure is not None:
            raise RuntimeError(
                f"the neighbor list failed ({self._failure}); call allocate() again",
            )
        return self._device

    def _device_tensors(self) -> dict[str, Tensor]:
        """Every device tensor of the list, by name, for an engine's snapshot and restore."""
        return dict(self._device.tensors)

    # -- results -------------------------------------------------------------------------

    def tensors(self) -> NeighborPairs:
        """The pairs of the last build, with the inner lists' in ``inner``, ascending."""
        device = self._live()
        return NeighborPairs(device["pairs"], device["sorted_ids"].numel(), self._cutoff,
                             tuple(inner.tensors() for inner in self._inner))

    @property
    def pair_capacity(self) -> int:
        """C, the columns of the list's own pair index; 0 before ``allocate``."""
        return 0 if self._device is None else self._device["pairs"].shape[1]

    @property
    def num_pairs(self) -> int:
        """The number of the list's own pairs at the last build. Syncs with the host."""
        return int(self._live()["pair_total"].item())

    @property
    def _rebuild_count(self) -> int:
        """The builds since allocate, counting allocate's own. Syncs with the host."""
        return int(self._device["rebuild_count"].item())


__all__ = ("NeighborList", "check_cell_lengths", "grid", "status_causes")
