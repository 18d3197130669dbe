"""The device state of one simulation and the calls into the MD engine of libnabladyn_b200.so.

``Engine`` sizes and owns every buffer of ``nd_md_system`` (include/nabladyn_b200.h) as torch
tensors on the model's device, loads a frame, and launches rebuilds, force evaluations and
steps on torch's current stream, so a step can be captured in a CUDA Graph.

Sizing follows the reference's capacity rule (src/nabladyn/neighbors/_neighbor_list.py:
256-261) with its own units: a first build with the smallest list counts the longest list (on
the brick path the longest whole list of a pair of centers, which either half of a pair's list
can approach once the pair's centers drift apart) and the largest brick tile; the list then
gets ``capacity_multiplier`` times each.
A later frame that needs more sets the overflow bit, and the run fails at its next status read,
as the reference's does.
"""

from __future__ import annotations

import math

import torch
from torch import Tensor

from .. import _native
from .._native import MDSystem, OVERFLOW, call, dtype_code, ptr, stream_handle
from ..neighbors._neighbor_list import check_cell_lengths, grid
from ..units import BOLTZMANN

_THREADS = 256           # kMDThreads in md.cu
_MAX_BRICK_CELLS = 14    # kMaxBrickCells in md.cu
_TILE_BYTES = 200 * 1024  # the dynamic shared memory a tile may take
_CENTERS_PER_BRICK = 224  # the brick size aimed at: about 7 warps of centers
# Offsets into the float64 thermostat block (enum Thermo in md.cu).
CHAIN_A, KINETIC_A, CHAIN_B, KINETIC_B, PENDING_SCALE = 0, 6, 7, 13, 14
CHAIN_MASS, THERMAL_ENERGY, DEGREES, TIMESTEP = 16, 19, 20, 21
STAGE_TIMEOUT = 16  # status bit: a tile copy did not complete (kStageTimeout in md.cu)


class StepGraph:
    """An instantiated step graph of the engine (``nd_md_graph_create``); ``replay`` launches
    it on torch's current stream."""

    def __init__(self, handle: int, device: torch.device):
        self.handle, self.device = handle, device

    def replay(self) -> None:
        call("nd_md_graph_launch", self.handle, stream_handle(self.device))

    def __del__(self):
        if getattr(self, "handle", None):
            try:
                _native.lib().nd_md_graph_destroy(self.handle)
            except Exception:
                pass
            self.handle = None


class Engine:
    """One Lennard-Jones system in the MD engine: its buffers, its frame and its calls."""

    def __init__(
        self,
        *,
        num_types: int,
        sigma: Tensor,
        epsilon: Tensor,
        cutoff: float,
        cell: Tensor,
        num_atoms: int,
        timestep: float,
        skin: float,
        capacity_multiplier: float,
        dtype: torch.dtype,
        device: torch.device,
    ):
        lengths = [float(length) for length in cell.tolist()]
        check_cell_lengths(lengths, cutoff)
        self.device, self.dtype = device, dtype
        self.num_atoms = n = int(num_atoms)
        self.cutoff, self.radius = float(cutoff), float(cutoff) + float(skin)
        self.lengths = lengths
        self.cell = cell.detach().to(device, dtype).contiguous()
        dims = grid(lengths, self.radius, dtype)
        small = min(dims) < 3
        position_bytes = 4 * torch.finfo(dtype).bits // 8
        if small and (n + 1) * position_bytes > _TILE_BYTES:
            raise ValueError(
                f"a cell with fewer than three list radii ({self.radius} nm) on an axis holds "
                f"at most {_TILE_BYTES // position_bytes - 1} atoms in this build",
            )
        bricks_x = 1
        if not small:
            per_cell = n / math.prod(dims)
            cells = max(1, min(_MAX_BRICK_CELLS, round(_CENTERS_PER_BRICK / max(per_cell, 1e-9))))
            bricks_x = max(1, math.ceil(dims[0] / cells))
            while math.ceil(dims[0] / bricks_x) > _MAX_BRICK_CELLS:
                bricks_x += 1
        eps = torch.finfo(dtype).eps
        allowance = self.radius - self.cutoff - 32 * eps * max(lengths)
        # A list without room to move rebuilds every step: any move exceeds a zero threshold.
        threshold = allowance * allowance / 4 if allowance > 0 else 0.0
        self.dims, self.small, self.bricks_x = dims, small, bricks_x
        self.capacity_multiplier = float(capacity_multiplier)
        # Tile slots, the sentinel's included, must fit shared memory and uint16 indices.
        self.tile_limit = min(65534, _TILE_BYTES // position_bytes - 1)
        num_cells = math.prod(dims)
        self.num_cells = num_cells

        floats = {"dtype": dtype, "device": device}
        ints = {"dtype": torch.int32, "device": device}
        longs = {"dtype": torch.int64, "device": device}
        doubles = {"dtype": torch.float64, "device": device}
        t = self.tensors = {}
        t["positions"] = torch.zeros((n, 4), **floats)
        t["velocities"] = torch.zeros((n, 3), **floats)
        t["forces"] = torch.zeros((n, 3), **floats)
        t["inverse_masses"] = torch.zeros(n, **floats)
        t["masses"] = torch.zeros(n, **floats)
        t["images"] = torch.zeros((n, 3), **longs)
        t["ids"] = torch.zeros(n, **ints)
        t["reference_positions"] = torch.zeros((n, 4), **floats)
        for name in ("positions", "velocities", "inverse_masses", "masses", "images", "ids"):
            t["shadow_" + name] = torch.zeros_like(t[name])
        t["cell_counts"] = torch.zeros(num_cells + 1, **ints)
        t["cell_offsets"] = torch.zeros(num_cells + 1, **ints)
        t["atom_cell"] = torch.zeros(n, **ints)
        t["slots"] = torch.zeros(n, **ints)
        t["unordered"] = torch.zeros(n, **ints)
        t["order"] = torch.zeros(n, **ints)
        scan_bytes = torch.empty(1, dtype=torch.int64)
        call("nd_neighbors_scan_temp_bytes", num_cells + 1,
             _native.ctypes.cast(scan_bytes.data_ptr(), _native.c_int64_p))
        t["scan_temp"] = torch.zeros(int(scan_bytes), dtype=torch.uint8, device=device)
        # List rows: one per atom on the small-box path; on the brick path two per center pair
        # (the halves of the pair's list; pairs never span two cells), fewer than
        # N + 2 cells + 2. The pair order holds two int32 per pair.
        self.list_rows = n if small else n + 2 * math.prod(dims) + 2
        t["neighbor_counts"] = torch.zeros(self.list_rows, **ints)
        t["pair_order"] = torch.zeros(2 * (self.list_rows // 2 + 1), **ints)
        t["rebuild"] = torch.zeros(2, **ints)  # the reuse flag; the step graph's drift count
        t["rebuild_count"] = torch.zeros(1, **ints)
        t["status"] = torch.zeros(4, **ints)
        t["totals"] = torch.zeros(16, **doubles)
        t["thermostat"] = torch.zeros(24, **doubles)
        t["sigma"] = sigma.detach().to(device, dtype).contiguous()
        t["epsilon"] = epsilon.detach().to(device, dtype).contiguous()
        self.num_types = int(num_types)
        self.system = MDSystem()
        s = self.system
        s.dtype = dtype_code(dtype)
        s.num_atoms = n
        s.num_types = self.num_types
        s.small = int(small)
        for axis in range(3):
            s.dims[axis] = dims[axis]
            s.cell[axis] = lengths[axis]
            s.widths[axis] = float(torch.tensor(lengths[axis] / dims[axis], dtype=dtype))
        s.bricks_x = bricks_x
        s.cutoff = self.cutoff
        s.radius = self.radius
        s.timestep = float(timestep)
        s.threshold_squared = float(threshold)
        # The sizing build: one chunk per atom, the largest tile shared memory allows.
        self._size_list(width=8, tile_capacity=self.tile_limit)
        slots = torch.empty(1, dtype=torch.int64)
        call("nd_md_partial_slots", s, _native.ctypes.cast(slots.data_ptr(), _native.c_int64_p))
        t["partials"] = torch.zeros(int(slots), **doubles)
        self._bind()

    # -- buffers ---------------------------------------------------------------------------

    def _size_list(self, width: int, tile_capacity: int) -> None:
        self.width, self.tile_capacity = int(width), int(tile_capacity)
        self.tensors["neighbors"] = torch.zeros(
            ((self.list_rows + 31) // 32) * 32 * self.width, dtype=torch.uint16,
            device=self.device,
        )
        self.system.width = self.width
        self.system.tile_capacity = self.tile_capacity

    def _bind(self) -> None:
        s, t = self.system, self.tensors
        for name in (
            "positions", "velocities", "forces", "inverse_masses", "masses", "images", "ids",
            "reference_positions", "shadow_positions", "shadow_velocities",
            "shadow_inverse_masses", "shadow_masses", "shadow_images", "shadow_ids",
            "cell_counts", "cell_offsets", "atom_cell", "slots", "unordered", "order",
            "scan_temp", "neighbors", "neighbor_counts", "pair_order", "rebuild", "rebuild_count",
            "status",
            "partials", "totals", "thermostat", "sigma", "epsilon",
        ):
            setattr(s, name, ptr(t[name]))

    def _stream(self) -> int:
        return stream_handle(self.device)

    # -- frame -----------------------------------------------------------------------------

    def load(self, positions: Tensor, velocities: Tensor, masses: Tensor, images: Tensor,
             types: Tensor | None) -> None:
        """Load a wrapped frame in the caller's order, size the list and compute the forces.

        Syncs with the host (the sizing reads the first build's needs).
        """
        s, t = self.system, self.tensors
        positions = positions.detach().to(self.dtype).contiguous()
        velocities = velocities.detach().to(self.dtype).contiguous()
        masses = masses.detach().to(self.dtype).contiguous()
        images = images.detach().to(torch.int64).contiguous()
        kernel_types = types.detach().to(torch.int32).contiguous() if types is not None else None
        for name in ("rebuild", "rebuild_count", "status", "cell_counts"):
            t[name].zero_()
        with torch.cuda.device(self.device):
            stream = self._stream()
            call("nd_md_import", s, ptr(positions), ptr(velocities), ptr(masses), ptr(images),
                 ptr(kernel_types), stream)
            call("nd_md_rebuild", s, stream)
            status = t["status"].tolist()
            needed_neighbors = max(status[1], 1)
            needed_tile = status[3] if not self.small else self.num_atoms
            if status[0] & ~OVERFLOW:
                raise ValueError("the first frame is not finite")
            if status[0] & OVERFLOW and status[2] > 0:
                raise ValueError(
                    f"a brick tile needs {status[2]} atoms, over the {self.tile_limit} that "
                    "shared memory holds; the density is too high for this build",
                )
            width = math.ceil(self.capacity_multiplier * needed_neighbors)
            width = max(8, -(-width // 8) * 8)
            # A tile sums thousands of atoms over tens of cells, so its count fluctuates by
            # about a percent in a liquid: it gets a quarter of the multiplier's margin plus
            # 64 slots (the list width, a count of a few atoms' neighbours, gets the whole
            # margin).
            tile_margin = 1.0 + (self.capacity_multiplier - 1.0) / 4
            tile = min(self.tile_limit, math.ceil(tile_margin * needed_tile) + 64)
            self._size_list(width, tile)
            self._bind()
            t["status"].zero_()
            t["rebuild_count"].zero_()
            # Reload: the sizing build permuted the state; importing again restores the order.
            call("nd_md_import", s, ptr(positions), ptr(velocities), ptr(masses), ptr(images),
                 ptr(kernel_types), stream)
            call("nd_md_rebuild", s, stream)
            call("nd_md_forces", s, 1, stream)

    def reload(self, positions: Tensor, velocities: Tensor, masses: Tensor, images: Tensor,
               types: Tensor | None) -> None:
        """Load another wrapped frame of the same system into the sized buffers: import,
        rebuild, forces. No host sync; a frame that needs more room than the buffers have
        sets the overflow bit, read with ``failure``."""
        s, t = self.system, self.tensors
        for name in ("rebuild", "status", "cell_counts"):
            t[name].zero_()
        with torch.cuda.device(self.device):
            stream = self._stream()
            call("nd_md_import", s, ptr(positions.contiguous()), ptr(velocities.contiguous()),
                 ptr(masses.contiguous()), ptr(images.contiguous()),
                 ptr(types.contiguous()) if types is not None else None, stream)
            call("nd_md_rebuild", s, stream)
            call("nd_md_forces", s, 0, stream)

    def set_thermostat(self, *, temperature: float, timescale: float, positions: Tensor,
                       momenta: Tensor, kinetic: float) -> None:
        """Load a Nose-Hoover chain of three at ``temperature`` with masses g kT tau^2, kT tau^2."""
        th = torch.zeros(24, dtype=torch.float64)
        kT = BOLTZMANN * temperature
        degrees = 3 * self.num_atoms - 3
        base = kT * timescale * timescale
        th[CHAIN_A:CHAIN_A + 3] = positions.detach().cpu().double()
        th[CHAIN_A + 3:CHAIN_A + 6] = momenta.detach().cpu().double()
        th[KINETIC_A] = kinetic
        th[PENDING_SCALE] = 1.0
        th[CHAIN_MASS:CHAIN_MASS + 3] = torch.tensor([degrees * base, base, base], dtype=torch.float64)
        th[THERMAL_ENERGY] = kT
        th[DEGREES] = degrees
        th[TIMESTEP] = self.system.timestep
        self.tensors["thermostat"].copy_(th)

    def make_graph(self, thermostat: bool, steps: int) -> "StepGraph":
        """A CUDA graph of ``steps`` steps whose rebuild runs behind a conditional node."""
        handle = _native.ctypes.c_void_p()
        with torch.cuda.device(self.device):
            call("nd_md_graph_create", self.system, int(thermostat), int(steps),
                 _native.ctypes.byref(handle))
        return StepGraph(handle.value, self.device)

    def step(self, thermostat: bool) -> None:
        with torch.cuda.device(self.device):
            call("nd_md_step", self.system, int(thermostat), 0, self._stream())

    # Small boxes up to this many atoms run many steps per launch (nd_md_run_small).
    ONE_LAUNCH_MAX_ATOMS = 4096

    @property
    def runs_in_one_launch(self) -> bool:
        """Whether ``run_steps`` applies: a small box of at most ONE_LAUNCH_MAX_ATOMS atoms."""
        return bool(self.small) and self.num_atoms <= self.ONE_LAUNCH_MAX_ATOMS

    def run_steps(self, thermostat: bool, steps: int) -> None:
        """``steps`` steps of a small box in one launch of one thread-block cluster
        (nd_md_run_small), as many ``step`` calls would make them."""
        with torch.cuda.device(self.device):
            call("nd_md_run_small", self.system, int(thermostat), int(steps), self._stream())

    def step_phase(self, phase: int, thermostat: bool) -> None:
        with torch.cuda.device(self.device):
            call("nd_md_step_phase", self.system, int(phase), int(thermostat), 0, self._stream())

    @property
    def step_launches(self) -> int:
        count = torch.empty(1, dtype=torch.int64)
        call("nd_md_step_launches", self.system,
             _native.ctypes.cast(count.data_ptr(), _native.c_int64_p))
        return int(count)

    def forces(self, virial: bool) -> None:
        with torch.cuda.device(self.device):
            call("nd_md_forces", self.system, int(virial), self._stream())

    def kinetic(self, thermostat: bool) -> None:
        with torch.cuda.device(self.device):
            call("nd_md_kinetic", self.system, int(thermostat), self._stream())

    def export(self, thermostat: bool) -> dict[str, Tensor]:
        """The frame in the caller's order: positions in [0, L), velocities, forces, images."""
        n = self.num_atoms
        out = {
            "positions": torch.empty((n, 3), dtype=self.dtype, device=self.device),
            "velocities": torch.empty((n, 3), dtype=self.dtype, device=self.device),
            "forces": torch.empty((n, 3), dtype=self.dtype, device=self.device),
            "images": torch.empty((n, 3), dtype=torch.int64, device=self.device),
        }
        with torch.cuda.device(self.device):
            call("nd_md_export", self.system, ptr(out["positions"]), ptr(out["velocities"]),
                 ptr(out["forces"]), ptr(out["images"]), int(thermostat), self._stream())
        return out

    def volume(self) -> float:
        """The cell volume in nm^3 (the LJ engine's cell is fixed)."""
        return math.prod(self.lengths)

    @property
    def status(self) -> Tensor:
        return self.tensors["status"]

    @property
    def totals(self) -> Tensor:
        return self.tensors["totals"]

    @property
    def thermostat(self) -> Tensor:
        return self.tensors["thermostat"]

    @property
    def rebuild_count(self) -> int:
        return int(self.tensors["rebuild_count"].item())

    def snapshot(self) -> dict[str, Tensor]:
        return {name: tensor.clone() for name, tensor in self.tensors.items()}

    def restore(self, saved: dict[str, Tensor]) -> None:
        for name, tensor in saved.items():
            self.tensors[name].copy_(tensor)

    def failure(self) -> str | None:
        """The decoded status, or None when sound. Syncs with the host."""
        flags, neighbors, tile, _ = self.tensors["status"].tolist()
        if not flags:
            return None
        causes = []
        if flags & _native.INVALID_CELL:
            causes.append("every cell length must be finite and above twice the cutoff")
        if flags & _native.NON_FINITE:
            causes.append("positions must be finite")
        if flags & STAGE_TIMEOUT:
            causes.append("a shared-memory tile copy did not complete")
        if flags & OVERFLOW:
            if neighbors > self.width:
                causes.append(
                    f"the neighbor capacity {self.width} per list is too small: a list needs "
                    f"{neighbors} neighbors within {self.radius} nm; raise capacity_multiplier",
                )
            if tile > self.tile_capacity:
                causes.append(
                    f"the tile capacity {self.tile_capacity} is too small: a brick needs {tile} "
                    "atoms; raise capacity_multiplier",
                )
        return "; ".join(causes)


__all__ = ("Engine",)
