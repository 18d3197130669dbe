"""The replica server: a device pool of resident replicas and the continuous-batching loop.

Each request is an independent one-type Lennard-Jones NVT simulation (the reference's
``md.nvt``, src/nabladyn/md/_ensembles/_nvt.py:132-179, in float32). The server

* admits a request when a slot and room in the HBM budget are free (first fit over the pool's
  atom ranges), uploads its frame and has the replica kernel build its list and first forces;
  the host work of an admission (the slot record, the frame in pinned memory) is done ahead,
  while the device runs the previous round, and the upload itself needs no host sync;
* every round launches the replica kernel once over all active slots, each slot with a budget
  of steps inversely proportional to its size, so a round costs about the same on every SM and
  small replicas are not held back by large ones;
* harvests replicas whose steps are done (their frames read back together, in one copy),
  hands back their frame and frees their room, so requests that arrived meanwhile are
  admitted in the next round;
* pipelines the rounds: the next round is on the device while the host reads the last one's
  slot table, harvests and admits, so the device does not wait for the host between rounds.

Replicas never interact on the device: each is advanced by its own CTA, so a replica's result
does not depend on which others share its rounds.
"""

from __future__ import annotations

import ctypes
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from .._native import Replica, ReplicaPool, call, stream_handle
from ..neighbors._neighbor_list import check_cell_lengths, grid
from ..units import BOLTZMANN

_ALIGN = 32          # atoms per allocation unit (one warp of list chunks)
_MAX_CELLS = 4096    # kServeMaxCells in serve.cu
_WIDTH = 192         # list slots per atom: room for ~1.5x the mean count at 22 atoms/nm^3
_BYTES_PER_ATOM = 16 + 12 + 12 + 4 + 4 + 24 + 16 + 2 * _WIDTH + 4 + 4 + 4 + 16
_CHAIN_A, _KINETIC_A, _PENDING, _CHAIN_MASS, _KT, _DEGREES, _TIMESTEP = 0, 6, 14, 16, 19, 20, 21


@dataclass
class ReplicaRequest:
    """One MD job: a frame, its thermostat settings and the number of NVT steps.

    positions and velocities [N, 3] in nm and nm/ps, masses [N] in Da, cell [3] in nm (host
    arrays); ``arrival`` in seconds after serving starts.
    """

    positions: np.ndarray
    velocities: np.ndarray
    masses: np.ndarray
    cell: np.ndarray
    temperature: float
    steps: int
    timestep: float = 0.004
    thermostat_timescale: float = 0.1
    sigma: float = 0.34
    epsilon: float = 0.996
    cutoff: float = 1.0
    skin: float = 0.1
    arrival: float = 0.0
    name: object = None


@dataclass
class ReplicaResult:
    """A finished replica: its final frame (positions wrapped into the cell), its potential
    energy, and its times in seconds after serving started."""

    name: object
    positions: np.ndarray
    velocities: np.ndarray
    images: np.ndarray
    energy: float
    status: int
    rebuilds: int
    arrival: float
    admitted: float
    finished: float
    num_atoms: int
    steps: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Active:
    request: ReplicaRequest
    slot: int
    offset: int
    units: int
    admitted: float
    steps_left: int = field(default=0)


@dataclass
class _Staged:
    """A request made ready on the host while the device runs a round: its slot record (all
    but the offsets) and its frame in pinned memory, uploaded without a host sync."""

    record: Replica
    frame: torch.Tensor  # [n, 9] float32: x, y, z, 0, vx, vy, vz, m, 1/m


@dataclass
class _Lane:
    """One stream of rounds: its active replicas by slot, its rounds launched and not yet read
    (slots, table copy, event), its table copies' host buffers and the room its harvested
    replicas free once its later rounds have run. ``steps`` is the fixed budget of a round
    (None: the round's atom-steps divided by the replica's size)."""

    name: str
    stream: torch.cuda.Stream
    steps: int | None
    active: dict = field(default_factory=dict)
    rounds: deque = field(default_factory=deque)
    deferred: deque = field(default_factory=deque)
    table_hosts: list | None = None
    table_turn: int = 0

    def budget(self, entry: _Active, round_atom_steps: int) -> int:
        n = entry.request.positions.shape[0]
        steps = self.steps if self.steps is not None else -(-round_atom_steps // n)
        return max(1, min(entry.steps_left, steps))


class ReplicaServer:
    """Resident replicas in one device pool, advanced in rounds by the replica kernel.

    ``budget_bytes`` bounds the pool (about 0.5 kB per atom); ``max_slots`` bounds the replicas
    resident at once; ``round_atom_steps`` is the work a slot gets per round, in atom-steps;
    ``stage_ahead`` is how many arrived requests the host makes ready (slot record, frame in
    pinned memory) while a round runs on the device (0: each at its admission).
    ``large_atoms``: replicas of at least this many atoms run in rounds of their own, on a
    second stream, ``large_round_steps`` steps a round (None: one stream for all).
    """

    def __init__(self, *, device: torch.device | str = "cuda", budget_bytes: int = 4 << 30,
                 max_slots: int = 2048, round_atom_steps: int = 200_000, stage_ahead: int = 32,
                 large_atoms: int | None = 8192, large_round_steps: int = 25):
        self.device = torch.device(device)
        self.stage_ahead = int(stage_ahead)
        self.large_atoms = None if large_atoms is None else int(large_atoms)
        self.large_round_steps = int(large_round_steps)
        self.max_slots = int(max_slots)
        self.round_atom_steps = int(round_atom_steps)
        self.capacity = max(_ALIGN, (int(budget_bytes) // _BYTES_PER_ATOM) // _ALIGN * _ALIGN)
        n, dev = self.capacity, self.device
        f32 = {"dtype": torch.float32, "device": dev}
        i32 = {"dtype": torch.int32, "device": dev}
        self.buffers = {
            "positions": torch.zeros((n, 4), **f32),
            "velocities": torch.zeros((n, 3), **f32),
            "forces": torch.zeros((n, 3), **f32),
            "masses": torch.ones(n, **f32),
            "inverse_masses": torch.ones(n, **f32),
            "images": torch.zeros((n, 3), dtype=torch.int64, device=dev),
            "reference_positions": torch.zeros((n, 4), **f32),
            "neighbors": torch.zeros(n * _WIDTH, dtype=torch.uint16, device=dev),
            "neighbor_counts": torch.zeros(n, **i32),
            "sorted": torch.zeros(n, **i32),
            "scratch": torch.zeros(n, **i32),
            "cell_starts": torch.zeros(self.max_slots * (_MAX_CELLS + 1), **i32),
            "ordered_positions": torch.zeros((n, 4), **f32),
        }
        self.table = torch.zeros(self.max_slots * ctypes.sizeof(Replica), dtype=torch.uint8,
                                 device=dev)
        pool = ReplicaPool(replicas=self.table.data_ptr())
        for name, tensor in self.buffers.items():
            setattr(pool, name, tensor.data_ptr())
        self.pool = pool
        self._free_units = [(0, n // _ALIGN)]  # (first unit, units), sorted, merged
        self._pinned: dict[str, list] = {}  # _upload's areas
        self._pinned_turn: dict[str, int] = {}
        self._free_slots = list(range(self.max_slots - 1, -1, -1))

    # -- room ----------------------------------------------------------------------------

    def _take(self, units: int) -> int | None:
        for k, (first, length) in enumerate(self._free_units):
            if length >= units:
                if length == units:
                    self._free_units.pop(k)
                else:
                    self._free_units[k] = (first + units, length - units)
                return first
        return None

    def _give(self, first: int, units: int) -> None:
        spans = sorted(self._free_units + [(first, units)])
        merged = []
        for start, length in spans:
            if merged and merged[-1][0] + merged[-1][1] == start:
                merged[-1] = (merged[-1][0], merged[-1][1] + length)
            else:
                merged.append((start, length))
        self._free_units = merged

    def fits(self, num_atoms: int) -> bool:
        units = -(-num_atoms // _ALIGN)
        return bool(self._free_slots) and any(length >= units for _, length in self._free_units)

    # -- admission -----------------------------------------------------------------------

    def _describe(self, request: ReplicaRequest, slot: int,
                  offset: int) -> tuple[Replica, np.ndarray]:
        """The slot record of a request and its float32 velocities, center of mass removed."""
        n = int(request.positions.shape[0])
        if not 2 <= n <= 65535:
            raise ValueError("a replica holds 2 to 65535 atoms")
        lengths = [float(x) for x in request.cell]
        check_cell_lengths(lengths, request.cutoff)
        radius = float(request.cutoff) + float(request.skin)
        dims = grid(lengths, radius, torch.float32)
        if min(dims) < 3:
            dims = [1, 1, 1]  # every pair is tested
        while math.prod(dims) > _MAX_CELLS:
            axis = int(np.argmax(dims))
            dims[axis] -= 1
        eps = float(np.finfo(np.float32).eps)
        allowance = radius - float(request.cutoff) - 32 * eps * max(lengths)
        record = Replica()
        record.atom_offset = offset
        record.list_offset = offset * _WIDTH
        record.cell_offset = slot * (_MAX_CELLS + 1)
        record.num_atoms = n
        record.width = _WIDTH
        for a in range(3):
            record.dims[a] = dims[a]
            record.cell[a] = lengths[a]
            record.widths[a] = float(np.float32(lengths[a] / dims[a]))
        record.cutoff = request.cutoff
        record.radius = radius
        record.threshold_squared = allowance * allowance / 4 if allowance > 0 else 0.0
        record.timestep = request.timestep
        record.sigma = request.sigma
        record.epsilon = request.epsilon
        record.steps_left = int(request.steps)
        masses = np.asarray(request.masses, dtype=np.float64)
        velocities = np.asarray(request.velocities, dtype=np.float64)
        velocities = velocities - (masses[:, None] * velocities).sum(axis=0) / masses.sum()
        velocities32 = velocities.astype(np.float32)
        kinetic = 0.5 * float((masses[:, None] * velocities32.astype(np.float64) ** 2).sum())
        kT = BOLTZMANN * float(request.temperature)
        degrees = 3 * n - 3
        base = kT * float(request.thermostat_timescale) ** 2
        record.thermostat[_KINETIC_A] = kinetic
        record.thermostat[_PENDING] = 1.0
        record.thermostat[_CHAIN_MASS] = degrees * base
        record.thermostat[_CHAIN_MASS + 1] = base
        record.thermostat[_CHAIN_MASS + 2] = base
        record.thermostat[_KT] = kT
        record.thermostat[_DEGREES] = degrees
        record.thermostat[_TIMESTEP] = request.timestep
        return record, velocities32

    def _stage(self, request: ReplicaRequest) -> _Staged:
        """The host part of an admission: the record and the frame (uploaded by _place)."""
        record, velocities32 = self._describe(request, 0, 0)
        n = record.num_atoms
        frame = torch.empty((n, 9), dtype=torch.float32)
        masses = np.asarray(request.masses, dtype=np.float32)
        host = frame.numpy()
        host[:, :3] = np.asarray(request.positions, dtype=np.float32)
        host[:, 3] = 0.0
        host[:, 4:7] = velocities32
        host[:, 7] = masses
        host[:, 8] = 1.0 / masses
        return _Staged(record, frame)

    def _upload(self, name: str, values: np.ndarray) -> torch.Tensor:
        """A host array on the device without a host sync, on the current stream: through one
        of two pinned areas kept per `name` and grown as needed (a copy from pageable memory
        would wait for the round running on the stream, and a new pinned block per call costs
        more than the copy). An area is reused after the copy made from it two calls before,
        which an earlier round's completion has already finished in the serve loop."""
        values = np.ascontiguousarray(values)
        areas = self._pinned.setdefault(name, [[None, None], [None, None]])
        turn = self._pinned_turn[name] = self._pinned_turn.get(name, 1) ^ 1
        area, copied = areas[turn]
        if copied is not None:
            copied.synchronize()
        if area is None or area.numel() < values.nbytes:
            grown = max(values.nbytes, 2 * (area.numel() if area is not None else 0), 1 << 16)
            area = torch.empty(grown, dtype=torch.uint8, pin_memory=True)
        host = area[:values.nbytes]
        host.numpy()[:] = values.reshape(-1).view(np.uint8)
        device = host.to(self.device, non_blocking=True)
        copied = torch.cuda.Event()
        copied.record(torch.cuda.current_stream(self.device))
        areas[turn] = [area, copied]
        dtype = torch.from_numpy(np.empty(0, dtype=values.dtype)).dtype
        return device.view(dtype).reshape(values.shape)

    def _place(self, batch: list[tuple[_Staged, int, int]], lane: str = "") -> None:
        """The device part of admissions, for a batch at once: the frames' pinned rows copied
        into one device block and scattered into the pool, the slot records written with their
        offsets; no host sync."""
        if not batch:
            return
        size = ctypes.sizeof(Replica)
        records = bytearray()
        destination = []
        for staged, slot, offset in batch:
            record = staged.record
            n = record.num_atoms
            record.atom_offset = offset
            record.list_offset = offset * _WIDTH
            record.cell_offset = slot * (_MAX_CELLS + 1)
            records += ctypes.string_at(ctypes.addressof(record), size)
            destination.append(np.arange(offset, offset + n, dtype=np.int64))
        frames = np.concatenate([staged.frame.numpy() for staged, _, _ in batch])
        rows = self._upload("frames" + lane, frames)
        index = self._upload("rows" + lane, np.concatenate(destination))
        b = self.buffers
        b["positions"].index_copy_(0, index, rows[:, :4])
        b["velocities"].index_copy_(0, index, rows[:, 4:7])
        b["forces"].index_fill_(0, index, 0.0)
        b["masses"].index_copy_(0, index, rows[:, 7])
        b["inverse_masses"].index_copy_(0, index, rows[:, 8])
        b["images"].index_fill_(0, index, 0)
        slots = self._upload("slots" + lane,
                             np.array([slot for _, slot, _ in batch], dtype=np.int64))
        table = self._upload("records" + lane,
                             np.frombuffer(bytes(records), dtype=np.uint8).reshape(-1, size))
        self.table.view(self.max_slots, size).index_copy_(0, slots, table)

    def _launch(self, slots: list[int], budgets: list[int] | None, mode: int,
                lane: str = "") -> None:
        if not slots:
            return
        slot_tensor = self._upload(f"launch_slots_{mode}{lane}",
                                   np.asarray(slots, dtype=np.int32))
        budget_tensor = (self._upload("launch_budgets" + lane,
                                      np.asarray(budgets, dtype=np.int32))
                         if budgets is not None else None)
        with torch.cuda.device(self.device):
            call("nd_serve_run", self.pool, slot_tensor.data_ptr(),
                 budget_tensor.data_ptr() if budget_tensor is not None else None,
                 len(slots), mode, stream_handle(self.device))

    @staticmethod
    def _int_field(raw: np.ndarray, name: str) -> np.ndarray:
        """One int32 field of every slot, read straight from the table's bytes."""
        offset = getattr(Replica, name).offset
        return np.ascontiguousarray(raw[:, offset:offset + 4]).view(np.int32)[:, 0]

    def _harvest(self, done: list[tuple[_Active, np.ndarray]], now: float,
                 freed: list[tuple[int, int, int]]) -> list[ReplicaResult]:
        """Finished replicas' frames (positions wrapped as space.wrap does, pending chain factor
        applied to the velocities, images with the last crossings): computed on the device for
        all of them together and read back in one copy; their room and slots go to `freed` as
        (first unit, units, slot)."""
        if not done:
            return []
        rows, cells, scales, sizes = [], [], [], []
        for active, raw in done:
            record = Replica.from_buffer_copy(raw.tobytes())
            n, offset = record.num_atoms, active.offset
            rows.append(np.arange(offset, offset + n, dtype=np.int64))
            cells.append(np.broadcast_to(np.asarray(record.cell, dtype=np.float32), (n, 3)))
            scales.append(np.full(n, np.float32(record.thermostat[_PENDING]), dtype=np.float32))
            sizes.append((record, n))
        index = self._upload("harvest_rows", np.concatenate(rows))
        cell = self._upload("harvest_cells", np.concatenate(cells))
        scale = self._upload("harvest_scales", np.concatenate(scales))
        unwrapped = self.buffers["positions"][index, :3]
        crossings = torch.floor(unwrapped / cell)
        wrapped = unwrapped - crossings * cell
        below = wrapped < 0
        wrapped = torch.where(below, wrapped + cell, wrapped)
        crossings = torch.where(below, crossings - 1, crossings)
        above = wrapped >= cell
        wrapped = torch.where(above, wrapped - cell, wrapped)
        crossings = torch.where(above, crossings + 1, crossings)
        velocities = self.buffers["velocities"][index] * scale[:, None]
        images = self.buffers["images"][index] + crossings.to(torch.int64)
        frame = torch.cat([wrapped, velocities], dim=1).cpu().numpy()
        images = images.cpu().numpy()
        results, begin = [], 0
        for (active, _), (record, n) in zip(done, sizes):
            end = begin + n
            results.append(ReplicaResult(
                name=active.request.name,
                positions=frame[begin:end, :3].copy(),
                velocities=frame[begin:end, 3:].copy(),
                images=images[begin:end].copy(),
                energy=float(record.energy),
                status=int(record.status),
                rebuilds=int(record.rebuild_count),
                arrival=float(active.request.arrival),
                admitted=active.admitted,
                finished=now,
                num_atoms=n,
                steps=int(active.request.steps) - int(record.steps_left),
            ))
            begin = end
            freed.append((active.offset // _ALIGN, active.units, active.slot))
        return results

    def _release(self, freed: list[tuple[int, int, int]]) -> None:
        for first, units, slot in freed:
            self._give(first, units)
            self._free_slots.append(slot)

    # -- the loop ------------------------------------------------------------------------

    def serve(self, requests: list[ReplicaRequest], *,
              realtime: bool = True) -> list[ReplicaResult]:
        """Serve requests by their arrival times; returns the results in completion order.

        With ``realtime`` the arrivals follow the wall clock from the call (a request is
        admitted only once its arrival time has passed); without, all are present at once.

        Replicas run in rounds on one of two lanes, each a stream of its own: replicas of at
        least ``large_atoms`` atoms ``large_round_steps`` steps a round, the others a budget of
        steps inversely proportional to their size. A large replica is then not held to a small
        share of every round while many small ones wait (it would finish last, on a nearly idle
        GPU), and a round of small replicas does not wait for the large ones' CTAs; the two
        lanes' CTAs share the SMs.

        The rounds are pipelined: each lane keeps its next round queued behind the running
        one, and the host polls the lanes, reading a round's slot table once it has run,
        harvesting the replicas that finished in it (on a side stream) and admitting new ones.
        A slot keeps its replica in every round launched before the host learns that it
        finished; the kernel clamps each budget to the steps left, so such a replica runs no
        further step, and its slot and room are reused only once those rounds have run.
        """
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        for request in pending:
            n = request.positions.shape[0]
            if -(-n // _ALIGN) > self.capacity // _ALIGN:
                raise ValueError(f"a replica of {n} atoms exceeds the server's budget")
        lanes = [_Lane("", torch.cuda.current_stream(self.device), None)]
        if self.large_atoms is not None:
            lanes.append(_Lane("_large", torch.cuda.Stream(self.device), self.large_round_steps))
        results: list[ReplicaResult] = []
        staged: dict[int, _Staged] = {}  # by id(request): host work done ahead of admission
        # High priority: the harvest's few small kernels go ahead of the rounds' waiting CTAs.
        side = torch.cuda.Stream(self.device, priority=-1)
        start = time.perf_counter()

        def lane_of(request: ReplicaRequest) -> _Lane:
            large = self.large_atoms is not None and request.positions.shape[0] >= self.large_atoms
            return lanes[-1] if large else lanes[0]

        def stage_ahead(now: float) -> None:
            # Host preparation of the requests that have arrived, a bounded number ahead.
            for request in list(pending)[:self.stage_ahead]:
                if realtime and request.arrival > now:
                    break
                if id(request) not in staged:
                    staged[id(request)] = self._stage(request)

        while pending or any(lane.active or lane.rounds for lane in lanes):
            for lane in lanes:  # room and slots whose last rounds have run
                while lane.deferred and (lane.deferred[0][0] is None or
                                         lane.deferred[0][0].query()):
                    self._release(lane.deferred.popleft()[1])
            now = time.perf_counter() - start
            placing: dict[str, list] = {lane.name: [] for lane in lanes}
            while pending and (not realtime or pending[0].arrival <= now):
                request = pending[0]
                units = -(-request.positions.shape[0] // _ALIGN)
                if not self._free_slots:
                    break
                first = self._take(units)
                if first is None:
                    break
                pending.popleft()
                slot = self._free_slots.pop()
                offset = first * _ALIGN
                ready = staged.pop(id(request)) if id(request) in staged else self._stage(request)
                lane = lane_of(request)
                placing[lane.name].append((ready, slot, offset))
                # The pinned frame may go once its copy is queued: the host allocator keeps
                # the block until the copy has run.
                lane.active[slot] = _Active(request, slot, offset, units, now,
                                            int(request.steps))
            progressed = False
            for lane in lanes:
                with torch.cuda.stream(lane.stream):
                    batch = placing[lane.name]
                    self._place(batch, lane.name)
                    self._launch([slot for _, slot, _ in batch], None, 0, lane.name)
                    if lane.active and len(lane.rounds) < 2:
                        launched = [(slot, lane.active[slot]) for slot in lane.active]
                        budgets = [lane.budget(entry, self.round_atom_steps)
                                   for _, entry in launched]
                        self._launch([slot for slot, _ in launched], budgets, 1, lane.name)
                        lane.rounds.append((launched, *self._table_copy(lane)))
                        progressed = True
            # While the rounds run: the next admissions' host work, then the finished rounds.
            if self.stage_ahead:
                stage_ahead(time.perf_counter() - start)
            for lane in lanes:
                # A round is read once it has run; with one lane, as soon as the next round is
                # queued behind it (or none will be), waiting for it.
                alone = len(lanes) == 1 and (len(lane.rounds) == 2 or not lane.active)
                if lane.rounds and (alone or lane.rounds[0][2].query()):
                    freed: list[tuple[int, int, int]] = []
                    results.extend(self._collect(lane.rounds.popleft(), lane.active, side,
                                                 start, freed))
                    if len(lanes) == 1:
                        self._release(freed)  # the stream's order keeps later rounds apart
                    elif freed:
                        last = lane.rounds[-1][2] if lane.rounds else None
                        lane.deferred.append((last, freed))
                    progressed = True
            if not progressed:
                if not any(lane.active or lane.rounds for lane in lanes) and pending and realtime:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.001)))
                else:
                    time.sleep(5e-5)
        for lane in lanes:
            lane.stream.synchronize()
        side.synchronize()
        for lane in lanes:
            for _, freed in lane.deferred:
                self._release(freed)
        return results

    def _table_copy(self, lane: "_Lane") -> tuple[torch.Tensor, torch.cuda.Event]:
        """The slot table after the round just launched on the lane's stream, copied to pinned
        host memory without a host sync (two buffers per lane in turn: a lane has at most two
        rounds outstanding, and a copy is read before the one after next is made)."""
        if lane.table_hosts is None:
            lane.table_hosts = [torch.empty_like(self.table, device="cpu").pin_memory()
                                for _ in range(2)]
        host = lane.table_hosts[lane.table_turn]
        lane.table_turn ^= 1
        host.copy_(self.table, non_blocking=True)
        event = torch.cuda.Event()
        event.record(torch.cuda.current_stream(self.device))
        return host, event

    def _collect(self, round_, active: dict[int, _Active], side: torch.cuda.Stream,
                 start: float, freed: list[tuple[int, int, int]]) -> list[ReplicaResult]:
        """Reads a round's slot table (waiting for that round only) and harvests the replicas
        it finished. A slot whose replica changed since the round was launched is skipped: its
        entry in that table still describes the replica that left."""
        launched, host, event = round_
        event.synchronize()
        raw = host.view(self.max_slots, ctypes.sizeof(Replica)).numpy()
        now = time.perf_counter() - start
        steps_left_all = self._int_field(raw, "steps_left")
        status_all = self._int_field(raw, "status")
        done = []
        for slot, entry in launched:
            if active.get(slot) is not entry:
                continue
            steps_left, status = int(steps_left_all[slot]), int(status_all[slot])
            entry.steps_left = steps_left
            if steps_left == 0 or status != 0:
                done.append((active.pop(slot), raw[slot].copy()))
        if not done:
            return []
        # The round after this one is running on the main stream; the finished replicas' rows
        # are not written by it (their budgets clamp to zero steps), so they are read on a side
        # stream after this round.
        side.wait_event(event)
        with torch.cuda.stream(side):
            return self._harvest(done, now, freed)

__all__ = ("ReplicaRequest", "ReplicaResult", "ReplicaServer")
