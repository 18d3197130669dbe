"""The MD engine for models other than Lennard-Jones: a frame in the caller's order, the
neighbor operator's list, the model's forces and the integrator kernels of csrc/integrate.cu.

``PairEngine`` has the interface ``Simulation`` drives (``Engine``'s): load/reload a frame,
step, forces, kinetic, export, snapshot/restore, failure. A step launches, on torch's current
stream and without a host sync (so it is captured in a CUDA Graph):

* ``nd_integrate_open``: the chain's opening half step (NVT), the first half kick, the drift
  and the wrap with image counts;
* the neighbor operator's reuse check and gated rebuild (``NeighborList._update_wrapped``,
  src/nabladyn/neighbors/_neighbor_list.py:310-322);
* the forces: a float32 SchNet of 64 features runs its fused tensor-core kernels into the
  engine's buffers; any other model is differentiated by torch.func, as the reference does;
* ``nd_integrate_close``: the second half kick, K in float64 and the chain's closing half step.
"""

from __future__ import annotations

import torch
from torch import Tensor

from .. import _native, quantity
from .._native import Integrator, call, dtype_code, ptr, stream_handle
from ..neighbors import NeighborList
from ..neighbors._neighbor_list import check_cell_lengths, status_causes
from ..potential._schnet import SchNet
from ..units import BOLTZMANN
from ._engine import (
    CHAIN_A, CHAIN_MASS, DEGREES, KINETIC_A, PENDING_SCALE, THERMAL_ENERGY, TIMESTEP,
)

TENSOR_CORE_LOST = 16  # SchNet status bit: a tensor-core product did not complete in time


class PairEngine:
    """One system of any potential in the pair engine: buffers, list, frame and calls."""

    def __init__(self, *, model, cell: Tensor, num_atoms: int, timestep: float, skin: float,
                 capacity_multiplier: float, dtype: torch.dtype, device: torch.device):
        lengths = [float(length) for length in cell.tolist()]
        check_cell_lengths(lengths, model.cutoff)
        self.model = model
        self.device, self.dtype = device, dtype
        self.num_atoms = n = int(num_atoms)
        self.lengths = lengths
        self.radius = float(model.cutoff) + float(skin)
        # A list per cutoff of the model's parts (a sum gives each part its own list).
        self.neighbors = NeighborList(model.cutoff, skin=skin,
                                      capacity_multiplier=capacity_multiplier,
                                      inner_cutoffs=tuple(model._list_cutoffs[:-1]))
        self._fused = isinstance(model, SchNet) and model._fused_kernel
        slots = torch.empty(1, dtype=torch.int64)
        call("nd_integrate_partial_slots", n,
             _native.ctypes.cast(slots.data_ptr(), _native.c_int64_p))
        floats = dict(dtype=dtype, device=device)
        self.tensors = {
            "positions": torch.zeros((n, 3), **floats),
            "velocities": torch.zeros((n, 3), **floats),
            "forces": torch.zeros((n, 3), **floats),
            "masses": torch.ones(n, **floats),
            "images": torch.zeros((n, 3), dtype=torch.int64, device=device),
            "thermostat": torch.zeros(24, dtype=torch.float64, device=device),
            "partials": torch.zeros(int(slots), dtype=torch.float64, device=device),
            "totals": torch.zeros(16, dtype=torch.float64, device=device),
            "status": torch.zeros(4, dtype=torch.int32, device=device),
            "model_status": torch.zeros(4, dtype=torch.int32, device=device),
            "energy": torch.zeros(1, dtype=torch.float64, device=device),
            "virial": torch.zeros(9, dtype=torch.float64, device=device),
            "cell": cell.detach().to(device, dtype).contiguous().clone(),
            "barostat": torch.zeros(32, dtype=torch.float64, device=device),
        }
        self.cell = self.tensors["cell"]  # NPT rescales it in place
        self._npt = False
        self.workspace = None
        t = self.tensors
        self.system = Integrator(
            dtype=dtype_code(dtype), num_atoms=n, positions=ptr(t["positions"]),
            velocities=ptr(t["velocities"]), forces=ptr(t["forces"]), masses=ptr(t["masses"]),
            images=ptr(t["images"]), cell=ptr(self.cell), thermostat=ptr(t["thermostat"]),
            partials=ptr(t["partials"]), totals=ptr(t["totals"]), status=ptr(t["status"]),
            timestep=float(timestep), barostat=ptr(t["barostat"]), virial=ptr(t["virial"]),
        )
        self._evaluate = None if self._fused else quantity.energy_force_virial(
            model._energy_wrapped)

    def _stream(self) -> int:
        return stream_handle(self.device)

    # -- frame -----------------------------------------------------------------------------

    def load(self, positions: Tensor, velocities: Tensor, masses: Tensor, images: Tensor,
             types: Tensor | None) -> None:
        """Load a wrapped frame, size and build the list, compute the forces. Syncs."""
        t = self.tensors
        t["positions"].copy_(positions.detach())
        t["velocities"].copy_(velocities.detach())
        t["masses"].copy_(masses.detach())
        t["images"].copy_(images.detach())
        t["status"].zero_()
        self.neighbors.allocate(t["positions"], self.cell)
        if self._fused:
            from ..potential import _schnet_kernels

            self.workspace = torch.empty(
                _schnet_kernels.workspace_bytes(self.num_atoms, self.neighbors.pair_capacity,
                                                len(self.model.blocks)),
                dtype=torch.uint8, device=self.device)
        self.forces(virial=True)

    def reload(self, positions: Tensor, velocities: Tensor, masses: Tensor, images: Tensor,
               types: Tensor | None) -> None:
        """Another wrapped frame into the sized buffers: forced rebuild and forces; no sync."""
        t = self.tensors
        t["positions"].copy_(positions.detach())
        t["velocities"].copy_(velocities.detach())
        t["masses"].copy_(masses.detach())
        t["images"].copy_(images.detach())
        t["status"].zero_()
        self.neighbors._rebuild_wrapped(t["positions"], self.cell)
        self.forces(virial=False)

    def set_thermostat(self, *, temperature: float, timescale: float, positions: Tensor,
                       momenta: Tensor, kinetic: float) -> None:
        """A Nose-Hoover chain of three at ``temperature``, masses g kT tau^2, kT tau^2."""
        th = torch.zeros(24, dtype=torch.float64)
        kT = BOLTZMANN * temperature
        degrees = 3 * self.num_atoms - 3
        base = kT * timescale * timescale
        th[CHAIN_A:CHAIN_A + 3] = positions.detach().cpu().double()
        th[CHAIN_A + 3:CHAIN_A + 6] = momenta.detach().cpu().double()
        th[KINETIC_A] = kinetic
        th[PENDING_SCALE] = 1.0
        th[CHAIN_MASS:CHAIN_MASS + 3] = torch.tensor([degrees * base, base, base],
                                                     dtype=torch.float64)
        th[THERMAL_ENERGY] = kT
        th[DEGREES] = degrees
        th[TIMESTEP] = self.system.timestep
        self.tensors["thermostat"].copy_(th)

    def set_barostat(self, *, temperature: float, pressure: float, timescale: float,
                     momentum: Tensor, positions: Tensor, momenta: Tensor) -> None:
        """The isotropic MTK barostat: box momentum, its chain of three (masses kT tau_b^2),
        box mass 3 (N + 1) kT tau_b^2, pressure, alpha = 1 + 1/N and the float64 cell."""
        box = torch.zeros(32, dtype=torch.float64)
        kT = BOLTZMANN * temperature
        base = kT * timescale * timescale
        box[0] = float(momentum)
        box[1:4] = positions.detach().cpu().double()
        box[4:7] = momenta.detach().cpu().double()
        box[7:10] = torch.tensor([base, base, base], dtype=torch.float64)
        box[10] = 3 * (self.num_atoms + 1) * base
        box[11] = pressure
        box[12] = 1.0 + 1.0 / self.num_atoms
        box[13:16] = self.cell.detach().cpu().double()
        self.tensors["barostat"].copy_(box)
        self._npt = True

    # -- calls -----------------------------------------------------------------------------

    def _model_forces(self, virial: bool) -> None:
        t = self.tensors
        pairs = self.neighbors.tensors()
        if self._fused:
            from ..potential import _schnet_kernels

            _schnet_kernels.launch(self.model, t["positions"], self.cell, pairs.index,
                                   energy=t["energy"], forces=t["forces"],
                                   virial=t["virial"] if virial else None,
                                   status=t["model_status"], workspace=self.workspace)
        else:
            energy, forces, w = self._evaluate(t["positions"], self.cell, pairs)
            t["energy"].copy_(energy.detach().reshape(1))
            t["forces"].copy_(forces.detach())
            t["virial"].copy_(w.detach().reshape(9))

    def step(self, mode: int) -> None:
        """One step: mode 0 NVE, 1 NVT, 2 NPT."""
        t = self.tensors
        with torch.cuda.device(self.device):
            stream = self._stream()
            call("nd_integrate_open", self.system, int(mode), stream)
            self.neighbors._update_wrapped(t["positions"], self.cell)
            self._model_forces(virial=int(mode) == 2)
            call("nd_integrate_close", self.system, int(mode), stream)
            t["totals"][0:1].copy_(t["energy"])

    def forces(self, virial: bool) -> None:
        """Forces, E and (with ``virial``) W of the current frame into the totals."""
        t = self.tensors
        with torch.cuda.device(self.device):
            self._model_forces(virial)
            t["totals"][0:1].copy_(t["energy"])
            if virial:
                w = t["virial"]
                t["totals"][2:8].copy_(torch.stack([w[0], w[4], w[8], w[1], w[2], w[5]]))

    def kinetic(self, thermostat: bool) -> None:
        with torch.cuda.device(self.device):
            call("nd_integrate_kinetic", self.system, int(thermostat), self._stream())

    def export(self, thermostat: bool) -> dict[str, Tensor]:
        """The frame: positions in [0, L), velocities (pending chain factor applied), forces,
        images."""
        t = self.tensors
        velocities = t["velocities"].clone()
        if thermostat:
            velocities *= t["thermostat"][PENDING_SCALE].to(self.dtype)
        return {"positions": t["positions"].clone(), "velocities": velocities,
                "forces": t["forces"].clone(), "images": t["images"].clone(),
                "cell": t["cell"].clone()}

    def volume(self) -> float:
        """The cell volume in nm^3 (the float64 master cell under NPT). Syncs."""
        if self._npt:
            return float(self.tensors["barostat"][13:16].prod())
        return float(self.tensors["cell"].double().prod())

    @property
    def barostat(self) -> Tensor:
        return self.tensors["barostat"]

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
        return self.neighbors._rebuild_count

    def _list_tensors(self) -> dict[str, Tensor]:
        return {f"list.{name}": tensor
                for name, tensor in self.neighbors._device_tensors().items()}

    def snapshot(self) -> dict[str, Tensor]:
        saved = {name: tensor.clone() for name, tensor in self.tensors.items()}
        saved.update({name: tensor.clone() for name, tensor in self._list_tensors().items()})
        return saved

    def restore(self, saved: dict[str, Tensor]) -> None:
        live = dict(self.tensors)
        live.update(self._list_tensors())
        for name, tensor in saved.items():
            live[name].copy_(tensor)

    def failure(self) -> str | None:
        """The decoded status of the integrator, the list and the model, or None. Syncs."""
        causes = []
        if int(self.tensors["status"][0]) & _native.NON_FINITE:
            causes.append("positions must be finite")
        flags, needed = self.neighbors._device_tensors()["status"].tolist()
        for cause in status_causes(flags, needed, self.neighbors.pair_capacity, self.radius):
            if cause not in causes:
                causes.append(cause)
        if self._fused:
            model_flags = self.tensors["model_status"].tolist()
            if model_flags[1] & 1:
                causes.append("a pair index lies outside the atoms")
            if model_flags[1] & TENSOR_CORE_LOST:
                causes.append(
                    f"a tensor-core product did not complete (stage {model_flags[2]}, "
                    f"tile {model_flags[3]})")
        return "; ".join(causes) if causes else None


__all__ = ("PairEngine",)
