"""The simulation: it owns a running frame in the MD engine and CUDA Graphs of its steps.

Mirrors src/nabladyn/md/_simulation.py (Simulation :126-421, nve/nvt in _ensembles): the same
constructors, ``run`` / ``sample`` / ``state`` contract, panel fields, status polling every
1,000 steps and failure latching. For Lennard-Jones the step is the engine's (md.cu): a drift
kernel with the reuse check, the rebuild behind a device flag, and a force kernel with the
second half kick and the float64 tail. Any other model runs in the pair engine
(``PairEngine``: the integrator kernels, the neighbor operator and the model's forces, fused
tensor-core kernels for SchNet). ``run`` replays graphs of one step and of ``_CHUNK`` steps.
"""

from __future__ import annotations

import math
import sys
from numbers import Integral, Real
from typing import TextIO

import torch
from torch import Tensor

from .. import space
from ..potential import Potential
from ..potential._lennard_jones import LennardJones
from ..units import BOLTZMANN
from ._engine import CHAIN_A, CHAIN_MASS, DEGREES, PENDING_SCALE, THERMAL_ENERGY, Engine
from ._output import FRAME, SampleWriter
from ._pair_engine import PairEngine
from ._state import BarostatState, ChainState, State

_STATUS_INTERVAL = 1000  # steps between reads of the status


def _kernel_types(model):
    """The int32 types the Lennard-Jones engine takes for a multi-type model, else None."""
    if isinstance(model, LennardJones) and model.num_types > 1:
        return model._kernel_types
    return None

_CHUNK = 64  # steps per replay of the long graph
FIELDS = ("potential_energy", "kinetic_energy", "total_energy", "temperature", "pressure")


def _positive(name: str, value) -> float:
    if isinstance(value, bool) or not isinstance(value, Real) or not math.isfinite(value) or value <= 0:
        raise ValueError(f"{name} must be a finite positive number")
    return float(value)


def _count(name: str, value) -> int:
    if isinstance(value, bool) or not isinstance(value, Integral) or value < 0:
        raise ValueError(f"{name} must be a nonnegative integer")
    return int(value)


def _check_frame(model, positions, velocities, masses, cell) -> None:
    num_atoms, dtype, device = model.num_atoms, model.dtype, model.device
    for name, value, shape in (
        ("positions", positions, (num_atoms, 3)),
        ("velocities", velocities, (num_atoms, 3)),
        ("masses", masses, (num_atoms,)),
        ("cell", cell, (3,)),
    ):
        if (
            not isinstance(value, Tensor)
            or value.shape != shape
            or value.dtype != dtype
            or value.device != device
        ):
            raise ValueError(
                f"{name} must be a {list(shape)} tensor of {dtype} on {device} to match the model",
            )


def _check_chain(chain, device, name: str) -> None:
    for field, value in zip(("positions", "momenta"), chain):
        if (
            not isinstance(value, Tensor)
            or value.shape != (3,)
            or value.dtype != torch.float64
            or value.device != device
        ):
            raise ValueError(f"{name}.{field} must be a [3] float64 tensor on {device}")


class Simulation:
    """Molecular dynamics of a Lennard-Jones model on the GPU; build it with ``nve`` or ``nvt``.

    It owns its frame in the engine (cell-ordered, resident on the device) and CUDA Graphs of
    its step. The panel of ``FIELDS`` (potential, kinetic and total energy in kJ/mol, the
    temperature over 3N - 3 degrees of freedom in K, the pressure in kJ/mol/nm^3), plus
    ``conserved_energy`` for NVT, is evaluated on demand.
    """

    def __init__(
        self,
        model: Potential,
        positions: Tensor,
        velocities: Tensor,
        masses: Tensor,
        cell: Tensor,
        *,
        ensemble: dict,
        timestep: Real,
        skin: Real,
        capacity_multiplier: Real,
        images: Tensor | None,
        step: Integral,
    ):
        if not isinstance(model, Potential):
            raise TypeError("model must be a Potential")
        num_atoms, device = model.num_atoms, model.device
        _check_frame(model, positions, velocities, masses, cell)
        if images is None:
            images = torch.zeros((num_atoms, 3), dtype=torch.int64, device=device)
        elif (
            not isinstance(images, Tensor)
            or images.shape != (num_atoms, 3)
            or images.dtype != torch.int64
            or images.device != device
        ):
            raise ValueError(f"images must be a [{num_atoms}, 3] int64 tensor on {device}")
        timestep = _positive("timestep", timestep)
        self._step = _count("step", step)
        velocities, masses = velocities.detach(), masses.detach().clone()
        if not bool(torch.isfinite(velocities).all()):
            raise ValueError("velocities must be finite")
        if not bool((torch.isfinite(masses) & (masses > 0)).all()):
            raise ValueError("masses must be finite and positive")
        for name, value in (("skin", skin), ("capacity_multiplier", capacity_multiplier)):
            if isinstance(value, bool) or not isinstance(value, Real) or not math.isfinite(value):
                raise ValueError(f"{name} must be a finite number")
        if skin < 0 or capacity_multiplier < 1:
            raise ValueError("skin must be nonnegative and capacity_multiplier at least 1")
        if not isinstance(positions, Tensor) or not positions.is_cuda:
            raise TypeError("positions must be a CUDA float32 or float64 tensor")
        if not bool(torch.isfinite(positions).all()):
            raise ValueError("positions must be finite")
        name = ensemble["name"]
        self._thermostat = name in ("NVT", "NPT")
        self._mode = {"NVE": 0, "NVT": 1, "NPT": 2}[name]
        if self._thermostat and num_atoms < 2:
            raise ValueError(f"{name} needs at least 2 atoms, for 3N - 3 degrees of freedom")
        cell = cell.detach().clone()
        if isinstance(model, LennardJones) and name != "NPT":
            self._engine = Engine(
                num_types=model.num_types,
                sigma=model.sigma,
                epsilon=model.epsilon,
                cutoff=model.cutoff,
                cell=cell,
                num_atoms=num_atoms,
                timestep=timestep,
                skin=float(skin),
                capacity_multiplier=float(capacity_multiplier),
                dtype=model.dtype,
                device=device,
            )
        else:
            self._engine = PairEngine(
                model=model,
                cell=cell,
                num_atoms=num_atoms,
                timestep=timestep,
                skin=float(skin),
                capacity_multiplier=float(capacity_multiplier),
                dtype=model.dtype,
                device=device,
            )
        wrapped, crossings = space.wrap(positions.detach(), cell)
        # The center-of-mass velocity is a constant of motion; at zero it leaves 3N - 3 degrees
        # of freedom for the temperature and the thermostat.
        column = masses[:, None]
        velocities = velocities - (column * velocities).sum(dim=0) / masses.sum()
        types = _kernel_types(model)
        self._engine.load(wrapped, velocities, masses, images + crossings, types)
        self._model, self._masses, self._timestep, self._cell = model, masses, timestep, cell
        self._degrees_of_freedom = 3 * num_atoms - 3
        self._settings = {key: value for key, value in ensemble.items()
                          if key not in ("chain", "barostat")}
        self._settings["ensemble"] = ensemble["name"]
        self._settings.pop("name")
        self._fields = FIELDS + {0: (), 1: ("conserved_energy",),
                                 2: ("volume", "conserved_energy")}[self._mode]
        if self._thermostat:
            chain = ensemble.get("chain")
            if chain is None:
                chain_q = torch.zeros(3, dtype=torch.float64)
                chain_p = torch.zeros(3, dtype=torch.float64)
            else:
                _check_chain(chain, device, "thermostat")
                chain_q, chain_p = chain[0], chain[1]
            kinetic = 0.5 * float((masses.double()[:, None] * velocities.double().square()).sum())
            self._engine.set_thermostat(
                temperature=ensemble["temperature"],
                timescale=ensemble["thermostat_timescale"],
                positions=chain_q,
                momenta=chain_p,
                kinetic=kinetic,
            )
        if self._mode == 2:
            barostat = ensemble.get("barostat")
            momentum = torch.zeros((), dtype=torch.float64)
            box_q = torch.zeros(3, dtype=torch.float64)
            box_p = torch.zeros(3, dtype=torch.float64)
            if barostat is not None:
                if (not isinstance(barostat.momentum, Tensor) or barostat.momentum.shape != ()
                        or barostat.momentum.dtype != torch.float64
                        or barostat.momentum.device != device):
                    raise ValueError(f"barostat.momentum must be a [] float64 tensor on {device}")
                momentum = barostat.momentum
                if barostat.chain is not None:
                    _check_chain(barostat.chain, device, "barostat.chain")
                    box_q, box_p = barostat.chain[0], barostat.chain[1]
            self._engine.set_barostat(
                temperature=ensemble["temperature"], pressure=ensemble["pressure"],
                timescale=ensemble["barostat_timescale"], momentum=momentum,
                positions=box_q, momenta=box_p,
            )
        self._failure: str | None = None
        self._graphs = self._capture()

    # -- public ------------------------------------------------------------------------------

    def run(
        self,
        steps: Integral,
        *,
        sample_every: Integral | None = None,
        echo: bool | TextIO = False,
        sample_file=None,
    ) -> dict[str, Tensor] | None:
        """Advance ``steps`` steps.

        With ``sample_every``, returns the panel at each step that is a multiple of it, as host
        tensors [S] under the names of the fields and ``step`` [S] int64; otherwise None.
        ``echo`` (True for stdout, or a text stream) prints a header and one row per sample.
        ``sample_file`` names an HDF5 file, overwritten, holding each sample's frame and panel
        (``read_sample_file``; h5py is needed only then). Syncs with the host every 1,000
        steps, at each sample and at the end. Raises ``ValueError`` for settings out of range
        and when the status reports a failure (which fails the simulation; the file keeps the
        samples written before it); ``RuntimeError`` after a failure.
        """
        steps = _count("steps", steps)
        if sample_every is not None and _count("sample_every", sample_every) == 0:
            raise ValueError("sample_every must be positive")
        if echo is not False and echo is not True and not hasattr(echo, "write"):
            raise ValueError("echo must be True, False or a text stream")
        if (echo is not False or sample_file is not None) and sample_every is None:
            raise ValueError("echo and sample_file need sample_every")
        self._require()
        start = self._step
        due: list[int] = []
        if sample_every is not None:
            first = (start // sample_every + 1) * sample_every
            due = list(range(first, start + steps + 1, sample_every))
        stream = echo if hasattr(echo, "write") else (sys.stdout if echo else None)
        if stream is not None:
            stream.write("".join(f"{name:>20}" for name in ("step", "time", *self._fields)) + "\n")
        rows = []
        writer = None
        if sample_file is not None:
            writer = SampleWriter(
                sample_file, masses=self._masses.cpu().numpy(), fields=self._fields,
                attributes={**self._settings, "timestep": self._timestep,
                            "cutoff": self._model.cutoff})
        try:
            self._run_stops(start, steps, due, rows, stream, writer)
        finally:
            if writer is not None:
                writer.close()
        self._step = start + steps
        if sample_every is None:
            return None
        table = torch.tensor(rows, dtype=torch.float64).reshape(len(due), len(self._fields))
        samples = {"step": torch.tensor(due, dtype=torch.int64)}
        samples.update(
            {name: table[:, k].to(self._model.dtype) for k, name in enumerate(self._fields)}
        )
        return samples

    def _run_stops(self, start: int, steps: int, due: list[int], rows: list, stream,
                   writer) -> None:
        """The steps of ``run`` between its stops: samples, status reads, the end."""
        # Stops: samples, status reads every 1,000 steps and the end.
        stops = sorted(
            set(due)
            | set(range(start + _STATUS_INTERVAL, start + steps, _STATUS_INTERVAL))
            | ({start + steps} if steps else set())
        )
        position = start
        for stop in stops:
            self._advance(stop - position)
            position = stop
            self._step = position
            if stop in due:
                values = self._panel_values()
                rows.append(values)
                if stream is not None or writer is not None:
                    self._check(stop)  # no sample of a failed run is echoed or written
                if stream is not None:
                    stream.write(
                        "".join(f"{v:>20.6g}" for v in (stop, stop * self._timestep, *values))
                        + "\n",
                    )
                if writer is not None:
                    state = self.state()
                    frame = {name: getattr(state, name).cpu().numpy() for name in FRAME}
                    writer.write(stop, stop * self._timestep, frame, values)
            if (stop - start) % _STATUS_INTERVAL == 0 or stop == start + steps:
                self._check(stop)

    @property
    def model(self) -> Potential:
        return self._model

    @property
    def settings(self) -> dict:
        return dict(self._settings)

    @property
    def masses(self) -> Tensor:
        return self._masses.clone()

    @property
    def _rebuild_count(self) -> int:
        """Builds of the neighbor list since the first frame, counting its own. Syncs."""
        return self._engine.rebuild_count

    def sample(self) -> dict[str, float]:
        """The current frame's panel under the field names. Syncs with the host."""
        self._require()
        return dict(zip(self._fields, self._panel_values()))

    def state(self) -> State:
        """A copy of the current frame as a ``State``. Raises ``RuntimeError`` after a failure."""
        self._require()
        frame = self._engine.export(self._thermostat)
        thermostat = None
        if self._thermostat:
            th = self._engine.thermostat
            thermostat = ChainState(
                th[CHAIN_A:CHAIN_A + 3].clone(), th[CHAIN_A + 3:CHAIN_A + 6].clone(),
            )
        barostat = None
        cell = self._cell.clone()
        if self._mode == 2:
            box = self._engine.barostat
            barostat = BarostatState(box[0].clone(), ChainState(box[1:4].clone(),
                                                                box[4:7].clone()))
            cell = frame["cell"]
        return State(
            frame["positions"],
            frame["velocities"],
            frame["forces"],
            cell,
            frame["images"],
            self._step,
            thermostat,
            barostat,
        )

    def set_frame(self, positions: Tensor, velocities: Tensor, *, images: Tensor | None = None,
                  step: Integral | None = None) -> None:
        """Replace the frame of this simulation, keeping its model, ensemble and graphs.

        An extension of the reference's API for callers that stream frames through one
        simulation (a resume without a new capture): positions [N, 3] (anywhere) and velocities
        [N, 3] in the model's dtype and device; the thermostat chain is kept. No host sync; a
        frame that needs a larger neighbor capacity fails at the next status read.
        """
        self._require()
        model = self._model
        _check_frame(model, positions, velocities, self._masses, self._cell)
        if images is None:
            images = torch.zeros((model.num_atoms, 3), dtype=torch.int64, device=model.device)
        wrapped, crossings = space.wrap(positions.detach(), self._cell)
        types = _kernel_types(model)
        self._engine.reload(wrapped, velocities.detach(), self._masses, images + crossings, types)
        if self._thermostat:
            self._engine.thermostat[PENDING_SCALE] = 1.0
        if step is not None:
            self._step = _count("step", step)

    # -- internals ---------------------------------------------------------------------------

    def _capture(self) -> dict[int, torch.cuda.CUDAGraph]:
        """Warm up, then capture graphs of 1 and ``_CHUNK`` steps; the state is restored after."""
        engine = self._engine
        saved = engine.snapshot()
        current = torch.cuda.current_stream(engine.device)
        side = torch.cuda.Stream(engine.device)
        side.wait_stream(current)
        with torch.cuda.stream(side):
            for _ in range(3):
                engine.step(self._mode)
        current.wait_stream(side)
        self._check(self._step + 3)  # a first frame that fails in the warm-up
        graphs = {}
        if isinstance(engine, Engine) and not engine.small:
            # On the grid path the LJ engine builds its own graphs, each step's nine rebuild
            # kernels behind a conditional node set from the device flag (on the small-box
            # path the three gated launches cost less than the node); the build only reads
            # the state.
            engine.restore(saved)
            torch.cuda.synchronize(engine.device)
            for length in (1, _CHUNK):
                graphs[length] = engine.make_graph(self._thermostat, length)
            return graphs
        for length in (1, _CHUNK):
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                for _ in range(length):
                    engine.step(self._mode)
            graphs[length] = graph
        engine.restore(saved)
        torch.cuda.synchronize(engine.device)
        return graphs

    def _advance(self, steps: int) -> None:
        engine = self._engine
        if isinstance(engine, Engine) and engine.runs_in_one_launch:
            # A small box runs whole stretches of steps in one launch; its step is a few
            # microseconds of work, which per-step launches would bound.
            engine.run_steps(self._thermostat, steps)
            return
        chunks, rest = divmod(steps, _CHUNK)
        for _ in range(chunks):
            self._graphs[_CHUNK].replay()
        for _ in range(rest):
            self._graphs[1].replay()

    def _panel_values(self) -> list[float]:
        """E, K, E + K, T, P (and the conserved energy): one force pass with the virial."""
        engine = self._engine
        engine.forces(virial=True)
        engine.kinetic(self._thermostat)
        totals = engine.totals.tolist()
        energy, kinetic = totals[0], totals[9]
        w_trace = totals[2] + totals[3] + totals[4]
        volume = engine.volume()
        values = [
            energy,
            kinetic,
            energy + kinetic,
            2.0 * kinetic / (self._degrees_of_freedom * BOLTZMANN),
            (2.0 * kinetic + w_trace) / (3.0 * volume),
        ]
        if self._thermostat:
            th = engine.thermostat.tolist()
            q, p = th[CHAIN_A:CHAIN_A + 3], th[CHAIN_A + 3:CHAIN_A + 6]
            mass = th[CHAIN_MASS:CHAIN_MASS + 3]
            kT, degrees = th[THERMAL_ENERGY], th[DEGREES]
            bath = sum(pk * pk / (2.0 * mk) for pk, mk in zip(p, mass))
            bath += degrees * kT * q[0] + kT * (q[1] + q[2])
            if self._mode == 2:
                # The barostat's chain (one degree of freedom), P V and the box's kinetic energy
                # (src/nabladyn/md/_ensembles/_npt.py:196-221).
                box = engine.barostat.tolist()
                box_q, box_p, box_mass = box[1:4], box[4:7], box[7:10]
                bath += sum(pk * pk / (2.0 * mk) for pk, mk in zip(box_p, box_mass))
                bath += kT * (box_q[0] + box_q[1] + box_q[2])
                bath += box[11] * volume + box[0] * box[0] / (2.0 * box[10])
                values.append(volume)
            values.append(energy + kinetic + bath)
        # Values in the model's dtype, as the reference's panel row.
        return torch.tensor(values, dtype=torch.float64).to(self._model.dtype).tolist()

    def _check(self, step: int) -> None:
        failure = self._engine.failure()
        if failure is not None:
            self._failure = f"by step {step}: {failure}"
            raise ValueError(f"the simulation failed {self._failure}")

    def _require(self) -> None:
        if self._failure is not None:
            raise RuntimeError(
                f"the simulation failed {self._failure}; start a new one from an earlier state()",
            )


def _check_thermostat_settings(temperature, thermostat_timescale) -> None:
    for name, value in (("temperature", temperature),
                        ("thermostat_timescale", thermostat_timescale)):
        if isinstance(value, bool) or not isinstance(value, Real) or not math.isfinite(value) or value <= 0:
            raise ValueError(f"{name} must be a finite positive number")


def nve(model, positions, velocities, masses, cell, *, timestep, skin=0.1,
        capacity_multiplier=1.25, images=None, step=0) -> Simulation:
    """Build a simulation at constant energy, by velocity Verlet.

    The arguments of src/nabladyn/md/_ensembles/_nve.py:70-107: positions [N, 3] in nm (may
    lie outside the cell), velocities [N, 3] in nm/ps, masses [N] in Da, cell [3] in nm, all in
    the model's dtype and on its device; ``timestep`` in ps; the list's ``skin`` and
    ``capacity_multiplier``; ``images`` and ``step`` to continue a run. The center-of-mass
    velocity is removed first. Syncs with the host.
    """
    return Simulation(model, positions, velocities, masses, cell, ensemble={"name": "NVE"},
                      timestep=timestep, skin=skin, capacity_multiplier=capacity_multiplier,
                      images=images, step=step)


def nvt(model, positions, velocities, masses, cell, *, timestep, temperature,
        thermostat_timescale, skin=0.1, capacity_multiplier=1.25, images=None, step=0,
        thermostat: ChainState | None = None) -> Simulation:
    """Build a simulation at constant temperature: velocity Verlet between Nose-Hoover halves.

    Takes ``nve``'s arguments plus ``temperature`` in K, ``thermostat_timescale`` tau in ps and,
    to continue a run, the ``thermostat`` chain (float64). The chain of three has masses
    g kT tau^2, kT tau^2, kT tau^2 with g = 3N - 3 (src/nabladyn/md/_ensembles/_nvt.py:132-179).
    """
    _check_thermostat_settings(temperature, thermostat_timescale)
    return Simulation(
        model, positions, velocities, masses, cell,
        ensemble={
            "name": "NVT",
            "temperature": float(temperature),
            "thermostat_timescale": float(thermostat_timescale),
            "chain": thermostat,
        },
        timestep=timestep, skin=skin, capacity_multiplier=capacity_multiplier, images=images,
        step=step,
    )


def npt(model, positions, velocities, masses, cell, *, timestep, temperature, pressure,
        thermostat_timescale, barostat_timescale, skin=0.1, capacity_multiplier=1.25,
        images=None, step=0, thermostat: ChainState | None = None,
        barostat: BarostatState | None = None) -> Simulation:
    """Build a simulation at constant pressure and temperature, by isotropic MTK.

    Takes ``nvt``'s arguments plus ``pressure`` in kJ/mol/nm^3 (``units.BAR`` converts),
    ``barostat_timescale`` tau_b in ps and, to continue a run, the ``barostat`` state (box
    momentum [] float64 and its chain). Chains of three act on the particles and on the
    barostat; the box mass is 3 (N + 1) kT tau_b^2; the cell keeps its aspect ratio and scales
    about the origin (src/nabladyn/md/_ensembles/_npt.py:66-311). The panel adds ``volume`` and
    ``conserved_energy`` (U + K + PV + the box's kinetic energy + both chains' energies). Runs
    in the pair engine for every model (the cell changes every step).
    """
    _check_thermostat_settings(temperature, thermostat_timescale)
    if (isinstance(barostat_timescale, bool) or not isinstance(barostat_timescale, Real)
            or not math.isfinite(barostat_timescale) or barostat_timescale <= 0):
        raise ValueError("barostat_timescale must be a finite positive number")
    if isinstance(pressure, bool) or not isinstance(pressure, Real) or not math.isfinite(pressure):
        raise ValueError("pressure must be a finite number")
    return Simulation(
        model, positions, velocities, masses, cell,
        ensemble={
            "name": "NPT",
            "temperature": float(temperature),
            "pressure": float(pressure),
            "thermostat_timescale": float(thermostat_timescale),
            "barostat_timescale": float(barostat_timescale),
            "chain": thermostat,
            "barostat": barostat,
        },
        timestep=timestep, skin=skin, capacity_multiplier=capacity_multiplier, images=images,
        step=step,
    )


__all__ = ("FIELDS", "Simulation", "nve", "nvt", "npt")
