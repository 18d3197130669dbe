"""Generate the golden fixtures of tests/golden from the reference itself, on CPU.

Run in a container where the reference is mounted (default /root/reference; override with
NABLADYN_REFERENCE): ``python tests/golden/make_golden.py``. It imports the reference's Python
package and evaluates its own code on CPU tensors; the GPU box never runs this script, it only
reads the .npz files written here.

Fixtures:
* argon_512.npz — the reference's example frame (examples/data/argon_512.npz) with the
  reference's E/F/W in float64 and float32 over every pair (i < j; the model masks by the
  cutoff, so no neighbor list is involved) and the documented known answers
  (examples/README.md:55-56): 29,014 pairs within 1.1 nm, 21,398 within 1.0 nm, capacity
  36,268, E = -2,526.17 kJ/mol, max |F| = 386.06 kJ/mol/nm.
* argon_512_md.npz — 20 NVE, 20 NVT and 20 NPT (50 bar, barostat timescale 0.5 ps) steps of
  that frame, float64 and float32, made by the reference's own ensemble halves (src/nabladyn/md/_ensembles/_nve.py, _nvt.py, _chain.py) in
  the order Simulation._capture runs them (src/nabladyn/md/_simulation.py:331-348), with the
  all-pairs index standing in for the neighbor list.
* lj_frames_4.npz — four frames of examples/data/lj_frames.npz (216 atoms, two types) with the
  file's labels and the reference's float64 E/F/W for the generating rows.
* lj_fit_gradient.npz — the reference's loss and its gradient in sigma and epsilon on those
  frames, from perturbed parameters (its training predict/loss under torch.func).
* schnet_343.npz — 343 coarse-grained beads (7^3 simple-cubic sites at 10 per nm^3, 0.02 nm
  seeded jitter, two seeded types), the reference's SchNet (64 features, 3 blocks, 50
  Gaussians, cutoff 1.2 nm, seed 0) built in float64 and float32, its E/F/W over every pair
  by quantity.energy_force_virial, and its seeded weights (also for one type, the bead
  workload's topology) under its state-dict names.
* sum_343.npz — the reference's potential.sum of a two-type Lennard-Jones (cutoff 1.0 nm) and
  its SchNet (cutoff 1.2 nm, seed 0) on the schnet_343 frame, float64 E/F/W over every pair.
* schnet_fit_gradient.npz — the reference's SchNet training loss over E/F/W on three frames of
  that system (labels from the seed-1 network) and its gradient in four of the seed-0
  network's parameters, by its training predict/loss under torch.func.
* observables.npz — the reference's kinetic_energy, temperature and pressure
  (src/nabladyn/observables.py:18-41) on seeded float64 velocities, masses, virials and cells.

``python tests/golden/make_golden.py observables schnet`` writes only the fixtures named.
"""

import os
import sys
from pathlib import Path

import numpy as np
import torch

REFERENCE = Path(os.environ.get("NABLADYN_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(REFERENCE / "src"))

from nabladyn import potential, quantity, space  # noqa: E402
from nabladyn.md._ensembles._nve import NVE  # noqa: E402
from nabladyn.md._ensembles._npt import NPT  # noqa: E402
from nabladyn.md._ensembles._nvt import NVT  # noqa: E402
from nabladyn.md._state import _Frame  # noqa: E402
from nabladyn.neighbors import NeighborPairs  # noqa: E402
from nabladyn import observables as reference_observables  # noqa: E402
from nabladyn.observables import kinetic_energy  # noqa: E402

SIGMA, EPSILON, MASS, CUTOFF = 0.34, 0.996, 39.948, 1.0
NPT_PRESSURE = 50 * 0.0602214076  # 50 bar in kJ/mol/nm^3


def all_pairs(n: int) -> torch.Tensor:
    i, j = torch.triu_indices(n, n, offset=1)
    return torch.stack([i, j]).to(torch.int32)


def argon_model(n: int, dtype):
    return potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64),
        sigma=torch.tensor([SIGMA], dtype=dtype),
        epsilon=torch.tensor([EPSILON], dtype=dtype),
        cutoff=CUTOFF,
    )


def argon() -> None:
    frame = np.load(REFERENCE / "examples" / "data" / "argon_512.npz")
    out = {name: frame[name] for name in frame.files}
    n = frame["positions"].shape[0]
    index = all_pairs(n)
    for dtype, tag in ((torch.float64, "f64"), (torch.float32, "f32")):
        positions = torch.tensor(frame["positions"], dtype=dtype)
        cell = torch.tensor(frame["cell"], dtype=dtype)
        model = argon_model(n, dtype)
        pairs = NeighborPairs(index, n, CUTOFF)
        energy, forces, virial = quantity.energy_force_virial(model)(positions, cell, pairs)
        out[f"energy_{tag}"] = energy.detach().numpy()
        out[f"forces_{tag}"] = forces.detach().numpy()
        out[f"virial_{tag}"] = virial.detach().numpy()
    # Counts by float64 distance, the documented known answers.
    positions = torch.tensor(frame["positions"], dtype=torch.float64)
    cell = torch.tensor(frame["cell"], dtype=torch.float64)
    wrapped, _ = space.wrap(positions, cell)
    r = space._displacement_wrapped(wrapped[index[0].long()], wrapped[index[1].long()], cell).norm(dim=-1)
    out["pairs_within_1_1"] = np.int64((r < 1.1).sum())
    out["pairs_within_1_0"] = np.int64((r < 1.0).sum())
    out["documented"] = np.array([29014, 21398, 36268, -2526.17, 386.06])
    np.savez_compressed(OUT / "argon_512.npz", **out)


def trajectory(dtype, ensemble_name: str, steps: int, record=(1, 5, 20)):
    frame_data = np.load(REFERENCE / "examples" / "data" / "argon_512.npz")
    n = frame_data["positions"].shape[0]
    positions = torch.tensor(frame_data["positions"], dtype=dtype)
    velocities = torch.tensor(frame_data["velocities"], dtype=dtype)
    cell = torch.tensor(frame_data["cell"], dtype=dtype)
    masses = torch.full((n,), MASS, dtype=dtype)
    model = argon_model(n, dtype)
    pairs = NeighborPairs(all_pairs(n), n, CUTOFF)
    # Simulation.__init__ (src/nabladyn/md/_simulation.py:171-192).
    positions, crossings = space.wrap(positions, cell)
    velocities = velocities - (masses[:, None] * velocities).sum(dim=0) / masses.sum()
    evaluate = quantity.energy_force_virial(model._energy_wrapped)
    with torch.no_grad():
        energy, forces, virial = evaluate(positions, cell, pairs)
    frame = _Frame(positions, velocities.clone(), forces, energy, virial, cell, crossings)
    start = {"positions": positions.numpy().copy(), "velocities": velocities.numpy().copy(),
             "energy": energy.detach().numpy().copy()}
    if ensemble_name == "NVE":
        ensemble = NVE(0.004, masses, frame)
    elif ensemble_name == "NVT":
        ensemble = NVT(0.004, masses, frame, temperature=120.0, timescale=0.1, chain=None)
    else:
        ensemble = NPT(0.004, masses, frame, temperature=120.0, pressure=NPT_PRESSURE,
                       thermostat_timescale=0.1, barostat_timescale=0.5, thermostat=None,
                       barostat=None)
    step_eval = quantity.energy_force_virial(model._energy_wrapped)
    records = {}
    with torch.no_grad():
        for step in range(1, steps + 1):
            ensemble.first_half(frame)
            energy, forces, virial = step_eval(frame.positions, frame.cell, pairs)
            frame.energy.copy_(energy)
            frame.forces.copy_(forces)
            frame.virial.copy_(virial)
            ensemble.second_half(frame)
            if ensemble.closing is not None:
                ensemble.closing(frame)
            if step in record:
                entry = {
                    "positions": frame.positions.numpy().copy(),
                    "velocities": frame.velocities.numpy().copy(),
                    "forces": frame.forces.numpy().copy(),
                    "images": frame.images.numpy().copy(),
                    "energy": frame.energy.numpy().copy(),
                    "kinetic": kinetic_energy(frame.velocities, masses).double().numpy().copy(),
                }
                if ensemble_name in ("NVT", "NPT"):
                    entry["chain_positions"] = ensemble._positions.numpy().copy()
                    entry["chain_momenta"] = ensemble._momenta.numpy().copy()
                if ensemble_name == "NPT":
                    entry["cell"] = frame.cell.numpy().copy()
                    entry["box_momentum"] = ensemble._box_momentum.numpy().copy()
                    entry["box_chain_positions"] = ensemble._box_positions.numpy().copy()
                    entry["box_chain_momenta"] = ensemble._box_momenta.numpy().copy()
                records[step] = entry
    return start, records


def md() -> None:
    out = {}
    for dtype, tag in ((torch.float64, "f64"), (torch.float32, "f32")):
        for name in ("NVE", "NVT", "NPT"):
            start, records = trajectory(dtype, name, 20)
            out[f"{name}_{tag}_start_positions"] = start["positions"]
            out[f"{name}_{tag}_start_velocities"] = start["velocities"]
            for step, entry in records.items():
                for key, value in entry.items():
                    out[f"{name}_{tag}_{step}_{key}"] = value
    np.savez_compressed(OUT / "argon_512_md.npz", **out)


def lj_frames() -> None:
    data = np.load(REFERENCE / "examples" / "data" / "lj_frames.npz")
    chosen = [0, 99, 150, 299]
    out = {
        "positions": data["positions"][chosen],
        "cells": data["cells"][chosen],
        "energy": data["energy"][chosen],
        "forces": data["forces"][chosen],
        "virial": data["virial"][chosen],
        "atom_types": data["atom_types"],
        "sigma": data["sigma"],
        "epsilon": data["epsilon"],
        "cutoff": data["cutoff"],
    }
    n = data["atom_types"].shape[0]
    model = potential.lennard_jones(
        atom_types=torch.tensor(data["atom_types"]),
        sigma=torch.tensor(data["sigma"]),
        epsilon=torch.tensor(data["epsilon"]),
        cutoff=float(data["cutoff"]),
    )
    pairs = NeighborPairs(all_pairs(n), n, float(data["cutoff"]))
    energies, forces, virials = [], [], []
    for k in range(len(chosen)):
        e, f, w = quantity.energy_force_virial(model)(
            torch.tensor(out["positions"][k]), torch.tensor(out["cells"][k]), pairs,
        )
        energies.append(e.detach().numpy())
        forces.append(f.detach().numpy())
        virials.append(w.detach().numpy())
    out["reference_energy"] = np.array(energies)
    out["reference_forces"] = np.array(forces)
    out["reference_virial"] = np.array(virials)
    np.savez_compressed(OUT / "lj_frames_4.npz", **out)


def lj_fit_gradient() -> None:
    """The reference's own loss and dLoss/d(sigma, epsilon) on the four lj_frames frames, by
    its predict/loss under torch.func (src/nabladyn/training/_loss.py, _fit.py:245-271),
    from parameters perturbed off the generating rows; the all-pairs index as every stack."""
    from nabladyn.training import _loss

    data = np.load(OUT / "lj_frames_4.npz")
    n = data["atom_types"].shape[0]
    sigma0, epsilon0 = data["sigma"], data["epsilon"]
    sigma = sigma0 * np.array([1.05, 0.97, 1.02])
    epsilon = epsilon0 * np.array([0.9, 1.1, 0.95])
    model = potential.lennard_jones(
        atom_types=torch.tensor(data["atom_types"]),
        sigma=torch.tensor(sigma), epsilon=torch.tensor(epsilon),
        cutoff=float(data["cutoff"]), trainable=("sigma", "epsilon"),
    )
    frames = data["positions"].shape[0]
    positions = torch.tensor(data["positions"])
    cells = torch.tensor(data["cells"])
    stack = all_pairs(n)[None].expand(frames, 2, -1).contiguous()
    labels = {"energy": torch.tensor(data["energy"]), "forces": torch.tensor(data["forces"]),
              "virial": torch.tensor(data["virial"])}
    channels = ("energy", "forces", "virial")
    scales = _loss.scales(**labels)
    weights = {"energy": 1.0, "forces": 1.0, "virial": 1.0}

    def loss(trained):
        predicted = _loss.predict(model, trained, positions, cells, (stack,), channels)
        return _loss.loss(predicted, labels, weights, scales)

    params = {"sigma": model.sigma.detach().clone(), "epsilon": model.epsilon.detach().clone()}
    gradient, (value, terms) = torch.func.grad_and_value(loss, has_aux=True)(params)
    np.savez_compressed(
        OUT / "lj_fit_gradient.npz",
        sigma=sigma, epsilon=epsilon, loss=value.detach().numpy(),
        sigma_grad=gradient["sigma"].numpy(), epsilon_grad=gradient["epsilon"].numpy(),
        scales=np.array([scales["energy"], scales["forces"], scales["virial"]]),
    )


def schnet() -> None:
    n_side, density, cutoff = 7, 10.0, 1.2
    n = n_side**3
    length = (n / density) ** (1.0 / 3.0)
    rng = np.random.default_rng(343)
    grid = np.stack(np.meshgrid(*(np.arange(n_side),) * 3, indexing="ij"), axis=-1).reshape(-1, 3)
    positions = ((grid + 0.5) * (length / n_side) + rng.normal(0.0, 0.02, (n, 3))) % length
    types = rng.permutation(np.arange(n) % 2)
    cell = np.full(3, length)
    # int64 columns: torch 2.11's CPU scatter_add takes no int32 index (the reference pins
    # torch 2.13); the pair set is the same.
    pairs = NeighborPairs(all_pairs(n).long(), n, cutoff)
    out = {"positions": positions, "cell": cell, "atom_types": types, "cutoff": cutoff}
    for dtype, tag in ((torch.float64, "64"), (torch.float32, "32")):
        model = potential.schnet(atom_types=torch.tensor(types), num_types=2, cutoff=cutoff,
                                 dtype=dtype)
        e, f, w = quantity.energy_force_virial(model)(
            torch.tensor(positions, dtype=dtype), torch.tensor(cell, dtype=dtype), pairs,
        )
        out[f"energy{tag}"] = e.detach().numpy()
        out[f"forces{tag}"] = f.detach().numpy()
        out[f"virial{tag}"] = w.detach().numpy()
        if dtype == torch.float64:
            for name, value in model.state_dict().items():
                out[f"weight:{name}"] = value.numpy()
    one_type = potential.schnet(atom_types=torch.zeros(4, dtype=torch.int64), num_types=1,
                                cutoff=cutoff, dtype=torch.float64)
    for name in ("embedding", "blocks.0.atoms.weight", "readout2.weight"):
        out[f"weight1:{name}"] = one_type.state_dict()[name].numpy()
    np.savez_compressed(OUT / "schnet_343.npz", **out)


SUM_SIGMA, SUM_EPSILON = [0.30, 0.32, 0.34], [0.5, 0.6, 0.7]


def sum_of_models() -> None:
    g = np.load(OUT / "schnet_343.npz")
    n = g["positions"].shape[0]
    types = torch.tensor(g["atom_types"])
    lj = potential.lennard_jones(atom_types=types,
                                 sigma=torch.tensor(SUM_SIGMA, dtype=torch.float64),
                                 epsilon=torch.tensor(SUM_EPSILON, dtype=torch.float64),
                                 cutoff=1.0)
    net = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, dtype=torch.float64)
    model = potential.sum(lj, net)
    pairs = NeighborPairs(all_pairs(n).long(), n, 1.2)
    e, f, w = quantity.energy_force_virial(model)(torch.tensor(g["positions"]),
                                                  torch.tensor(g["cell"]), pairs)
    np.savez_compressed(OUT / "sum_343.npz", energy=e.detach().numpy(),
                        forces=f.detach().numpy(), virial=w.detach().numpy(),
                        sigma=np.array(SUM_SIGMA), epsilon=np.array(SUM_EPSILON))


def schnet_fit_gradient() -> None:
    from nabladyn.training import _loss

    g = np.load(OUT / "schnet_343.npz")
    n, cutoff = g["positions"].shape[0], 1.2
    rng = np.random.default_rng(3)
    frames = np.stack([(g["positions"] + rng.normal(0.0, 0.01, g["positions"].shape))
                       % g["cell"] for _ in range(3)])
    types = torch.tensor(g["atom_types"])
    positions = torch.tensor(frames)
    cells = torch.tensor(np.stack([g["cell"]] * 3))
    stack = all_pairs(n).long()[None].expand(3, 2, -1).contiguous()
    channels = ("energy", "forces", "virial")
    target = potential.schnet(atom_types=types, num_types=2, cutoff=cutoff, seed=1,
                              dtype=torch.float64)
    labels = _loss.predict(target, {}, positions, cells, (stack,), channels)
    labels = {k: v.detach() for k, v in labels.items()}
    model = potential.schnet(atom_types=types, num_types=2, cutoff=cutoff, trainable=True,
                             dtype=torch.float64)
    scales = _loss.scales(**labels)
    weights = {"energy": 1.0, "forces": 1.0, "virial": 1.0}
    names = ("embedding", "blocks.0.filter1.weight", "blocks.2.update2.bias", "readout1.weight")
    params = {k: v.detach().clone() for k, v in model.named_parameters()}

    def loss(trained):
        predicted = _loss.predict(model, trained, positions, cells, (stack,), channels)
        return _loss.loss(predicted, labels, weights, scales)

    gradient, (value, _) = torch.func.grad_and_value(loss, has_aux=True)(params)
    out = {"positions": frames, "cells": cells.numpy(), "loss": value.detach().numpy(),
           "scales": np.array([scales["energy"], scales["forces"], scales["virial"]])}
    for name in names:
        out[f"grad:{name}"] = gradient[name].numpy()
    for name in channels:
        out[f"label:{name}"] = labels[name].numpy()
    np.savez_compressed(OUT / "schnet_fit_gradient.npz", **out)


def observables() -> None:
    generator = torch.Generator().manual_seed(21)
    out = {}
    for case, n in enumerate((1, 7, 512)):
        velocities = torch.randn((n, 3), generator=generator, dtype=torch.float64)
        masses = 1.0 + 50.0 * torch.rand(n, generator=generator, dtype=torch.float64)
        virial = 100.0 * torch.randn((3, 3), generator=generator, dtype=torch.float64)
        cell = 1.0 + 4.0 * torch.rand(3, generator=generator, dtype=torch.float64)
        kinetic = reference_observables.kinetic_energy(velocities, masses)
        out[f"{case}:velocities"] = velocities.numpy()
        out[f"{case}:masses"] = masses.numpy()
        out[f"{case}:virial"] = virial.numpy()
        out[f"{case}:cell"] = cell.numpy()
        out[f"{case}:kinetic"] = kinetic.numpy()
        out[f"{case}:temperature"] = reference_observables.temperature(
            kinetic, max(3 * n - 3, 1)).numpy()
        out[f"{case}:pressure"] = reference_observables.pressure(kinetic, virial, cell).numpy()
    np.savez_compressed(OUT / "observables.npz", **out)


FIXTURES = {"argon": argon, "md": md, "lj_frames": lj_frames, "lj_fit_gradient": lj_fit_gradient,
            "schnet": schnet, "schnet_fit_gradient": schnet_fit_gradient,
            "sum_of_models": sum_of_models, "observables": observables}


if __name__ == "__main__":
    torch.set_num_threads(os.cpu_count() or 1)
    for name in sys.argv[1:] or FIXTURES:
        FIXTURES[name]()
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))
