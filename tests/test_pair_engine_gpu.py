"""The pair engine (models other than Lennard-Jones through md.nve/md.nvt): its integrator
kernels against the float64 oracle, and SchNet MD on the fused tensor-core kernels.

* A float64 SchNet runs the engine's integrator with torch.func forces; 10 NVT steps from the
  reference's 343-bead frame match the oracle's velocity Verlet + Nose-Hoover chain with the
  oracle's SchNet forces to 1e-9 (positions nm, velocities nm/ps, chain positions and momenta).
* A float32 SchNet on the fused kernels: after a step its forces match the model's float32
  definition under torch.func to BF16 accuracy; a longer NVT run holds its temperature, and
  NVE from there holds its total energy.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice, md, neighbors, potential, quantity
from oracle import integrator
from oracle import schnet as oracle_schnet

pytestmark = pytest.mark.gpu

BEAD_MASS = 32.04


def test_integrator_matches_oracle_nvt_float64(cuda):
    g = dict(np.load("tests/golden/schnet_343.npz"))
    n = g["positions"].shape[0]
    model = potential.schnet(atom_types=torch.tensor(g["atom_types"], device=cuda), num_types=2,
                             cutoff=1.2, dtype=torch.float64)
    masses = torch.full((n,), BEAD_MASS, dtype=torch.float64, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 300.0, seed=5)
    cell = torch.tensor(g["cell"], device=cuda)
    simulation = md.nvt(model, torch.tensor(g["positions"], device=cuda), velocities, masses,
                        cell, timestep=0.01, temperature=300.0, thermostat_timescale=0.1)
    assert type(simulation._engine).__name__ == "PairEngine"
    simulation.run(10)
    state = simulation.state()
    weights = {k: v.detach().cpu().numpy() for k, v in model.state_dict().items()}
    first, second = np.triu_indices(n, 1)

    def evaluate(x):
        e, f, _ = oracle_schnet.energy_force_virial(x, g["cell"], first, second, g["atom_types"],
                                                    weights, 1.2, 50, 3)
        return e, f

    reference = integrator.run(g["positions"], velocities.cpu().numpy(), masses.cpu().numpy(),
                               g["cell"], None, None, None, 0.01, 10, temperature=300.0,
                               timescale=0.1, evaluate=evaluate)
    np.testing.assert_allclose(state.positions.cpu().numpy(), reference["positions"], atol=1e-9)
    np.testing.assert_allclose(state.velocities.cpu().numpy(), reference["velocities"], atol=1e-9)
    np.testing.assert_allclose(state.thermostat.positions.cpu().numpy(),
                               reference["chain_positions"], atol=1e-9)
    np.testing.assert_allclose(state.thermostat.momenta.cpu().numpy(),
                               reference["chain_momenta"], atol=1e-9)


def bead_system(cuda, n_side, seed=3):
    n = n_side**3
    positions, cell = lattice.simple_cubic(n_side, (n / 10.0) ** (1 / 3), 0.02, seed=seed)
    model = potential.schnet(atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
                             num_types=1, cutoff=1.2)
    masses = torch.full((n,), BEAD_MASS, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 300.0, seed=seed)
    return (model, torch.tensor(positions % cell, dtype=torch.float32, device=cuda),
            velocities, masses, torch.tensor(cell, dtype=torch.float32, device=cuda))


def test_fused_step_agrees_with_torch_path(cuda):
    model, x, v, m, cell = bead_system(cuda, 12)
    fused = md.nve(model, x, v, m, cell, timestep=0.01)
    assert fused._engine._fused
    fused.run(1)
    state = fused.state()
    listing = neighbors.NeighborList(1.2, skin=0.1)
    listing.allocate(state.positions, cell)
    _, forces, _ = quantity.energy_force_virial(model._energy_wrapped)(
        state.positions, cell, listing.tensors())
    relative = float((state.forces - forces).norm() / forces.norm())
    assert relative < 1.5e-2


def test_fused_nvt_holds_temperature_and_nve_energy(cuda):
    model, x, v, m, cell = bead_system(cuda, 16)
    simulation = md.nvt(model, x, v, m, cell, timestep=0.01, temperature=300.0,
                        thermostat_timescale=0.1)
    simulation.run(300)
    samples = simulation.run(200, sample_every=20)
    temperature = float(samples["temperature"].mean())
    assert abs(temperature - 300.0) < 15.0
    assert simulation._rebuild_count > 1
    state = simulation.state()
    nve = md.nve(model, state.positions, state.velocities, m, cell, timestep=0.01)
    energies = nve.run(200, sample_every=20)["total_energy"]
    kinetic = 1.5 * 4096 * 0.00831446261815324 * 300.0
    assert float(energies.max() - energies.min()) < 0.02 * kinetic
