"""The 1,048,576-atom Lennard-Jones box of the headline workload (64^3-cell FCC in L = 36.77 nm)
in float32 against float64, after 30 NVE steps (positions unwrapped since the last rebuild).

Tolerances: forces ||F32 - F64|| / ||F64|| <= 1e-5, on a seeded sample of 4,096 atoms against
the float64 oracle (each atom with its complete neighbor set) and on all atoms against the
float64 kernels over the neighbor operator's pairs; energy and virial within 1e-5 relative of
the float64 kernels, which match the oracle to 1e-9 on the smaller boxes of test_lj_gpu.py.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice, md, neighbors, potential, quantity, space
from oracle import lj

pytestmark = pytest.mark.gpu


def test_large_box_float32_against_float64(cuda):
    positions, cell = lattice.large_lj()
    n = positions.shape[0]
    dtype = torch.float32
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
        sigma=torch.tensor([0.34], dtype=dtype, device=cuda),
        epsilon=torch.tensor([0.996], dtype=dtype, device=cuda),
        cutoff=1.0,
    )
    masses = torch.full((n,), 39.948, dtype=dtype, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 120.0, seed=2024)
    box = torch.tensor(cell, dtype=dtype, device=cuda)
    simulation = md.nve(model, torch.tensor(positions, dtype=dtype, device=cuda), velocities,
                        masses, box, timestep=0.004, skin=0.1)
    simulation.run(30)
    engine = simulation._engine
    assert not engine.small and engine.rebuild_count >= 2
    for _ in range(40):  # on to a frame where some atoms have left the cell since the rebuild
        x = engine.tensors["positions"][:, :3]
        if bool(((x < 0) | (x >= box)).any()):
            break
        simulation.run(1)
    panel = simulation.sample()  # forces and virial of the current frame
    x32 = engine.tensors["positions"][:, :3].clone()  # cell order, as the kernels used them
    f32 = engine.tensors["forces"].double()
    totals = engine.totals.tolist()
    w32 = np.array([[totals[2], totals[5], totals[6]],
                    [totals[5], totals[3], totals[7]],
                    [totals[6], totals[7], totals[4]]])
    assert bool(((x32 < 0) | (x32 >= box)).any())

    # All atoms: the float64 kernels on the same coordinates.
    cell64 = box.double()
    x64, _ = space.wrap(x32.double(), cell64)
    exact = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
        sigma=torch.tensor([0.34], dtype=torch.float64, device=cuda),
        epsilon=torch.tensor([0.996], dtype=torch.float64, device=cuda),
        cutoff=1.0,
    )
    listing = neighbors.NeighborList(1.0, skin=0.0)
    listing.allocate(x64, cell64)
    e64, f64, w64 = quantity.energy_force_virial(exact)(x64, cell64, listing.tensors())
    force_error = float((f32 - f64).norm() / f64.norm())
    assert force_error <= 1e-5, force_error
    assert abs(float(panel["potential_energy"]) - float(e64)) <= 1e-5 * abs(float(e64))
    w64 = w64.cpu().numpy()
    assert np.linalg.norm(w32 - w64) <= 1e-5 * np.linalg.norm(w64)

    # A seeded sample of 4,096 atoms against the float64 oracle.
    sample = np.random.default_rng(36).choice(n, 4096, replace=False)
    oracle_forces = lj.sample_forces(x32.cpu().numpy(), cell.astype(np.float32), sample,
                                     [0.34], [0.996], 1.0)
    got = f32.cpu().numpy()[sample]
    sample_error = np.linalg.norm(got - oracle_forces) / np.linalg.norm(oracle_forces)
    assert sample_error <= 1e-5, sample_error
    np.testing.assert_allclose(f64.cpu().numpy()[sample], oracle_forces, rtol=0, atol=1e-9)
