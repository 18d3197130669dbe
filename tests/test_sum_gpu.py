"""potential.sum on the GPU against the reference's own sum (tests/golden/sum_343.npz: a
two-type Lennard-Jones at 1.0 nm plus its SchNet at 1.2 nm, float64 E/F/W over every pair):
float64 through torch.func to 1e-9; float32 on the fused kernels, each part on its own list
of a NeighborList with an inner list, within the SchNet BF16 bounds; and MD of the sum."""

import numpy as np
import pytest
import torch

from nabladyn_b200 import md, neighbors, potential, quantity
from nabladyn_b200.neighbors import NeighborPairs

pytestmark = pytest.mark.gpu


def build(g, s, dtype, cuda):
    types = torch.tensor(g["atom_types"], device=cuda)
    lj = potential.lennard_jones(atom_types=types,
                                 sigma=torch.tensor(s["sigma"], dtype=dtype, device=cuda),
                                 epsilon=torch.tensor(s["epsilon"], dtype=dtype, device=cuda),
                                 cutoff=1.0)
    net = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, dtype=dtype)
    return potential.sum(lj, net)


def test_sum_float64_matches_reference(cuda):
    g, s = dict(np.load("tests/golden/schnet_343.npz")), dict(np.load("tests/golden/sum_343.npz"))
    n = g["positions"].shape[0]
    model = build(g, s, torch.float64, cuda)
    first, second = np.triu_indices(n, 1)
    pairs = NeighborPairs(torch.tensor(np.stack([first, second]), dtype=torch.int32,
                                       device=cuda), n, 1.2)
    e, f, w = quantity.energy_force_virial(model)(torch.tensor(g["positions"], device=cuda),
                                                  torch.tensor(g["cell"], device=cuda), pairs)
    assert float(e) == pytest.approx(float(s["energy"]), rel=1e-10)
    np.testing.assert_allclose(f.cpu().numpy(), s["forces"], atol=1e-9)
    np.testing.assert_allclose(w.cpu().numpy(), s["virial"], atol=1e-8)


def test_sum_float32_fused_on_own_lists(cuda):
    g, s = dict(np.load("tests/golden/schnet_343.npz")), dict(np.load("tests/golden/sum_343.npz"))
    model = build(g, s, torch.float32, cuda)
    assert model._fused_kernel
    x = torch.tensor(g["positions"], dtype=torch.float32, device=cuda)
    box = torch.tensor(g["cell"], dtype=torch.float32, device=cuda)
    listing = neighbors.NeighborList(1.2, skin=0.1, inner_cutoffs=(1.0,))
    listing.allocate(x, box)
    e, f, w = quantity.energy_force_virial(model)(x, box, listing.tensors())
    n = g["positions"].shape[0]
    assert abs(float(e) - float(s["energy"])) <= 3e-3 * n
    assert np.linalg.norm(f.cpu().numpy() - s["forces"]) <= 1.5e-2 * np.linalg.norm(s["forces"])
    assert np.linalg.norm(w.cpu().numpy() - s["virial"]) <= 1e-2 * np.linalg.norm(s["virial"])


def test_sum_runs_md_with_inner_lists(cuda):
    g, s = dict(np.load("tests/golden/schnet_343.npz")), dict(np.load("tests/golden/sum_343.npz"))
    model = build(g, s, torch.float32, cuda)
    n = g["positions"].shape[0]
    masses = torch.full((n,), 32.04, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 300.0, seed=2)
    simulation = md.nvt(model, torch.tensor(g["positions"], dtype=torch.float32, device=cuda),
                        velocities, masses, torch.tensor(g["cell"], dtype=torch.float32,
                                                         device=cuda),
                        timestep=0.005, temperature=300.0, thermostat_timescale=0.1)
    engine = simulation._engine
    assert len(engine.neighbors.tensors().inner) == 1
    samples = simulation.run(200, sample_every=50)
    assert np.isfinite(samples["total_energy"].numpy()).all()
    assert 150.0 < float(samples["temperature"][-1]) < 450.0
