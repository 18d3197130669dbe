"""SchNet on the B200: the fused tcgen05 kernels against the float64 oracle and the
reference's own numbers.

The filter network and the atom-wise layers take BF16 operands with FP32 accumulation, so E,
F and W carry BF16-level errors. The bounds against float64: energy 3e-3 kJ/mol per atom (the
total is a sum of per-atom terms of both signs, so a bound relative to it would be
meaningless when it nears zero), forces ||F - F64|| / ||F64|| <= 1.5e-2, virial
||W - W64|| / ||W64|| <= 1e-2. The pairs within the cutoff are counted exactly.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice, neighbors, potential, quantity
from nabladyn_b200.neighbors import NeighborPairs
from oracle import schnet as oracle

pytestmark = pytest.mark.gpu

ENERGY_PER_ATOM_TOL, FORCE_TOL, VIRIAL_TOL = 3e-3, 1.5e-2, 1e-2


def relative(ours, reference):
    return float(np.linalg.norm(np.asarray(ours) - reference) / np.linalg.norm(reference))


def test_fused_matches_reference_golden(cuda):
    g = dict(np.load("tests/golden/schnet_343.npz"))
    n = g["positions"].shape[0]
    first, second = np.triu_indices(n, 1)
    pairs = NeighborPairs(torch.tensor(np.stack([first, second]), dtype=torch.int32,
                                       device=cuda), n, 1.2)
    model = potential.schnet(atom_types=torch.tensor(g["atom_types"], device=cuda),
                             num_types=2, cutoff=1.2)
    assert model._fused_kernel
    e, f, w = quantity.energy_force_virial(model)(
        torch.tensor(g["positions"], dtype=torch.float32, device=cuda),
        torch.tensor(g["cell"], dtype=torch.float32, device=cuda), pairs)
    d = g["positions"][first] - g["positions"][second]
    d -= g["cell"] * np.round(d / g["cell"])
    assert model._status.tolist() == [int(((d * d).sum(1) < 1.44).sum()), 0, 0, 0]
    assert abs(float(e) - float(g["energy64"])) <= ENERGY_PER_ATOM_TOL * n
    assert relative(f.cpu().numpy(), g["forces64"]) <= FORCE_TOL
    assert relative(w.cpu().numpy(), g["virial64"]) <= VIRIAL_TOL


@pytest.mark.parametrize("types", [1, 3])
def test_fused_matches_oracle_on_listed_pairs(cuda, types):
    """4,096 beads at 10 per nm^3 over the neighbor list's pairs (radius 1.3 nm, skin and
    padding columns included), one and three bead types."""
    positions, cell = lattice.simple_cubic(16, (4096 / 10) ** (1 / 3), 0.02, seed=9)
    positions = positions % cell
    rng = np.random.default_rng(types)
    kinds = rng.integers(0, types, 4096)
    model = potential.schnet(atom_types=torch.tensor(kinds, device=cuda), num_types=types,
                             cutoff=1.2, seed=types)
    x = torch.tensor(positions, dtype=torch.float32, device=cuda)
    box = torch.tensor(cell, dtype=torch.float32, device=cuda)
    listing = neighbors.NeighborList(1.2, skin=0.1)
    listing.allocate(x, box)
    pairs = listing.tensors()
    e, f, w = quantity.energy_force_virial(model)(x, box, pairs)
    index = pairs.index.cpu().numpy()
    weights = {k: v.detach().double().cpu().numpy() for k, v in model.state_dict().items()}
    eo, fo, wo = oracle.energy_force_virial(positions, cell, index[0], index[1], kinds, weights,
                                            1.2, 50, 3)
    assert abs(float(e) - eo) <= ENERGY_PER_ATOM_TOL * 4096
    assert relative(f.cpu().numpy(), fo) <= FORCE_TOL
    assert relative(w.cpu().numpy(), wo) <= VIRIAL_TOL
    assert int(model._status[1]) == 0


def test_forces_sum_to_zero_and_repeat(cuda):
    """Newton's third law holds pair by pair. Messages are summed with FP32 atomics, whose
    order varies between calls; each BF16 rounding downstream can turn that into a one-ulp
    difference, so two calls agree to the BF16 accuracy bound (forces) and the energy, a sum
    over atoms, to 1e-5."""
    positions, cell = lattice.simple_cubic(12, (1728 / 10) ** (1 / 3), 0.02, seed=4)
    positions = positions % cell
    model = potential.schnet(atom_types=torch.zeros(1728, dtype=torch.int64, device=cuda),
                             num_types=1, cutoff=1.2)
    x = torch.tensor(positions, dtype=torch.float32, device=cuda)
    box = torch.tensor(cell, dtype=torch.float32, device=cuda)
    listing = neighbors.NeighborList(1.2, skin=0.1)
    listing.allocate(x, box)
    evaluate = quantity.energy_force_virial(model)
    e1, f1, w1 = evaluate(x, box, listing.tensors())
    e2, f2, w2 = evaluate(x, box, listing.tensors())
    scale = float(f1.abs().max())
    assert float(f1.double().sum(0).abs().max()) <= 1e-4 * scale * 1728 ** 0.5
    assert relative(f2.cpu().numpy(), f1.cpu().numpy()) <= FORCE_TOL
    assert abs(float(e1) - float(e2)) <= 1e-5 * abs(float(e1))
