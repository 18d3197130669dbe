"""Edge cases on the GPU against the oracle: a lone atom, pairs out of range, mostly empty
bins, atoms exactly on the cell faces, a nearly full and a partial SchNet tile, and a frame
with no pair inside the cutoff. Pair sets bit for bit; energies and forces within each
model's bounds (LJ float64 1e-9; SchNet the BF16 bounds of its tests)."""

import numpy as np
import pytest
import torch

from nabladyn_b200 import neighbors, potential, quantity, space
from nabladyn_b200.neighbors import NeighborPairs
from oracle import neighbors as on
from oracle import schnet as oracle_schnet

pytestmark = pytest.mark.gpu


def pairs_match_oracle(positions, cell, cutoff, skin, dtype, cuda):
    x = torch.tensor(positions, dtype=dtype, device=cuda)
    box = torch.tensor(cell, dtype=dtype, device=cuda)
    listing = neighbors.NeighborList(cutoff, skin=skin)
    listing.allocate(x, box)
    index = listing.tensors().index.cpu().numpy()
    total = listing.num_pairs
    wrapped = space.wrap(x, box)[0].cpu().numpy()
    first, second, _ = on.pairs(wrapped, box.cpu().numpy(), listing.radius)
    assert total == len(first)
    np.testing.assert_array_equal(on.pair_set(index[0, :total], index[1, :total]),
                                  on.pair_set(first, second))
    n = positions.shape[0]
    columns = np.arange(total, index.shape[1])
    np.testing.assert_array_equal(index[0, total:], columns % n)
    return listing, total


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_lone_atom_and_distant_pair(cuda, dtype):
    _, total = pairs_match_oracle(np.array([[1.0, 1.0, 1.0]]), np.full(3, 5.0), 1.0, 0.1,
                                  dtype, cuda)
    assert total == 0
    _, total = pairs_match_oracle(np.array([[0.5, 0.5, 0.5], [3.0, 3.0, 3.0]]),
                                  np.full(3, 6.0), 1.0, 0.1, dtype, cuda)
    assert total == 0
    # The same pair across the periodic face is within range.
    _, total = pairs_match_oracle(np.array([[0.05, 2.0, 2.0], [5.95, 2.0, 2.0]]),
                                  np.full(3, 6.0), 1.0, 0.1, dtype, cuda)
    assert total == 1


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_dilute_box_mostly_empty_bins(cuda, dtype):
    rng = np.random.default_rng(17)
    positions = rng.uniform(0.0, 20.0, (300, 3))
    pairs_match_oracle(positions, np.full(3, 20.0), 1.0, 0.1, dtype, cuda)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_atoms_on_cell_faces(cuda, dtype):
    """Coordinates exactly 0, exactly L (wraps to 0), just below L, and on bin boundaries."""
    length = 6.6
    np_dtype = np.float32 if dtype == torch.float32 else np.float64
    below = float(np.nextafter(np_dtype(length), np_dtype(0)))
    rng = np.random.default_rng(3)
    positions = rng.uniform(0.0, length, (200, 3))
    special = [0.0, length, below, length / 6, 2 * length / 6, length / 2]
    for k, value in enumerate(special):
        positions[k, k % 3] = value
        positions[k + len(special), :] = value
    pairs_match_oracle(positions, np.full(3, length), 1.0, 0.1, dtype, cuda)


def test_lj_without_pairs_in_cutoff(cuda):
    model = potential.lennard_jones(atom_types=torch.zeros(2, dtype=torch.int64, device=cuda),
                                    sigma=torch.tensor([0.34], dtype=torch.float64, device=cuda),
                                    epsilon=torch.tensor([0.996], dtype=torch.float64, device=cuda),
                                    cutoff=1.0)
    x = torch.tensor([[0.5, 0.5, 0.5], [2.0, 0.5, 0.5]], dtype=torch.float64, device=cuda)
    box = torch.full((3,), 5.0, dtype=torch.float64, device=cuda)
    listing = neighbors.NeighborList(1.0, skin=0.6)
    listing.allocate(x, box)
    assert listing.num_pairs == 1  # listed (within 1.6 nm) but beyond the cutoff
    e, f, w = quantity.energy_force_virial(model)(x, box, listing.tensors())
    assert float(e) == 0.0
    assert float(f.abs().max()) == 0.0 and float(w.abs().max()) == 0.0


@pytest.mark.parametrize("atoms", [5, 127, 129])
def test_schnet_partial_tiles(cuda, atoms):
    """Fewer pairs than one 128-row tile, and atom counts around one tile of atoms."""
    rng = np.random.default_rng(atoms)
    length = max(2.7, (atoms / 10.0) ** (1 / 3))
    positions = rng.uniform(0.0, length, (atoms, 3))
    cell = np.full(3, length)
    types = rng.integers(0, 2, atoms)
    model = potential.schnet(atom_types=torch.tensor(types, device=cuda), num_types=2,
                             cutoff=1.2)
    first, second = np.triu_indices(atoms, 1)
    pairs = NeighborPairs(torch.tensor(np.stack([first, second]), dtype=torch.int32,
                                       device=cuda), atoms, 1.2)
    x = torch.tensor(positions, dtype=torch.float32, device=cuda)
    box = torch.tensor(cell, dtype=torch.float32, device=cuda)
    e, f, w = quantity.energy_force_virial(model)(x, box, pairs)
    weights = {k: v.detach().double().cpu().numpy() for k, v in model.state_dict().items()}
    wrapped = space.wrap(x.double(), box.double())[0].cpu().numpy()
    eo, fo, wo = oracle_schnet.energy_force_virial(wrapped, cell, first, second, types, weights,
                                                   1.2, 50, 3)
    assert abs(float(e) - eo) <= 3e-3 * atoms
    scale = max(np.linalg.norm(fo), 1e-6)
    assert np.linalg.norm(f.cpu().numpy() - fo) <= 1.5e-2 * scale + 1e-4
    assert int(model._status[1]) == 0


def test_schnet_without_pairs_in_cutoff(cuda):
    """Every listed pair beyond the cutoff: no pair tile runs; E is the readout of the
    embedding alone and the forces and virial are exactly zero."""
    model = potential.schnet(atom_types=torch.zeros(3, dtype=torch.int64, device=cuda),
                             num_types=1, cutoff=1.2)
    x = torch.tensor([[0.5, 0.5, 0.5], [2.2, 0.5, 0.5], [0.5, 2.2, 0.5]], device=cuda)
    box = torch.full((3,), 6.0, device=cuda)
    pairs = NeighborPairs(torch.tensor([[0, 0, 1], [1, 2, 2]], dtype=torch.int32, device=cuda),
                          3, 1.2)
    e, f, w = quantity.energy_force_virial(model)(x, box, pairs)
    assert int(model._status[0]) == 0
    weights = {k: v.detach().double().cpu().numpy() for k, v in model.state_dict().items()}
    eo, fo, _ = oracle_schnet.energy_force_virial(x.double().cpu().numpy(), np.full(3, 6.0),
                                                  np.array([0, 0, 1]), np.array([1, 2, 2]),
                                                  np.zeros(3, int), weights, 1.2, 50, 3)
    assert abs(float(e) - eo) <= 3e-3 * 3
    assert float(f.abs().max()) == 0.0 and float(w.abs().max()) == 0.0
