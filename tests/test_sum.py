"""potential.sum on the CPU: construction rules, parameter names, list cutoffs and the choice of
each part's own list (src/nabladyn/potential/_sum/_potential.py)."""

import pytest
import torch

from nabladyn_b200 import potential
from nabladyn_b200.neighbors import NeighborPairs
from nabladyn_b200.potential._sum import own_pairs


def parts(dtype=torch.float64, n=4):
    types = torch.zeros(n, dtype=torch.int64)
    lj = potential.lennard_jones(atom_types=types, sigma=torch.tensor([0.34], dtype=dtype),
                                 epsilon=torch.tensor([0.996], dtype=dtype), cutoff=1.0)
    net = potential.schnet(atom_types=types, num_types=1, cutoff=1.2, dtype=dtype)
    return lj, net


def test_sum_rules_and_names():
    lj, net = parts()
    total = potential.sum(lj, net)
    assert total.cutoff == 1.2 and total.num_atoms == 4
    assert total._list_cutoffs == (1.0, 1.2)
    names = {name for name, _ in total.named_parameters()}
    assert "parts.0.sigma" in names and "parts.1.embedding" in names
    with pytest.raises(ValueError):
        potential.sum(lj)
    with pytest.raises(TypeError):
        potential.sum(lj, torch.nn.Linear(2, 2))
    with pytest.raises(ValueError):
        potential.sum(lj, parts(torch.float32)[1])


def test_each_part_reads_its_own_list():
    index = torch.zeros((2, 8), dtype=torch.int32)
    inner = NeighborPairs(index[:, :3], 4, 1.0)
    outer = NeighborPairs(index, 4, 1.2, (inner,))
    assert own_pairs(outer, 1.0).cutoff == 1.0 and own_pairs(outer, 1.0).inner == ()
    chosen = own_pairs(outer, 1.2)
    assert chosen.cutoff == 1.2 and chosen.inner == (inner,)
    assert own_pairs(outer, 1.1).cutoff == 1.2
