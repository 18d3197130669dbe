"""Data-parallel loss gradients on the host: two gloo ranks on the CPU (one process each,
rendezvous on 127.0.0.1) split each batch's frames, differentiate their shares and sum them by
one all-reduce; the loss and every parameter's gradient equal one process's over the whole
batch to 1e-12 relative, for an even split, an uneven one and a batch smaller than the ranks.

The model is a pure-torch pair potential defined here (harmonic springs within a cutoff), so
the generic torch.func gradient runs on CPU tensors; the split and the all-reduce do not
depend on the model.
"""

import math
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp
from torch import nn

from nabladyn_b200 import space
from nabladyn_b200.neighbors import NeighborPairs
from nabladyn_b200.potential import Potential
from nabladyn_b200.training import _fit, predict, scales

ATOMS, FRAMES, LENGTH, CUTOFF = 48, 6, 3.0, 1.1
CHANNELS = ("energy", "forces", "virial")
WEIGHTS = {"energy": 1.0, "forces": 1.0, "virial": 0.5}
BATCHES = ([0, 1, 2, 3], [5, 2, 0, 4, 1], [3])


class Springs(Potential):
    """E = sum over pairs closer than the cutoff of k (r - r0)^2."""

    def __init__(self, stiffness: float, rest: float):
        super().__init__()
        self.stiffness = nn.Parameter(torch.tensor(stiffness, dtype=torch.float64))
        self.rest = nn.Parameter(torch.tensor(rest, dtype=torch.float64))

    cutoff = property(lambda self: CUTOFF)
    num_atoms = property(lambda self: ATOMS)
    dtype = property(lambda self: torch.float64)
    device = property(lambda self: torch.device("cpu"))

    def _energy_wrapped(self, positions, cell, pairs, strain=None):
        first, second = pairs.index[0], pairs.index[1]
        d = space.strained(space._displacement_wrapped(positions[first], positions[second], cell),
                           strain)
        r = torch.sqrt((d * d).sum(-1))
        inside = (r < CUTOFF) & (first != second)
        return torch.where(inside, self.stiffness * (r - self.rest) ** 2, 0.0).sum()


def prepared_data():
    rng = np.random.default_rng(8)
    positions = torch.tensor(rng.uniform(0, LENGTH, (FRAMES, ATOMS, 3)))
    cells = torch.full((FRAMES, 3), LENGTH, dtype=torch.float64)
    first, second = np.triu_indices(ATOMS, k=1)
    stack = torch.tensor(np.stack([first, second]))[None].expand(FRAMES, 2, -1).contiguous()
    with torch.no_grad():
        labels = predict(Springs(2.0, 0.7), {}, positions, cells, (stack,), CHANNELS)
    return positions, cells, stack, labels


def gradients(process_group=None):
    model = Springs(1.6, 0.8)
    trained = dict(model.named_parameters())
    prepared = prepared_data()
    label_scales = scales(**prepared[3])
    out = []
    for batch in BATCHES:
        value, grads = _fit._gradient(model, trained, prepared, torch.tensor(batch), WEIGHTS,
                                      label_scales, CHANNELS, 2, process_group)
        out.append((float(value), {k: float(v) for k, v in grads.items()}))
    return out


def _free_port() -> int:
    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        return probe.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, queue) -> None:
    import torch.distributed as dist

    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    dist.init_process_group("gloo")
    try:
        queue.put((rank, gradients(dist.group.WORLD)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_give_the_single_process_gradient():
    want = gradients()
    world, port = 2, _free_port()
    context = mp.get_context("spawn")
    queue = context.Queue()
    processes = [context.Process(target=_rank_main, args=(r, world, port, queue))
                 for r in range(world)]
    for process in processes:
        process.start()
    results = dict(queue.get(timeout=180) for _ in range(world))
    for process in processes:
        process.join(timeout=60)
        assert process.exitcode == 0
    for rank in range(world):
        for (value, grads), (want_value, want_grads) in zip(results[rank], want):
            assert math.isclose(value, want_value, rel_tol=1e-12)
            for name, expected in want_grads.items():
                assert math.isclose(grads[name], expected, rel_tol=1e-12, abs_tol=1e-14)
