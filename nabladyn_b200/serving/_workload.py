"""The serving workload: independent argon replicas of uneven sizes with Poisson arrivals.

Sizes log-uniform in [64, 16384] atoms, densities uniform in [18, 22] per nm^3, temperatures
uniform in [90, 150] K, jittered (0.02 nm) simple-cubic starts (the first N sites of a
ceil(N^(1/3))^3 grid), cubic boxes of at least 2.2 nm (a smaller replica's density drops, as
the reference rejects L <= 2 r_c), Maxwell-Boltzmann velocities at T, all seeded.
"""

from __future__ import annotations

import math

import numpy as np

from ..units import BOLTZMANN
from ._server import ReplicaRequest


def serving_requests(count: int = 4096, *, seed: int = 7, rate: float | None = None,
                     steps: int = 500, smallest: int = 64, largest: int = 16384) -> list[ReplicaRequest]:
    """``count`` requests; ``rate`` requests per second of Poisson arrivals (None: all at 0)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(smallest), math.log(largest), count)).astype(int)
    densities = rng.uniform(18.0, 22.0, count)
    temperatures = rng.uniform(90.0, 150.0, count)
    gaps = rng.exponential(1.0 / rate, count) if rate else np.zeros(count)
    arrivals = np.cumsum(gaps)
    requests = []
    for k in range(count):
        n = int(sizes[k])
        length = max(2.2, (n / densities[k]) ** (1.0 / 3.0))
        side = math.ceil(n ** (1.0 / 3.0))
        spacing = length / side
        grid = np.stack(np.meshgrid(*(np.arange(side),) * 3, indexing="ij"), axis=-1).reshape(-1, 3)
        positions = (grid[:n] + 0.5) * spacing + rng.normal(0.0, 0.02, (n, 3))
        masses = np.full(n, 39.948)
        velocities = rng.normal(0.0, 1.0, (n, 3)) * np.sqrt(BOLTZMANN * temperatures[k] / masses)[:, None]
        requests.append(ReplicaRequest(
            positions=positions, velocities=velocities, masses=masses, cell=np.full(3, length),
            temperature=float(temperatures[k]), steps=steps, arrival=float(arrivals[k]), name=k,
        ))
    return requests


__all__ = ("serving_requests",)
