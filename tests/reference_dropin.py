"""Runs the reference's own, unchanged NeighborList and md.nve (installed in baseline/_ref) in a
process of its own, on the reference's CUDA operator or on this package's drop-in one.

    python tests/reference_dropin.py own|b200 <outputs.npz>

``b200`` loads nabladyn_b200/_lib/_nabladyn_neighbors_ops.so (the same torch.library schemas
over this package's kernels) and marks the reference's loader as done, which is the one
change a user makes (its _extension._load); no reference file is edited. Outputs: the pair
keys, rebuild counts and capacities of a NeighborList over three frames (allocate, an update
that reuses, one that rebuilds), and the state after 20 float64 NVE steps of md.nve.
Used by tests/test_dropin_gpu.py.
"""

import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "baseline" / "_ref"))
sys.path.insert(1, str(ROOT))


def main(mode: str, outputs: str) -> None:
    if mode == "b200":
        torch.ops.load_library(str(ROOT / "nabladyn_b200" / "_lib" / "_nabladyn_neighbors_ops.so"))
        from nabladyn.neighbors import _extension

        _extension._loaded = True  # the namespace is registered: skip the reference's .so
    from nabladyn import md, potential
    from nabladyn.neighbors import NeighborList

    from nabladyn_b200 import lattice  # seeded inputs only

    device = torch.device("cuda", 0)
    dtype = torch.float64
    positions, cell = lattice.fcc(7, 7 * 0.5745, 0.02, seed=41)  # 1,372 atoms, 3 bins per axis
    rng = np.random.default_rng(41)
    frames = [positions, positions + rng.normal(0, 0.004, positions.shape),
              positions + rng.normal(0, 0.06, positions.shape)]
    box = torch.tensor(cell, dtype=dtype, device=device)
    out = {}
    neighbor_list = NeighborList(1.0, skin=0.1)
    for k, frame in enumerate(frames):
        x = torch.tensor(frame % cell, dtype=dtype, device=device)
        if k == 0:
            neighbor_list.allocate(x, box)
        else:
            neighbor_list.update(x, box)
        index = neighbor_list.tensors().index[:, :neighbor_list.num_pairs].cpu().numpy()
        low, high = np.minimum(index[0], index[1]), np.maximum(index[0], index[1])
        out[f"keys_{k}"] = np.sort(low.astype(np.int64) * (1 << 32) + high)
        out[f"rebuilds_{k}"] = np.int64(neighbor_list._rebuild_count)
        out[f"capacity_{k}"] = np.int64(neighbor_list.pair_capacity)
    n = positions.shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([0.34], dtype=dtype, device=device),
        epsilon=torch.tensor([0.996], dtype=dtype, device=device),
        cutoff=1.0,
    )
    masses = torch.full((n,), 39.948, dtype=dtype, device=device)
    velocities = md.maxwell_boltzmann(masses, 300.0, seed=41)
    simulation = md.nve(model, torch.tensor(positions, dtype=dtype, device=device), velocities,
                        masses, box, timestep=0.004)
    simulation.run(20)
    state = simulation.state()
    out["positions"] = state.positions.cpu().numpy()
    out["velocities"] = state.velocities.cpu().numpy()
    out["images"] = state.images.cpu().numpy()
    out["md_rebuilds"] = np.int64(simulation._neighbors._rebuild_count)
    np.savez(outputs, **out)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
