"""Runs the reference's own neighbor operator (installed in baseline/_ref) in a process of its
own, since it registers the same torch.library namespace as this package.

    python tests/reference_pairs.py <inputs.npz> <outputs.npz>

Inputs: ``positions`` [F, N, 3] (frame 0 allocates, the others update), ``cell`` [3],
``cutoff``, ``skin``, ``dtype`` ("float32" or "float64"). Outputs per frame k: ``pairs_k``
[2, total], ``rebuilds_k``. Used only by tests/test_reference_op_gpu.py.
"""

import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "baseline" / "_ref"))

from nabladyn.neighbors import NeighborList  # noqa: E402


def main(inputs: str, outputs: str) -> None:
    data = np.load(inputs)
    dtype = getattr(torch, str(data["dtype"]))
    device = torch.device("cuda", 0)
    cell = torch.tensor(data["cell"], dtype=dtype, device=device)
    frames = torch.tensor(data["positions"], dtype=dtype, device=device)
    neighbor_list = NeighborList(float(data["cutoff"]), skin=float(data["skin"]))
    out = {}
    for k in range(frames.shape[0]):
        if k == 0:
            neighbor_list.allocate(frames[0], cell)
        else:
            neighbor_list.update(frames[k], cell)
        total = neighbor_list.num_pairs
        out[f"pairs_{k}"] = neighbor_list.tensors().index[:, :total].cpu().numpy()
        out[f"rebuilds_{k}"] = np.int64(neighbor_list._rebuild_count)
        out[f"capacity_{k}"] = np.int64(neighbor_list.pair_capacity)
    np.savez(outputs, **out)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
