"""Our neighbor operator against the reference's own CUDA operator on the same B200.

The reference (installed in baseline/_ref, built from its sources for sm_100a) runs in a
separate process (tests/reference_pairs.py); the pair sets must be equal as sorted sets, bit
for bit, for allocate and for updates that reuse and that rebuild, on both build paths and in
float32 and float64. Skipped when baseline/_ref holds no reference build.
"""

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice
from nabladyn_b200.neighbors import NeighborList
from oracle import neighbors as on

ROOT = Path(__file__).resolve().parents[1]
REFERENCE = ROOT / "baseline" / "_ref" / "nabladyn" / "neighbors"

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not any(REFERENCE.glob("_C*.so")), reason="no reference build"),
]


def frames_for(case: str, dtype):
    rng = np.random.default_rng(17)
    if case == "all_pairs":
        positions, cell = lattice.simple_cubic(8, 2.9, 0.02, seed=1)
    elif case == "grid":
        positions, cell = lattice.fcc(12, 12 * 0.5745, 0.02, seed=2)
    else:  # a slab: a short axis searched whole, minimum images
        positions, cell = lattice.random_box(1500, (8.0, 2.5, 6.0), seed=3)
    frames = [positions]
    frames.append(positions + rng.normal(0, 0.005, positions.shape))   # reuse
    frames.append(positions + rng.normal(0, 0.05, positions.shape))    # rebuild
    frames.append(frames[-1] + rng.normal(0, 0.08, positions.shape))   # rebuild
    return np.stack(frames).astype(dtype), cell.astype(dtype)


@pytest.mark.parametrize("case", ["all_pairs", "grid", "slab"])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_pairs_equal_reference_operator(tmp_path, case, dtype):
    frames, cell = frames_for(case, np.dtype(dtype))
    inputs, outputs = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(inputs, positions=frames, cell=cell, cutoff=1.0, skin=0.1, dtype=dtype)
    subprocess.run([sys.executable, str(ROOT / "tests" / "reference_pairs.py"), str(inputs),
                    str(outputs)], check=True, timeout=600)
    reference = np.load(outputs)
    device = torch.device("cuda", 0)
    torch_dtype = getattr(torch, dtype)
    box = torch.tensor(cell, dtype=torch_dtype, device=device)
    neighbor_list = NeighborList(1.0, skin=0.1)
    for k in range(frames.shape[0]):
        x = torch.tensor(frames[k], dtype=torch_dtype, device=device)
        if k == 0:
            neighbor_list.allocate(x, box)
        else:
            neighbor_list.update(x, box)
        total = neighbor_list.num_pairs
        index = neighbor_list.tensors().index[:, :total].cpu().numpy()
        want = reference[f"pairs_{k}"]
        assert neighbor_list._rebuild_count == int(reference[f"rebuilds_{k}"])
        assert neighbor_list.pair_capacity == int(reference[f"capacity_{k}"])
        np.testing.assert_array_equal(on.pair_set(index[0], index[1]),
                                      on.pair_set(want[0], want[1]))
