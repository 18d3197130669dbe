"""Our neighbor operator against the reference's own CUDA operator on the same B200.

The reference (installed in baseline/_ref, built from its sources for sm_100a) runs in a
separate process (tests/reference_pairs.py); the pair sets must be equal as sorted sets, bit
for bit, for allocate and for updates that reuse and that rebuild, on both build paths and in
float32 and float64. The designed frames (tests/boundary_frames.py) hold pairs at the list
radius whose listing depends on how r^2 is rounded: equal sets there show that the kernels'
rounding of r^2 is the reference's. Skipped when baseline/_ref holds no reference build.
"""

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

import boundary_frames as bf
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


def reference_operator(tmp_path, frames, cell, dtype: str):
    inputs, outputs = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(inputs, positions=frames, cell=cell, cutoff=1.0, skin=0.1, dtype=dtype)
    subprocess.run([sys.executable, str(ROOT / "tests" / "reference_pairs.py"), str(inputs),
                    str(outputs)], check=True, timeout=600)
    return np.load(outputs)


def our_operator(frames, cell, dtype: str):
    """Per frame: the pair keys, the rebuild count and the capacity."""
    device = torch.device("cuda", 0)
    torch_dtype = getattr(torch, dtype)
    box = torch.tensor(cell, dtype=torch_dtype, device=device)
    neighbor_list = NeighborList(1.0, skin=0.1)
    out = []
    for k in range(frames.shape[0]):
        x = torch.tensor(frames[k], dtype=torch_dtype, device=device)
        if k == 0:
            neighbor_list.allocate(x, box)
        else:
            neighbor_list.update(x, box)
        total = neighbor_list.num_pairs
        index = neighbor_list.tensors().index[:, :total].cpu().numpy()
        out.append((on.pair_set(index[0], index[1]), neighbor_list._rebuild_count,
                    neighbor_list.pair_capacity))
    return out


@pytest.mark.parametrize("case", ["all_pairs", "grid", "slab"])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_pairs_equal_reference_operator(tmp_path, case, dtype):
    frames, cell = frames_for(case, np.dtype(dtype))
    reference = reference_operator(tmp_path, frames, cell, dtype)
    for k, (keys, rebuilds, capacity) in enumerate(our_operator(frames, cell, dtype)):
        want = reference[f"pairs_{k}"]
        assert rebuilds == int(reference[f"rebuilds_{k}"])
        assert capacity == int(reference[f"capacity_{k}"])
        np.testing.assert_array_equal(keys, on.pair_set(want[0], want[1]))


@pytest.mark.parametrize("length, path", [(6.0, "grid"), (3.2, "all")])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_rounding_of_r2_equals_reference_operator(tmp_path, length, path, dtype):
    """Pairs within 0.6 ulp of the squared list radius: the reference operator, ours and the
    oracle list the same ones, and on these frames the candidate roundings of r^2 disagree."""
    positions, cell, first, second = bf.designed_frame(length, 1200 if path == "grid" else 300,
                                                       1.1, dtype, seed=3)
    decisions = {name: bf.listed_under(name, positions, first, second, 1.1) for name in bf.ORDERS}
    for name, listed in decisions.items():  # the frame tells the orders apart
        assert name == bf.PINNED or (listed != decisions[bf.PINNED]).sum() >= 10
    reference = reference_operator(tmp_path, positions[None], cell, dtype)
    want = reference["pairs_0"]
    want_keys = on.pair_set(want[0], want[1])
    keys, _, capacity = our_operator(positions[None], cell, dtype)[0]
    a, b, oracle_path = on.pairs(positions, cell, 1.1)
    assert oracle_path == path
    reference_listed = bf.designed_listed(want_keys, first, second)
    ours_listed = bf.designed_listed(keys, first, second)
    assert np.array_equal(keys, want_keys), (
        f"reference rounds r^2 as {bf.matching_orders(reference_listed, positions, first, second, 1.1)}, "
        f"ours as {bf.matching_orders(ours_listed, positions, first, second, 1.1)}")
    assert capacity == int(reference["capacity_0"])
    np.testing.assert_array_equal(keys, on.pair_set(a, b))
    assert bf.matching_orders(reference_listed, positions, first, second, 1.1) == [bf.PINNED]
