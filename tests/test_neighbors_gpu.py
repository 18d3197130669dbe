"""The neighbor operator on the GPU against the oracle: the pair set bit for bit.

Drives the kernels through NeighborList (the torch.library schema layer) and directly through
the C-ABI, and checks the pair sets, totals, padding, the reuse decision and the status bits.
"""

import ctypes
import math

import numpy as np
import pytest
import torch

from nabladyn_b200 import _native, lattice
from nabladyn_b200.neighbors import NeighborList
from oracle import neighbors as on

pytestmark = pytest.mark.gpu

DTYPES = {"f32": (torch.float32, np.float32), "f64": (torch.float64, np.float64)}


def listed(neighbor_list: NeighborList):
    index = neighbor_list.tensors().index.cpu().numpy()
    total = neighbor_list.num_pairs
    return index, total


def check_against_oracle(positions, cell, radius, torch_dtype, device, skin=0.1):
    n = positions.shape[0]
    x = torch.tensor(positions, dtype=torch_dtype, device=device)
    box = torch.tensor(cell, dtype=torch_dtype, device=device)
    neighbor_list = NeighborList(radius - skin, skin=skin)
    neighbor_list.allocate(x, box)
    index, total = listed(neighbor_list)
    wrapped = on.wrap(np.asarray(positions, dtype=x.cpu().numpy().dtype),
                      np.asarray(cell, dtype=x.cpu().numpy().dtype))
    # The device wrap is the reference's torch wrap; compare against that exact input.
    from nabladyn_b200 import space
    wrapped = space.wrap(x, box)[0].cpu().numpy()
    first, second, path = on.pairs(wrapped, box.cpu().numpy(), neighbor_list.radius)
    assert total == len(first)
    assert neighbor_list.pair_capacity == on.capacity(len(first))
    got = on.pair_set(index[0, :total], index[1, :total])
    want = on.pair_set(first, second)
    np.testing.assert_array_equal(got, want)
    # Padding: column k >= total holds (k mod N, k mod N).
    columns = np.arange(total, index.shape[1])
    np.testing.assert_array_equal(index[0, total:], columns % n)
    np.testing.assert_array_equal(index[1, total:], columns % n)
    return neighbor_list, path


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_argon_512_known_answers(argon, cuda, tag):
    torch_dtype, _ = DTYPES[tag]
    neighbor_list, path = check_against_oracle(argon["positions"], argon["cell"], 1.1,
                                               torch_dtype, cuda)
    assert path == "all"
    if tag == "f64":
        assert neighbor_list.num_pairs == 29014
        assert neighbor_list.pair_capacity == 36268


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize(
    "lengths, count, seed",
    [
        ((4.6, 4.6, 4.6), 2000, 1),
        ((7.3, 3.4, 5.1), 2600, 2),
        ((8.0, 2.5, 6.0), 1800, 3),   # a short axis: the grid path with minimum images
        ((12.0, 12.0, 12.0), 36000, 4),
    ],
)
def test_grid_path_pair_set_bit_exact(cuda, tag, lengths, count, seed):
    torch_dtype, _ = DTYPES[tag]
    positions, cell = lattice.random_box(count, lengths, seed)
    positions[::7] += np.asarray(lengths) * 1.5  # some atoms outside the cell
    _, path = check_against_oracle(positions, cell, 1.1, torch_dtype, cuda)
    assert path == "grid"


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_boundary_pairs_bit_exact(cuda, tag):
    """Pairs placed at the list radius plus or minus a few ulp: the rounding decides them."""
    torch_dtype, np_dtype = DTYPES[tag]
    rng = np.random.default_rng(5)
    length = 6.0
    radius = 1.1
    centers = rng.uniform(0.5, length - 0.5, (400, 3))
    directions = rng.normal(size=(400, 3))
    directions /= np.linalg.norm(directions, axis=1, keepdims=True)
    ulps = rng.integers(-6, 7, 400)
    r = np.array([np.float64(np_dtype(radius)) for _ in range(400)])
    r = r * (1 + ulps * float(np.finfo(np_dtype).eps))
    partners = centers + directions * r[:, None]
    positions = np.concatenate([centers, partners]).astype(np_dtype)
    check_against_oracle(positions, np.full(3, length), radius, torch_dtype, cuda)


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("length, path", [(6.0, "grid"), (3.2, "all")])
def test_designed_rounding_frames_bit_exact(cuda, tag, length, path):
    """Pairs within 0.6 ulp of the squared radius (tests/boundary_frames.py): the kernels list
    exactly the pairs that r^2 = fma(dz, dz, fma(dx, dx, dy * dy)) lists."""
    import boundary_frames as bf

    torch_dtype, np_dtype = DTYPES[tag]
    positions, cell, first, second = bf.designed_frame(length, 1200 if path == "grid" else 300,
                                                       1.1, np_dtype, seed=4)
    neighbor_list, found = check_against_oracle(positions, cell, 1.1, torch_dtype, cuda)
    assert found == path
    index, total = listed(neighbor_list)
    listed_here = bf.designed_listed(on.pair_set(index[0, :total], index[1, :total]), first,
                                     second)
    np.testing.assert_array_equal(
        listed_here, bf.listed_under(bf.PINNED, positions, first, second, 1.1))


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_update_reuses_then_rebuilds(cuda, tag):
    torch_dtype, np_dtype = DTYPES[tag]
    positions, cell = lattice.simple_cubic(14, 5.2, 0.02, seed=9)
    x = torch.tensor(positions, dtype=torch_dtype, device=cuda)
    box = torch.tensor(cell, dtype=torch_dtype, device=cuda)
    neighbor_list = NeighborList(1.0, skin=0.1)
    neighbor_list.allocate(x, box)
    before = listed(neighbor_list)[0].copy()
    assert neighbor_list._rebuild_count == 1
    small = x.clone()
    small[3, 0] += 0.04  # under half the skin: reuse
    neighbor_list.update(small, box)
    assert neighbor_list._rebuild_count == 1
    np.testing.assert_array_equal(listed(neighbor_list)[0], before)
    large = x.clone()
    large[3, 0] += 0.3  # past half the skin: rebuild at the new frame
    large[100] -= 5.2 * 2  # outside the cell
    neighbor_list.update(large, box)
    assert neighbor_list._rebuild_count == 2
    from nabladyn_b200 import space
    wrapped = space.wrap(large, box)[0].cpu().numpy()
    first, second, _ = on.pairs(wrapped, cell.astype(np_dtype), neighbor_list.radius)
    index, total = listed(neighbor_list)
    np.testing.assert_array_equal(on.pair_set(index[0, :total], index[1, :total]),
                                  on.pair_set(first, second))


def test_status_bits_fail_the_list(cuda):
    positions, cell = lattice.simple_cubic(10, 4.0, 0.02, seed=4)
    x = torch.tensor(positions, dtype=torch.float32, device=cuda)
    box = torch.tensor(cell, dtype=torch.float32, device=cuda)
    neighbor_list = NeighborList(1.0, skin=0.1, capacity_multiplier=1.0)
    neighbor_list.allocate(x, box)
    bad = x.clone()
    bad[4, 1] = float("nan")
    with pytest.raises(ValueError, match="positions must be finite"):
        neighbor_list.update(bad, box)
    with pytest.raises(RuntimeError, match="call allocate"):
        neighbor_list.tensors()
    neighbor_list.allocate(x, box)  # recovers
    squeezed = (x - 2.0) * 0.8 + 2.0  # denser: more pairs than the capacity
    with pytest.raises(ValueError, match="raise capacity_multiplier"):
        neighbor_list.update(squeezed, box)
    neighbor_list.allocate(x, box)
    with pytest.raises(ValueError, match="above twice the cutoff"):
        neighbor_list.update(x, torch.tensor([1.9, 4.0, 4.0], dtype=torch.float32, device=cuda))
    with pytest.raises(ValueError):
        NeighborList(1.0).allocate(x, torch.tensor([1.5, 4.0, 4.0], device=cuda))


def test_c_abi_count_and_fill(cuda):
    """The C-ABI alone, with buffers allocated here, gives the oracle's pairs."""
    positions, cell = lattice.random_box(3000, (5.0, 5.0, 5.0), seed=21)
    dtype = torch.float32
    x = torch.tensor(positions, dtype=dtype, device=cuda)
    box = torch.tensor(cell, dtype=dtype, device=cuda)
    n, radius = 3000, 1.1
    dims = on.grid_dims(cell, radius, np.float32)
    bins = math.prod(dims)
    scan = ctypes.c_int64(0)
    _native.call("nd_neighbors_scan_temp_bytes", max(bins + 1, n), ctypes.byref(scan))
    ints = {"dtype": torch.int32, "device": cuda}
    t = {
        "dims": torch.tensor(dims, **ints),
        "widths": torch.tensor([c / d for c, d in zip(cell, dims)], dtype=dtype, device=cuda),
        "atom_bin": torch.empty(n, **ints),
        "bin_counts": torch.zeros(bins + 1, **ints),
        "bin_offsets": torch.empty(bins + 1, **ints),
        "unordered_ids": torch.empty(n, **ints),
        "sorted_ids": torch.empty(n, **ints),
        "sorted_positions": torch.empty((n, 3), dtype=dtype, device=cuda),
        "scan_temp": torch.empty(scan.value, dtype=torch.uint8, device=cuda),
        "pair_counts": torch.empty(n, **ints),
        "pair_offsets": torch.empty(n, **ints),
        "pair_total": torch.zeros(1, **ints),
        "status": torch.zeros(2, **ints),
    }
    t["pairs"] = torch.empty((2, 1), **ints)  # sized after the count, as allocate does
    buffers = _native.NeighborBuffers(
        **{k: v.data_ptr() for k, v in t.items()},
        num_bin_slots=bins + 1, scan_temp_bytes=scan.value, capacity=1, bits=None, bits_numel=0,
    )
    stream = torch.cuda.current_stream(cuda).cuda_stream
    _native.call("nd_neighbors_count_first_frame", _native.ND_FLOAT32, x.data_ptr(),
                 box.data_ptr(), n, radius, ctypes.byref(buffers), stream)
    count = int(t["pair_counts"].sum())
    pairs = torch.empty((2, count + 5), **ints)
    buffers.pairs, buffers.capacity = pairs.data_ptr(), count + 5
    _native.call("nd_neighbors_fill_first_frame", _native.ND_FLOAT32, x.data_ptr(),
                 box.data_ptr(), n, radius, ctypes.byref(buffers), stream)
    torch.cuda.synchronize()
    first, second, _ = on.pairs(positions.astype(np.float32), cell.astype(np.float32), radius)
    index = pairs.cpu().numpy()
    assert int(t["pair_total"]) == count == len(first)
    np.testing.assert_array_equal(on.pair_set(index[0, :count], index[1, :count]),
                                  on.pair_set(first, second))
    np.testing.assert_array_equal(t["sorted_ids"].cpu().numpy(),
                                  np.lexsort((np.arange(n), t["atom_bin"].cpu().numpy())))
