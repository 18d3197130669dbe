"""The allocation-free pair build against the regular entry points, through the C-ABI.

nd_neighbors_build_no_alloc serves callers that cannot call cudaMalloc (code inside another
framework's graph capture or memory pool, hosts that forbid allocation): it keeps its
intermediate buffers in a fixed device array instead of caller-allocated ones. This test
builds the same frames with nd_neighbors_count_first_frame + nd_neighbors_fill_first_frame
(buffers allocated here) and with the new entry point, two calls in a row on different frames
so the second call starts from the first call's leftovers, and requires the same pair sets,
totals and status, bit for bit. The file is named to be collected last.
"""

import ctypes
import math

import numpy as np
import pytest
import torch

from nabladyn_b200 import _native, lattice
from oracle import neighbors as on

pytestmark = pytest.mark.gpu


def regular_build(x, box, cell, radius, dims, capacity):
    """count_first_frame + fill_first_frame with buffers allocated by torch."""
    device, dtype = x.device, x.dtype
    n = x.shape[0]
    bins = math.prod(dims)
    scan = ctypes.c_int64(0)
    _native.call("nd_neighbors_scan_temp_bytes", max(bins + 1, n), ctypes.byref(scan))
    ints = {"dtype": torch.int32, "device": device}
    all_pairs = max(dims) <= 3
    t = {
        "dims": torch.tensor(dims, **ints),
        "widths": torch.tensor([c / d for c, d in zip(cell, dims)], dtype=dtype, device=device),
        "atom_bin": torch.empty(n, **ints),
        "bin_counts": torch.zeros(bins + 1, **ints),
        "bin_offsets": torch.empty(bins + 1, **ints),
        "unordered_ids": torch.empty(n, **ints),
        "sorted_ids": torch.empty(n, **ints),
        "sorted_positions": torch.empty((n, 3), dtype=dtype, device=device),
        "scan_temp": torch.empty(scan.value, dtype=torch.uint8, device=device),
        "pair_counts": torch.empty(n, **ints),
        "pair_offsets": torch.empty(n, **ints),
        "pair_total": torch.zeros(1, **ints),
        "status": torch.zeros(2, **ints),
        "pairs": torch.empty((2, capacity), **ints),
        "bits": torch.zeros(n * ((n + 31) // 32) if all_pairs else 1, **ints),
    }
    buffers = _native.NeighborBuffers(
        **{k: v.data_ptr() for k, v in t.items()},
        num_bin_slots=bins + 1, scan_temp_bytes=scan.value, capacity=capacity,
        bits_numel=t["bits"].numel() if all_pairs else 0,
    )
    if not all_pairs:
        buffers.bits = None
    stream = torch.cuda.current_stream(device).cuda_stream
    code = _native.dtype_code(dtype)
    for name in ("nd_neighbors_count_first_frame", "nd_neighbors_fill_first_frame"):
        _native.call(name, code, x.data_ptr(), box.data_ptr(), n, radius,
                     ctypes.byref(buffers), stream)
    return t["pairs"], t["pair_total"], t["status"]


def no_alloc_build(x, box, cell, radius, dims, capacity):
    device = x.device
    ints = {"dtype": torch.int32, "device": device}
    pairs = torch.full((2, capacity), -1, **ints)
    total = torch.full((1,), -1, **ints)
    status = torch.full((2,), -1, **ints)
    dims_host = (ctypes.c_int32 * 3)(*dims)
    widths_host = (ctypes.c_double * 3)(*[c / d for c, d in zip(cell, dims)])
    _native.call("nd_neighbors_build_no_alloc", _native.dtype_code(x.dtype), x.data_ptr(),
                 box.data_ptr(), x.shape[0], radius, dims_host, widths_host, pairs.data_ptr(),
                 capacity, total.data_ptr(), status.data_ptr(),
                 torch.cuda.current_stream(device).cuda_stream)
    return pairs, total, status


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_no_alloc_build_matches_regular_build(dtype):
    device = torch.device("cuda", 0)
    np_dtype = np.float32 if dtype == torch.float32 else np.float64
    frames = [
        lattice.fcc(10, 10 * 0.5745, 0.03, seed=31),             # 4,000 atoms, grid path
        lattice.random_box(1500, (8.0, 2.5, 6.0), seed=32),      # a short axis, grid path
        lattice.simple_cubic(8, 2.9, 0.02, seed=33),             # 512 atoms, all-pairs path
    ]
    radius = 1.1
    for positions, cell in frames:
        positions = on.wrap(positions.astype(np_dtype), cell.astype(np_dtype))
        x = torch.tensor(positions, dtype=dtype, device=device)
        box = torch.tensor(cell, dtype=dtype, device=device)
        dims = on.grid_dims(cell, radius, np_dtype)
        first, _, _ = on.pairs(positions, cell.astype(np_dtype), radius, dims)
        capacity = on.capacity(len(first))
        want_pairs, want_total, want_status = regular_build(x, box, cell, radius, dims, capacity)
        for _ in range(2):  # two calls in a row share the array
            pairs, total, status = no_alloc_build(x, box, cell, radius, dims, capacity)
            torch.cuda.synchronize()
            assert int(total) == int(want_total) == len(first)
            assert status.tolist() == want_status.tolist() == [0, 0]
            count = int(total)
            got = pairs.cpu().numpy()
            want = want_pairs.cpu().numpy()
            np.testing.assert_array_equal(on.pair_set(got[0, :count], got[1, :count]),
                                          on.pair_set(want[0, :count], want[1, :count]))
            np.testing.assert_array_equal(got[:, count:], want[:, count:])  # the padding


def test_no_alloc_rejects_sizes_beyond_its_array():
    device = torch.device("cuda", 0)
    positions, cell = lattice.random_box(20000, (20.0, 20.0, 20.0), seed=34)
    x = torch.tensor(positions, dtype=torch.float32, device=device)
    box = torch.tensor(cell, dtype=torch.float32, device=device)
    with pytest.raises(_native.NativeError, match="at most 16384 atoms"):
        no_alloc_build(x, box, cell, 1.1, on.grid_dims(cell, 1.1, np.float32), 10)


@pytest.mark.parametrize("widths, message", [
    ((1.0, 2.0, 2.0), "at least the radius wide"),      # narrower than the radius
    ((0.0, 2.0, 2.0), "positive and finite"),
    ((float("nan"), 2.0, 2.0), "positive and finite"),
])
def test_no_alloc_rejects_bad_widths(widths, message):
    """Bins narrower than the radius would drop pairs: such widths return ND_EINVAL before
    anything is launched."""
    device = torch.device("cuda", 0)
    positions, cell = lattice.random_box(100, (6.0, 6.0, 6.0), seed=35)
    x = torch.tensor(positions, dtype=torch.float32, device=device)
    box = torch.tensor(cell, dtype=torch.float32, device=device)
    ints = {"dtype": torch.int32, "device": device}
    pairs, total, status = (torch.zeros((2, 64), **ints), torch.zeros(1, **ints),
                            torch.zeros(2, **ints))
    rc = _native.lib().nd_neighbors_build_no_alloc(
        _native.ND_FLOAT32, x.data_ptr(), box.data_ptr(), 100, ctypes.c_double(1.1),
        (ctypes.c_int32 * 3)(3, 3, 3), (ctypes.c_double * 3)(*widths), pairs.data_ptr(), 64,
        total.data_ptr(), status.data_ptr(), torch.cuda.current_stream(device).cuda_stream)
    assert rc == 1  # ND_EINVAL
    assert message in _native.lib().nd_last_error().decode()
