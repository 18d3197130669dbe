"""The C-ABI library loads, exports every declared symbol and rejects bad arguments (CPU)."""

import ctypes
import re
from pathlib import Path

import pytest
import torch

from nabladyn_b200 import _native

HEADER = Path(__file__).resolve().parents[1] / "include" / "nabladyn_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    library = _native.lib()
    names = declared_functions()
    assert "nd_md_step" in names and "nd_neighbors_update" in names
    for name in names:
        assert hasattr(library, name), name
    assert set(names) == set(_native.EXPORTED)
    assert library.nd_abi_version() == 1


def test_scan_temp_bytes_and_argument_errors():
    library = _native.lib()
    value = ctypes.c_int64(0)
    assert library.nd_neighbors_scan_temp_bytes(100, ctypes.byref(value)) == _native.ND_OK
    assert value.value > 0
    assert library.nd_neighbors_scan_temp_bytes(0, ctypes.byref(value)) == _native.ND_EINVAL
    assert b"int32" in library.nd_last_error()


def test_lj_rejects_null_arguments():
    library = _native.lib()
    args = _native.LJPairsArgs(dtype=0, num_atoms=10, capacity=4, num_types=1, cutoff=1.0)
    assert library.nd_lj_energy_force_virial(ctypes.byref(args), None) == _native.ND_EINVAL
    assert b"null" in library.nd_last_error()
    args.dtype = 7
    assert library.nd_lj_energy_force_virial(ctypes.byref(args), None) == _native.ND_EINVAL


def test_md_rejects_small_box_too_large():
    library = _native.lib()
    system = _native.MDSystem(dtype=0, num_atoms=100000, num_types=1, small=1, width=8)
    slots = ctypes.c_int64(0)
    assert library.nd_md_partial_slots(ctypes.byref(system), ctypes.byref(slots)) == _native.ND_EINVAL
    system.num_atoms = 500
    assert library.nd_md_partial_slots(ctypes.byref(system), ctypes.byref(slots)) == _native.ND_OK
    assert slots.value == 32 * 8  # ceil(500 x 16 lanes / 256) force blocks x 8 sums


def test_neighbor_schemas_match_the_reference():
    """src/nabladyn/neighbors/csrc/ops.cpp:11-41, byte for byte."""
    ops = _native.neighbor_ops()
    buffers = (
        "Tensor(a!) dims, Tensor(b!) widths, Tensor(c!) atom_bin, Tensor(d!) bin_counts, "
        "Tensor(e!) bin_offsets, Tensor(f!) unordered_ids, Tensor(g!) sorted_ids, "
        "Tensor(h!) sorted_positions, Tensor(i!) scan_temp, Tensor(j!) pair_counts, "
        "Tensor(k!) pair_offsets, Tensor(l!) pair_total, Tensor(m!) status, Tensor(n!) pairs, "
        "Tensor(t!) bits"
    )
    expected = {
        "scan_temp_bytes": "nabladyn_neighbors::scan_temp_bytes(Tensor reference, int items) -> int",
        "count_first_frame": "nabladyn_neighbors::count_first_frame(Tensor positions, Tensor cell, "
        f"float radius, {buffers}) -> ()",
        "fill_first_frame": "nabladyn_neighbors::fill_first_frame(Tensor positions, Tensor cell, "
        f"float radius, {buffers}) -> ()",
        "update": "nabladyn_neighbors::update(Tensor positions, Tensor cell, float cutoff, "
        "float radius, Tensor(o!) reference_positions, Tensor(p!) reference_cell, Tensor limits, "
        "Tensor(q!) reuse, Tensor(r!) rebuild, Tensor(s!) rebuild_count, "
        f"{buffers}) -> ()",
    }
    for name, schema in expected.items():
        assert str(getattr(ops, name).default._schema) == schema
    assert ops.scan_temp_bytes(torch.zeros(1), 5000) == 8


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_native, "_lib", None)
    monkeypatch.setattr(_native, "CORE_PATH", tmp_path / "libnabladyn_b200.so")
    with pytest.raises(RuntimeError, match="not built"):
        _native.lib()


def test_replica_record_layout_and_pool_allocator():
    """The ctypes record matches the header's layout; the server's first-fit allocator merges
    freed ranges (no device needed)."""
    from nabladyn_b200.serving import ReplicaServer

    assert ctypes.sizeof(_native.Replica) == 304
    assert _native.Replica.energy.offset == 104
    server = ReplicaServer(device="cpu", budget_bytes=1 << 22, max_slots=4)
    total = server.capacity // 32
    a, b = server._take(3), server._take(5)
    assert (a, b) == (0, 3)
    server._give(a, 3)
    assert server._free_units == [(0, 3), (8, total - 8)]
    server._give(b, 5)
    assert server._free_units == [(0, total)]
    assert server._take(total + 1) is None
    # Freed room and slots are handed back together, in the order given.
    server._take(4)
    server._release([(0, 4, 3)])
    assert server._free_units == [(0, total)] and server._free_slots[-1] == 3


def test_serving_lane_budgets():
    """A round's budget: the large lane's fixed steps, the other lane's atom-steps over the
    replica's size (at least one step), both clamped to the steps left (no device needed)."""
    import numpy as np

    from nabladyn_b200.serving._server import ReplicaRequest, _Active, _Lane

    def entry(n, left):
        request = ReplicaRequest(positions=np.zeros((n, 3)), velocities=np.zeros((n, 3)),
                                 masses=np.ones(n), cell=np.full(3, 5.0), temperature=100.0,
                                 steps=500)
        return _Active(request, 0, 0, -(-n // 32), 0.0, left)

    small = _Lane("", None, None)  # the stream is not needed for a budget
    large = _Lane("_large", None, 25)
    assert small.budget(entry(1000, 500), 200_000) == 200
    assert small.budget(entry(64, 500), 200_000) == 500  # clamped to the steps left
    assert small.budget(entry(16384, 500), 200_000) == 13
    assert small.budget(entry(300_000, 500), 200_000) == 1
    assert large.budget(entry(16384, 500), 200_000) == 25
    assert large.budget(entry(16384, 7), 200_000) == 7


def test_torch_ops_load_first_in_a_fresh_process():
    """Loading the torch.library layer before any other native call (a NeighborList as the
    first use) loads the core library under the same lock and returns."""
    import subprocess
    import sys

    code = ("from nabladyn_b200 import _native; ops = _native.neighbor_ops(); "
            "print(ops.scan_temp_bytes is not None)")
    done = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                          timeout=120)
    assert done.returncode == 0, done.stderr
    assert done.stdout.strip() == "True"


def test_schnet_training_entry_points_check_arguments():
    """nd_schnet_tangent and nd_schnet_atoms reject null buffers, bad stages and directions
    before any launch; the atom workspace's arrays are 256-byte aligned and in order."""
    library = _native.lib()
    tangent = _native.SchNetTangentArgs(num_atoms=100, num_columns=10, interactions=3,
                                        num_types=1, gaussians=50, block=0, cutoff=1.2,
                                        capacity=10)
    assert library.nd_schnet_tangent(ctypes.byref(tangent), 0, None) == _native.ND_EINVAL
    assert b"null" in library.nd_last_error()
    assert library.nd_schnet_tangent(ctypes.byref(tangent), 2, None) == _native.ND_EINVAL
    assert b"direction" in library.nd_last_error()
    atoms = _native.SchNetAtomArgs(num_atoms=100, interactions=3, num_types=2)
    assert library.nd_schnet_atoms(ctypes.byref(atoms), 0, 0, None) == _native.ND_EINVAL
    assert b"null" in library.nd_last_error()
    assert library.nd_schnet_atoms(ctypes.byref(atoms), 5, 0, None) == _native.ND_EINVAL
    assert b"stage" in library.nd_last_error()
    assert library.nd_schnet_atoms(ctypes.byref(atoms), 1, 3, None) == _native.ND_EINVAL
    assert library.nd_schnet_atom_parameter_floats(3, 2) == 3 * (3 * 4096 + 128) + 2144 + 128
    offsets = [library.nd_schnet_atom_offset(100, 3, kind, 2 if kind < 8 else 0)
               for kind in range(17)]
    assert all(offset >= 0 and offset % 256 == 0 for offset in offsets)
    assert library.nd_schnet_atom_workspace_bytes(100, 3) > max(offsets)
    assert library.nd_schnet_atom_offset(100, 3, 17, 0) == -1


def test_schnet_tangent_rejects_small_row_capacity():
    """The reverse pass needs pair rows for every column: a smaller capacity is refused before
    anything is launched (the pointers here are never dereferenced)."""
    library = _native.lib()
    fake = ctypes.c_void_p(1 << 20)
    tangent = _native.SchNetTangentArgs(
        num_atoms=100, num_columns=10, interactions=3, num_types=1, gaussians=50, block=0,
        cutoff=1.2, weights=fake, workspace=fake, force_adjoint=fake, virial_adjoint=fake,
        v=fake, v_dot=fake, m=fake, m_dot=fake, m_bar=fake, m_dot_bar=fake, v_bar=fake,
        v_dot_bar=fake, pair_rows=fake, capacity=5, status=fake)
    assert library.nd_schnet_tangent(ctypes.byref(tangent), 1, None) == _native.ND_EINVAL
    assert b"capacity" in library.nd_last_error()
