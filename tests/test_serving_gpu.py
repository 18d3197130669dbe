"""The replica server on the GPU: each served replica against the reference's own NVT
trajectory, the same result alone and in a mix (bit for bit: replicas never interact), and
admission within the HBM budget.

Tolerances: float32 replicas against the reference's float32 20-step trajectory to 2e-4 nm and
2e-3 nm/ps (two float32 summation orders); alone against mixed exactly.
"""

import ctypes

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice
from nabladyn_b200._native import Replica
from nabladyn_b200.serving import ReplicaRequest, ReplicaServer, serving_requests
from oracle import lj
from oracle import neighbors as on

pytestmark = pytest.mark.gpu


def argon_request(argon, steps, name="argon"):
    return ReplicaRequest(positions=argon["positions"], velocities=argon["velocities"],
                          masses=np.full(512, 39.948), cell=argon["cell"], temperature=120.0,
                          steps=steps, name=name)


def test_served_replica_matches_reference_trajectory(argon, argon_md, cuda):
    server = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=64)
    others = serving_requests(12, seed=3, steps=20, largest=3000)
    results = {r.name: r for r in server.serve([argon_request(argon, 20)] + others,
                                                realtime=False)}
    mine = results["argon"]
    assert mine.status == 0 and mine.steps == 20
    np.testing.assert_allclose(mine.positions, argon_md["NVT_f32_20_positions"], atol=2e-4)
    np.testing.assert_allclose(mine.velocities, argon_md["NVT_f32_20_velocities"], atol=2e-3)
    np.testing.assert_array_equal(mine.images, argon_md["NVT_f32_20_images"])
    assert mine.energy == pytest.approx(float(argon_md["NVT_f32_20_energy"]), rel=1e-4)


def test_alone_equals_mixed(cuda):
    requests = serving_requests(24, seed=5, steps=60, largest=6000, rate=400.0)
    chosen = [requests[3], requests[10]]
    alone = {}
    for request in chosen:
        server = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=8)
        alone[request.name] = server.serve([request], realtime=False)[0]
    server = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=32,
                           round_atom_steps=50_000)
    mixed = {r.name: r for r in server.serve(requests, realtime=True)}
    for request in chosen:
        a, b = alone[request.name], mixed[request.name]
        assert a.status == b.status == 0
        np.testing.assert_array_equal(a.positions, b.positions)
        np.testing.assert_array_equal(a.velocities, b.velocities)
        assert a.energy == b.energy


def test_two_lanes_equal_one_lane(cuda):
    # Replicas of at least 1,500 atoms run in the second stream's rounds (9 steps a round),
    # the rest beside them; every result equals its run on a single lane, bit for bit (a
    # replica's trajectory does not depend on how its steps are split into rounds).
    requests = serving_requests(20, seed=13, steps=45, smallest=200, largest=6000, rate=300.0)
    assert sum(r.positions.shape[0] >= 1500 for r in requests) >= 4
    one = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=32, large_atoms=None)
    single = {r.name: r for r in one.serve(requests, realtime=False)}
    two = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=32, large_atoms=1500,
                        large_round_steps=9, round_atom_steps=30_000)
    lanes = {r.name: r for r in two.serve(requests, realtime=True)}
    assert set(lanes) == set(single)
    for name, a in single.items():
        b = lanes[name]
        assert a.status == b.status == 0 and a.steps == b.steps == 45
        np.testing.assert_array_equal(a.positions, b.positions)
        np.testing.assert_array_equal(a.velocities, b.velocities)
        np.testing.assert_array_equal(a.images, b.images)
        assert a.energy == b.energy


def test_two_lanes_reuse_slots_and_room(cuda):
    # Four slots and room for about 8,000 atoms: harvested slots and room are taken again,
    # across the lanes, only after the rounds that still named them have run; every result
    # equals its single-lane run bit for bit.
    requests = serving_requests(14, seed=17, steps=30, smallest=300, largest=3000, rate=500.0)
    one = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=16, large_atoms=None)
    single = {r.name: r for r in one.serve(requests, realtime=False)}
    two = ReplicaServer(device=cuda, budget_bytes=4 << 20, max_slots=4, large_atoms=1200,
                        large_round_steps=7, round_atom_steps=20_000)
    results = two.serve(requests, realtime=True)
    assert len(results) == len(requests) and len({r.name for r in results}) == len(requests)
    assert len({r.admitted for r in results}) > 4  # slots and room were reused
    for b in results:
        a = single[b.name]
        assert a.status == b.status == 0 and a.steps == b.steps == 30
        np.testing.assert_array_equal(a.positions, b.positions)
        np.testing.assert_array_equal(a.velocities, b.velocities)
        assert a.energy == b.energy


def test_grid_replica_energy_against_oracle(cuda):
    positions, cell = lattice.fcc(10, 10 * 0.5745, 0.03, seed=9)  # 4,000 atoms, >= 3 cells/axis
    request = ReplicaRequest(positions=positions, velocities=np.zeros_like(positions),
                             masses=np.full(len(positions), 39.948), cell=cell,
                             temperature=120.0, steps=0, name="grid")
    server = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=4)
    result = server.serve([request], realtime=False)[0]
    wrapped = on.wrap(positions, cell)
    first, second, _ = on.pairs(wrapped, cell, 1.0)
    energy, _, _ = lj.energy_force_virial(wrapped, cell, first, second, [0.34], [0.996], 1.0)
    assert result.energy == pytest.approx(energy, rel=1e-5)


def _served_lists(server, slot: int):
    """The replica's lists as of its last rebuild, read from the pool: (atom, neighbor) for
    every entry, whether the entry is a direct one (listed before the row's entries that need
    an image), the reference frame (that rebuild's wrapped positions) and its record."""
    size = ctypes.sizeof(Replica)
    raw = server.table.view(server.max_slots, size)[slot].cpu().numpy().tobytes()
    record = Replica.from_buffer_copy(raw)
    n, width, a0 = record.num_atoms, record.width, record.atom_offset
    b = server.buffers
    reference = b["reference_positions"][a0:a0 + n, :3].cpu().numpy()
    order = b["sorted"][a0:a0 + n].cpu().numpy()
    packed = b["neighbor_counts"][a0:a0 + n].cpu().numpy()
    counts, direct = packed & 0xFFFF, packed >> 16
    assert np.all(direct <= counts)
    words = b["neighbors"].view(torch.int16).cpu().numpy().view(np.uint16)
    words = words[record.list_offset:record.list_offset + n * width]
    assert counts.max() <= width
    rows = np.repeat(np.arange(n), counts)
    slots = np.concatenate([np.arange(c) for c in counts])
    # chunk c of row r is 16-B word ((r / 32) * width / 8 + c) * 32 + r % 32
    word = ((rows >> 5) * (width // 8) + slots // 8) * 32 + (rows & 31)
    neighbors = words[word * 8 + slots % 8].astype(np.int64)
    return order[rows].astype(np.int64), neighbors, slots < direct[rows], reference, record


def test_grid_replica_lists_equal_minimum_image_scan(cuda):
    # The in-CTA rebuild scans each stencil cell with one image per cell; its lists must hold
    # exactly the pairs a per-candidate minimum image puts within the list radius (the oracle's
    # all-pairs path, contraction pinned), after rebuilds along a trajectory.
    positions, cell = lattice.fcc(10, 10 * 0.5745, 0.03, seed=21)  # 4,000 atoms, 5 cells/axis
    velocities = np.random.default_rng(22).normal(0.0, 0.4, positions.shape)
    request = ReplicaRequest(positions=positions, velocities=velocities,
                             masses=np.full(len(positions), 39.948), cell=cell,
                             temperature=300.0, steps=80, name="grid")
    server = ReplicaServer(device=cuda, budget_bytes=64 << 20, max_slots=1)
    result = server.serve([request], realtime=False)[0]
    assert result.status == 0 and result.rebuilds >= 3
    atoms, neighbors, direct, reference, record = _served_lists(server, 0)
    assert min(record.dims) >= 3
    cell32 = np.asarray(record.cell, dtype=np.float32)
    first, second, path = on.pairs(reference.astype(np.float32), cell32,
                                   float(np.float32(record.radius)), dims=(3, 3, 3))
    assert path == "all"
    n = record.num_atoms
    want = np.sort(np.concatenate([first * n + second, second * n + first]).astype(np.int64))
    got = np.sort(atoms * n + neighbors)
    assert len(np.unique(got)) == len(got)  # no entry twice
    np.testing.assert_array_equal(got, want)
    # Direct entries are evaluated without the minimum image until the next rebuild: at the
    # rebuild, their plain difference was within the list radius on every axis.
    plain = np.abs(reference[atoms[direct]] - reference[neighbors[direct]])
    assert direct.mean() > 0.5 and np.all(plain < np.float32(record.radius))
    # The last step's energy, from lists reused since that rebuild, against the oracle at the
    # final positions.
    final = result.positions.astype(np.float64)
    first, second, _ = on.pairs(final, cell, 1.0)
    energy, _, _ = lj.energy_force_virial(final, cell, first, second, [0.34], [0.996], 1.0)
    assert result.energy == pytest.approx(energy, rel=1e-5)


def test_admission_stays_within_budget(cuda):
    requests = serving_requests(16, seed=11, steps=40, smallest=300, largest=2500)
    server = ReplicaServer(device=cuda, budget_bytes=3 << 20, max_slots=16)
    capacity = server.capacity
    results = server.serve(requests, realtime=False)
    assert len(results) == 16 and all(r.status == 0 and r.steps == 40 for r in results)
    # At any admission time, the atoms resident (rounded to 32) fit the pool.
    events = sorted(set(r.admitted for r in results))
    for t in events:
        resident = sum(-(-r.num_atoms // 32) * 32 for r in results
                       if r.admitted <= t < r.finished)
        assert resident <= capacity
    assert len({r.admitted for r in results}) > 1  # the budget made some wait
