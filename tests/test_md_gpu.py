"""MD on the GPU: trajectories against the reference's own step, conservation, rebuilds,
state and resume, panel and failure detection.

Tolerances: float64 trajectories match the reference's 20-step trajectories to 1e-9 nm and
1e-8 nm/ps (the reference's own float64 run is the golden, made by its ensemble halves); the
float32 ones to 2e-4, the divergence of two float32 trajectories with different summation
orders over 20 steps.
"""

import math

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice, md, potential
from oracle import lj
from oracle import neighbors as on

pytestmark = pytest.mark.gpu


def argon_system(argon, dtype, device):
    n = argon["positions"].shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([0.34], dtype=dtype, device=device),
        epsilon=torch.tensor([0.996], dtype=dtype, device=device),
        cutoff=1.0,
    )
    x = torch.tensor(argon["positions"], dtype=dtype, device=device)
    v = torch.tensor(argon["velocities"], dtype=dtype, device=device)
    cell = torch.tensor(argon["cell"], dtype=dtype, device=device)
    masses = torch.full((n,), 39.948, dtype=dtype, device=device)
    return model, x, v, masses, cell


def build(ensemble, model, x, v, masses, cell, **kwargs):
    if ensemble == "NVE":
        return md.nve(model, x, v, masses, cell, timestep=0.004, **kwargs)
    return md.nvt(model, x, v, masses, cell, timestep=0.004, temperature=120.0,
                  thermostat_timescale=0.1, **kwargs)


@pytest.mark.parametrize("ensemble", ["NVE", "NVT"])
@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_trajectory_matches_reference(argon, argon_md, cuda, ensemble, tag):
    dtype = torch.float64 if tag == "f64" else torch.float32
    simulation = build(ensemble, *argon_system(argon, dtype, cuda))
    atol_x, atol_v = (1e-9, 1e-8) if tag == "f64" else (2e-4, 2e-3)
    done = 0
    for step in (1, 5, 20):
        simulation.run(step - done)
        done = step
        state = simulation.state()
        key = f"{ensemble}_{tag}_{step}"
        assert state.step == step
        np.testing.assert_allclose(state.positions.cpu().numpy(), argon_md[f"{key}_positions"],
                                   atol=atol_x)
        np.testing.assert_allclose(state.velocities.cpu().numpy(),
                                   argon_md[f"{key}_velocities"], atol=atol_v)
        np.testing.assert_array_equal(state.images.cpu().numpy(), argon_md[f"{key}_images"])
        if ensemble == "NVT" and tag == "f64":
            np.testing.assert_allclose(state.thermostat.momenta.cpu().numpy(),
                                       argon_md[f"{key}_chain_momenta"], atol=1e-9)


@pytest.mark.parametrize("ensemble", ["NVE", "NVT"])
@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_one_launch_run_matches_step_graphs(argon, cuda, monkeypatch, ensemble, tag):
    """The 512-atom box's one-launch runs (nd_md_run_small, the small-box path) against the same
    300 steps from the per-step graphs, with rebuilds on the way: the same trajectory and
    panel. Only the float64 order of the totals differs, which the thermostat's factor sees:
    float64 to 1e-9, float32 NVE exactly, float32 NVT to 1e-4 nm."""
    from nabladyn_b200.md._engine import Engine

    dtype = torch.float64 if tag == "f64" else torch.float32

    def run(one_launch: bool):
        with monkeypatch.context() as patch:
            if not one_launch:
                patch.setattr(Engine, "ONE_LAUNCH_MAX_ATOMS", 0)
            simulation = build(ensemble, *argon_system(argon, dtype, cuda))
            assert simulation._engine.runs_in_one_launch == one_launch
            panel = simulation.run(300, sample_every=100)
            return simulation.state(), panel

    state, panel = run(True)
    expected, expected_panel = run(False)
    atol = 1e-9 if tag == "f64" else (0.0 if ensemble == "NVE" else 1e-4)
    np.testing.assert_allclose(state.positions.cpu().numpy(),
                               expected.positions.cpu().numpy(), atol=atol, rtol=0)
    np.testing.assert_allclose(state.velocities.cpu().numpy(),
                               expected.velocities.cpu().numpy(), atol=10 * atol, rtol=0)
    np.testing.assert_array_equal(state.images.cpu().numpy(), expected.images.cpu().numpy())
    for name, values in expected_panel.items():
        np.testing.assert_allclose(panel[name].numpy(), values.numpy(),
                                   rtol=1e-9 if tag == "f64" else 1e-4, err_msg=name)


def test_resume_from_state_is_the_same_run(argon, cuda):
    model, x, v, masses, cell = argon_system(argon, torch.float64, cuda)
    straight = build("NVT", model, x, v, masses, cell)
    straight.run(40)
    first = build("NVT", model, x, v, masses, cell)
    first.run(15)
    saved = first.state()
    second = md.nvt(model, saved.positions, saved.velocities, masses, cell, timestep=0.004,
                    temperature=120.0, thermostat_timescale=0.1, images=saved.images,
                    step=saved.step, thermostat=saved.thermostat)
    second.run(25)
    a, b = straight.state(), second.state()
    assert a.step == b.step == 40
    np.testing.assert_allclose(a.positions.cpu(), b.positions.cpu(), atol=1e-9)
    np.testing.assert_allclose(a.velocities.cpu(), b.velocities.cpu(), atol=1e-9)


def test_panel_matches_state(argon, cuda):
    model, x, v, masses, cell = argon_system(argon, torch.float64, cuda)
    simulation = build("NVT", model, x, v, masses, cell)
    samples = simulation.run(30, sample_every=10)
    assert samples["step"].tolist() == [10, 20, 30]
    state = simulation.state()
    wrapped = state.positions.cpu().numpy()
    first, second = lj.all_pairs(512)
    energy, _, virial = lj.energy_force_virial(wrapped, argon["cell"], first, second, [0.34],
                                               [0.996], 1.0)
    kinetic = 0.5 * 39.948 * float((state.velocities.cpu().numpy() ** 2).sum())
    assert float(samples["potential_energy"][-1]) == pytest.approx(energy, abs=1e-8)
    assert float(samples["kinetic_energy"][-1]) == pytest.approx(kinetic, rel=1e-10)
    temperature = 2 * kinetic / ((3 * 512 - 3) * 0.00831446261815324)
    assert float(samples["temperature"][-1]) == pytest.approx(temperature, rel=1e-10)
    volume = float(np.prod(argon["cell"]))
    pressure = (2 * kinetic + np.trace(virial)) / (3 * volume)
    assert float(samples["pressure"][-1]) == pytest.approx(pressure, rel=1e-9)
    assert set(samples) == {"step", *md.FIELDS, "conserved_energy"}


def test_nve_conserves_energy_and_rebuilds_on_gpu(cuda):
    """4,000 atoms, float32, 2,000 steps: the total energy drifts by under 1e-4 relative, and
    the neighbor rebuilds are decided inside the captured step."""
    positions, cell = lattice.simple_cubic(16, 16 / 21.0 ** (1 / 3) * 1.0, 0.02, seed=5,
                                           count=4000)
    cell = np.full(3, (4000 / 21.0) ** (1 / 3))
    positions, _ = lattice.simple_cubic(16, float(cell[0]), 0.02, seed=5, count=4000)
    dtype = torch.float32
    n = positions.shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
        sigma=torch.tensor([0.34], dtype=dtype, device=cuda),
        epsilon=torch.tensor([0.996], dtype=dtype, device=cuda),
        cutoff=1.0,
    )
    masses = torch.full((n,), 39.948, dtype=dtype, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 120.0, seed=1)
    simulation = md.nve(model, torch.tensor(positions, dtype=dtype, device=cuda), velocities,
                        masses, torch.tensor(cell, dtype=dtype, device=cuda), timestep=0.002)
    simulation.run(500)  # equilibrate from the lattice
    start = simulation.sample()["total_energy"]
    samples = simulation.run(2000, sample_every=100)
    drift = np.abs(samples["total_energy"].double().numpy() - start).max()
    assert drift < 1e-4 * abs(start) + 0.5
    assert simulation._rebuild_count > 10


def test_non_finite_fails_the_simulation(argon, cuda):
    model, x, v, masses, cell = argon_system(argon, torch.float32, cuda)
    simulation = build("NVE", model, x, v, masses, cell)
    simulation._engine.tensors["velocities"][7, 0] = float("inf")
    with pytest.raises(ValueError, match="positions must be finite"):
        simulation.run(10)
    with pytest.raises(RuntimeError, match="start a new one"):
        simulation.run(1)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_engine_forces_on_grid_path(cuda, dtype):
    """A system with >= 3 cells per axis: the brick-tile force kernel against the oracle."""
    positions, cell = lattice.fcc(10, 10 * 0.5745, 0.03, seed=12)  # 4,000 atoms, 5.2 cells
    n = positions.shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
        sigma=torch.tensor([0.34], dtype=dtype, device=cuda),
        epsilon=torch.tensor([0.996], dtype=dtype, device=cuda),
        cutoff=1.0,
    )
    masses = torch.full((n,), 39.948, dtype=dtype, device=cuda)
    x = torch.tensor(positions, dtype=dtype, device=cuda)
    box = torch.tensor(cell, dtype=dtype, device=cuda)
    simulation = md.nve(model, x, torch.zeros_like(x), masses, box, timestep=0.004)
    assert not simulation._engine.small
    state = simulation.state()
    wrapped = on.wrap(positions.astype(np.float64), cell)
    first, second, _ = on.pairs(wrapped, cell, 1.0)
    _, f64, _ = lj.energy_force_virial(wrapped, cell, first, second, [0.34], [0.996], 1.0)
    error = np.linalg.norm(state.forces.cpu().double().numpy() - f64) / np.linalg.norm(f64)
    assert error < (1e-5 if dtype == torch.float32 else 1e-12)


def test_two_types_on_grid_path_match_oracle(cuda):
    """A 50/50 two-type mixture on the brick-tile path (2,048 atoms, 4 cells per axis), float64:
    20 NVE steps of md.nve against the oracle's velocity Verlet (positions to 1e-9 nm), then
    the panel's potential energy and pressure of the last frame against the oracle's E and
    virial (1e-9 relative): the multi-type force kernel and the grid path's virial."""
    from oracle import integrator

    positions, cell = lattice.fcc(8, 8 * 0.5745, 0.02, seed=23)
    n = positions.shape[0]
    types = np.random.default_rng(23).permutation(np.arange(n) % 2)
    sigma, epsilon = [0.34, 0.32, 0.30], [0.996, 0.8, 0.6]
    dtype = torch.float64
    model = potential.lennard_jones(
        atom_types=torch.tensor(types, device=cuda),
        sigma=torch.tensor(sigma, dtype=dtype, device=cuda),
        epsilon=torch.tensor(epsilon, dtype=dtype, device=cuda),
        cutoff=1.0,
    )
    masses = torch.full((n,), 39.948, dtype=dtype, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 120.0, seed=23)
    simulation = md.nve(model, torch.tensor(positions, dtype=dtype, device=cuda), velocities,
                        masses, torch.tensor(cell, dtype=dtype, device=cuda), timestep=0.004)
    assert not simulation._engine.small and simulation._engine.num_types == 2
    simulation.run(20)
    state = simulation.state()

    def evaluate(frame):
        first, second, _ = on.pairs(frame, cell, 1.0)
        energy, forces, _ = lj.energy_force_virial(frame, cell, first, second, sigma, epsilon,
                                                   1.0, atom_types=types)
        return energy, forces

    want = integrator.run(positions, velocities.cpu().numpy(), np.full(n, 39.948), cell, sigma,
                          epsilon, 1.0, 0.004, 20, evaluate=evaluate)
    np.testing.assert_allclose(state.positions.cpu().numpy(), want["positions"], rtol=0,
                               atol=1e-9)
    np.testing.assert_allclose(state.velocities.cpu().numpy(), want["velocities"], rtol=0,
                               atol=1e-8)
    panel = simulation.sample()
    x = state.positions.cpu().numpy()
    first, second, _ = on.pairs(x, cell, 1.0)
    energy, _, virial = lj.energy_force_virial(x, cell, first, second, sigma, epsilon, 1.0,
                                               atom_types=types)
    v = state.velocities.cpu().numpy()
    kinetic = 0.5 * 39.948 * float((v * v).sum())
    pressure = (2 * kinetic + np.trace(virial)) / (3 * float(np.prod(cell)))
    assert float(panel["potential_energy"]) == pytest.approx(energy, rel=1e-9)
    assert float(panel["pressure"]) == pytest.approx(pressure, rel=1e-9)


def test_run_writes_sample_file(argon, cuda, monkeypatch, tmp_path):
    """run(..., sample_file=) writes each sample's frame and panel (through the in-memory h5py
    stand-in of tests/fake_h5py.py): the samples equal run's returned panel and the last
    frame equals state()."""
    import sys

    import fake_h5py

    monkeypatch.setitem(sys.modules, "h5py", fake_h5py)
    simulation = build("NVT", *argon_system(argon, torch.float32, cuda))
    path = tmp_path / "run.h5"
    samples = simulation.run(20, sample_every=10, sample_file=path)
    state = simulation.state()
    data, attributes = md.read_sample_file(path)
    assert data["step"].tolist() == [10, 20]
    np.testing.assert_allclose(data["time"], [0.04, 0.08])
    np.testing.assert_array_equal(data["positions"][-1], state.positions.cpu().numpy())
    np.testing.assert_array_equal(data["images"][-1], state.images.cpu().numpy())
    for name, values in samples.items():
        if name != "step":
            np.testing.assert_array_equal(data[name], values.numpy(), err_msg=name)
    assert attributes["ensemble"] == "NVT" and attributes["timestep"] == 0.004
    assert attributes["cutoff"] == 1.0 and attributes["schema"] == "nabladyn.samples"


def test_melting_lattice_keeps_its_pair_lists(cuda):
    """A jittered simple-cubic start melting at 150 K on the brick path (the serving workload's
    kind of replica): the pairs of centers drift apart as the lattice melts, and their lists
    must keep fitting the capacity sized on the first frame. 500 NVT steps run without a
    failure, and the last frame's forces match the oracle's."""
    from nabladyn_b200.serving import serving_requests

    request = next(r for r in serving_requests(64, seed=11) if 3000 <= r.positions.shape[0] <= 9000)
    n = request.positions.shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
        sigma=torch.tensor([0.34], device=cuda), epsilon=torch.tensor([0.996], device=cuda),
        cutoff=1.0,
    )
    simulation = md.nvt(
        model, torch.tensor(request.positions, dtype=torch.float32, device=cuda),
        torch.tensor(request.velocities, dtype=torch.float32, device=cuda),
        torch.full((n,), 39.948, device=cuda),
        torch.tensor(request.cell, dtype=torch.float32, device=cuda), timestep=0.004,
        temperature=150.0, thermostat_timescale=0.1)
    assert not simulation._engine.small
    simulation.run(500)
    state = simulation.state()
    assert simulation._rebuild_count >= 5
    cell = request.cell.astype(np.float64)
    x = on.wrap(state.positions.cpu().double().numpy(), cell)
    first, second, _ = on.pairs(x, cell, 1.0)
    _, f64, _ = lj.energy_force_virial(x, cell, first, second, [0.34], [0.996], 1.0)
    error = np.linalg.norm(state.forces.cpu().double().numpy() - f64) / np.linalg.norm(f64)
    assert error < 1e-5


def test_small_box_tile_near_the_default_shared_memory(cuda):
    """3,040 atoms in a 5.0 nm box with a 1.6 nm cutoff take the small-box path with a
    48,656-B tile: under 48 KB alone, over it with the force kernel's static shared memory, so
    the launch needs the raised limit. The first frame's forces and energy match the oracle,
    and the one-launch run steps on."""
    positions, cell = lattice.simple_cubic(15, 5.0, 0.01, seed=3040, count=3040)
    n = positions.shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=cuda),
        sigma=torch.tensor([0.34], device=cuda), epsilon=torch.tensor([0.996], device=cuda),
        cutoff=1.6,
    )
    masses = torch.full((n,), 39.948, device=cuda)
    velocities = md.maxwell_boltzmann(masses, 120.0, seed=3040)
    simulation = md.nve(model, torch.tensor(positions, dtype=torch.float32, device=cuda),
                        velocities, masses, torch.tensor(cell, dtype=torch.float32, device=cuda),
                        timestep=0.002)
    assert simulation._engine.small and simulation._engine.runs_in_one_launch
    state = simulation.state()
    cell64 = np.asarray(cell, dtype=np.float64)
    x = on.wrap(state.positions.cpu().double().numpy(), cell64)
    first, second, _ = on.pairs(x, cell64, 1.6)
    _, f64, _ = lj.energy_force_virial(x, cell64, first, second, [0.34], [0.996], 1.6)
    error = np.linalg.norm(state.forces.cpu().double().numpy() - f64) / np.linalg.norm(f64)
    assert error < 1e-5
    simulation.run(20)
    assert np.isfinite(simulation.state().positions.cpu().numpy()).all()
