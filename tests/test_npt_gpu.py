"""NPT (isotropic MTK with chains on the particles and the barostat) in the pair engine,
against the reference's own 20-step trajectories of the 512-atom argon frame at 50 bar
(tests/golden/argon_512_md.npz, made by its NPT halves in its Simulation's order).

Tolerances as for NVE/NVT: float64 positions 1e-9 nm, velocities 1e-8 nm/ps, cell, box
momentum and both chains 1e-9 (absolute or relative, as written); float32 positions 2e-4 nm,
velocities 2e-3 nm/ps, cell 1e-5 nm.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import md, potential, units

pytestmark = pytest.mark.gpu

PRESSURE = 50 * units.BAR


def npt_system(argon, dtype, device, **kwargs):
    n = argon["positions"].shape[0]
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([0.34], dtype=dtype, device=device),
        epsilon=torch.tensor([0.996], dtype=dtype, device=device), cutoff=1.0)
    return md.npt(model, torch.tensor(argon["positions"], dtype=dtype, device=device),
                  torch.tensor(argon["velocities"], dtype=dtype, device=device),
                  torch.full((n,), 39.948, dtype=dtype, device=device),
                  torch.tensor(argon["cell"], dtype=dtype, device=device), timestep=0.004,
                  temperature=120.0, pressure=PRESSURE, thermostat_timescale=0.1,
                  barostat_timescale=0.5, **kwargs)


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_npt_matches_reference(argon, argon_md, cuda, tag):
    dtype = torch.float64 if tag == "f64" else torch.float32
    simulation = npt_system(argon, dtype, cuda)
    assert type(simulation._engine).__name__ == "PairEngine"
    atol_x, atol_v, atol_l = (1e-9, 1e-8, 1e-10) if tag == "f64" else (2e-4, 2e-3, 1e-5)
    done = 0
    for step in (1, 5, 20):
        simulation.run(step - done)
        done = step
        state = simulation.state()
        key = f"NPT_{tag}_{step}"
        np.testing.assert_allclose(state.cell.cpu().numpy(), argon_md[f"{key}_cell"], atol=atol_l)
        np.testing.assert_allclose(state.positions.cpu().numpy(), argon_md[f"{key}_positions"],
                                   atol=atol_x)
        np.testing.assert_allclose(state.velocities.cpu().numpy(),
                                   argon_md[f"{key}_velocities"], atol=atol_v)
        np.testing.assert_array_equal(state.images.cpu().numpy(), argon_md[f"{key}_images"])
        if tag == "f64":
            np.testing.assert_allclose(float(state.barostat.momentum),
                                       float(argon_md[f"{key}_box_momentum"]), rtol=1e-9)
            np.testing.assert_allclose(state.barostat.chain.momenta.cpu().numpy(),
                                       argon_md[f"{key}_box_chain_momenta"], rtol=1e-8,
                                       atol=1e-12)
            np.testing.assert_allclose(state.thermostat.momenta.cpu().numpy(),
                                       argon_md[f"{key}_chain_momenta"], atol=1e-9)


def test_npt_resume_and_panel(argon, cuda):
    """A state taken mid-run resumes to the same trajectory; the panel has volume and a
    conserved energy that stays flat over a short run."""
    straight = npt_system(argon, torch.float64, cuda)
    straight.run(10)
    half = straight.state()
    straight.run(10)
    end = straight.state()
    resumed = npt_system(argon, torch.float64, cuda)
    resumed = md.npt(resumed.model, half.positions, half.velocities, resumed.masses, half.cell,
                     timestep=0.004, temperature=120.0, pressure=PRESSURE,
                     thermostat_timescale=0.1, barostat_timescale=0.5, images=half.images,
                     step=half.step, thermostat=half.thermostat, barostat=half.barostat)
    resumed.run(10)
    again = resumed.state()
    np.testing.assert_allclose(again.positions.cpu().numpy(), end.positions.cpu().numpy(),
                               atol=1e-8)
    np.testing.assert_allclose(again.cell.cpu().numpy(), end.cell.cpu().numpy(), atol=1e-10)
    samples = straight.run(100, sample_every=10)
    assert "volume" in samples and "conserved_energy" in samples
    conserved = samples["conserved_energy"]
    assert float(conserved.max() - conserved.min()) < 0.5
