"""The oracle against the reference's golden vectors and known answers (CPU)."""

import numpy as np
import pytest

from nabladyn_b200 import lattice
from oracle import integrator, lj
from oracle import neighbors as on


def test_documented_pair_counts(argon):
    """examples/README.md:55-56: 29,014 pairs within 1.1 nm, 21,398 within 1.0 nm."""
    wrapped = on.wrap(argon["positions"], argon["cell"])
    documented = argon["documented"]
    first, second, path = on.pairs(wrapped, argon["cell"], 1.1)
    assert path == "all"
    assert len(first) == int(documented[0]) == int(argon["pairs_within_1_1"])
    assert on.capacity(len(first)) == int(documented[2])
    first, _, _ = on.pairs(wrapped, argon["cell"], 1.0)
    assert len(first) == int(documented[1]) == int(argon["pairs_within_1_0"])


def test_lj_matches_reference_float64(argon):
    wrapped = on.wrap(argon["positions"], argon["cell"])
    first, second = lj.all_pairs(len(wrapped))
    energy, forces, virial = lj.energy_force_virial(
        wrapped, argon["cell"], first, second, [0.34], [0.996], 1.0,
    )
    assert energy == pytest.approx(float(argon["energy_f64"]), abs=1e-9)
    np.testing.assert_allclose(forces, argon["forces_f64"], atol=1e-10)
    np.testing.assert_allclose(virial, argon["virial_f64"], atol=1e-9)
    assert energy == pytest.approx(argon["documented"][3], abs=0.005)
    assert np.linalg.norm(forces, axis=1).max() == pytest.approx(argon["documented"][4], abs=0.005)


def test_lj_two_types_matches_labels(lj_frames):
    """Two-type rows against the file's labels and the reference's own float64 evaluation."""
    first, second = lj.all_pairs(lj_frames["atom_types"].shape[0])
    for k in range(len(lj_frames["energy"])):
        wrapped = on.wrap(lj_frames["positions"][k], lj_frames["cells"][k])
        energy, forces, virial = lj.energy_force_virial(
            wrapped, lj_frames["cells"][k], first, second, lj_frames["sigma"],
            lj_frames["epsilon"], float(lj_frames["cutoff"]), lj_frames["atom_types"],
        )
        assert energy == pytest.approx(float(lj_frames["reference_energy"][k]), abs=1e-9)
        np.testing.assert_allclose(forces, lj_frames["reference_forces"][k], atol=1e-9)
        np.testing.assert_allclose(virial, lj_frames["reference_virial"][k], atol=1e-8)
        assert energy == pytest.approx(float(lj_frames["energy"][k]), abs=1e-8)


@pytest.mark.parametrize("ensemble", ["NVE", "NVT"])
def test_integrator_matches_reference_float64(argon, argon_md, ensemble):
    kwargs = {"temperature": 120.0, "timescale": 0.1} if ensemble == "NVT" else {}
    result = integrator.run(argon["positions"], argon["velocities"], np.full(512, 39.948),
                            argon["cell"], [0.34], [0.996], 1.0, 0.004, 20, **kwargs)
    np.testing.assert_allclose(result["positions"], argon_md[f"{ensemble}_f64_20_positions"],
                               atol=1e-12)
    np.testing.assert_allclose(result["velocities"], argon_md[f"{ensemble}_f64_20_velocities"],
                               atol=1e-12)
    if ensemble == "NVT":
        np.testing.assert_allclose(result["chain_momenta"],
                                   argon_md["NVT_f64_20_chain_momenta"], atol=1e-10)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize(
    "lengths, count",
    [((4.6, 4.6, 4.6), 2000), ((7.3, 3.4, 5.1), 2600), ((8.0, 2.5, 6.0), 1800)],
)
def test_grid_path_finds_every_pair(dtype, lengths, count):
    """The grid path (27 bins, or whole short axes) equals a brute-force search of all pairs,
    except for pairs within a few ulp of the radius, where the two roundings may differ."""
    positions, cell = lattice.random_box(count, lengths, seed=11)
    positions = positions.astype(dtype)
    cell = cell.astype(dtype)
    radius = 1.1
    dims = on.grid_dims(cell, radius, dtype)
    assert max(dims) > 3
    grid_first, grid_second, path = on.pairs(positions, cell, radius, dims)
    assert path == "grid"
    brute_first, brute_second, _ = on.pairs(positions, cell, radius, dims=[1, 1, 1])
    grid, brute = on.pair_set(grid_first, grid_second), on.pair_set(brute_first, brute_second)
    assert len(np.unique(grid)) == len(grid)  # each pair once
    differ = np.setxor1d(grid, brute)
    if len(differ):
        i, j = differ >> 32, differ & 0xFFFFFFFF
        d = lj.displacement(positions[i].astype(np.float64), positions[j].astype(np.float64),
                            cell.astype(np.float64))
        r2 = (d * d).sum(axis=1)
        assert np.all(np.abs(r2 - radius * radius) < 64 * np.finfo(dtype).eps)


def test_reuse_rule_threshold():
    positions, cell = lattice.simple_cubic(8, 4.0, 0.02, seed=3)
    cutoff, radius = 1.0, 1.1
    limits = on.grid_dims(cell, radius, np.float64)
    decision, dims = on.reuse(positions, positions, cell, cell, cutoff, radius, limits)
    assert decision == 0 and list(dims) == limits
    moved = positions.copy()
    moved[5, 0] += 0.0499
    assert on.reuse(moved, positions, cell, cell, cutoff, radius, limits)[0] == 0
    moved[5, 0] += 0.0002
    assert on.reuse(moved, positions, cell, cell, cutoff, radius, limits)[0] == 1
    moved[7, 1] = np.nan
    assert on.reuse(moved, positions, cell, cell, cutoff, radius, limits)[0] == -2
    assert on.reuse(positions, positions, np.array([1.9, 4.0, 4.0]), cell, cutoff, radius,
                    limits)[0] == -1
