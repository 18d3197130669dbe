"""Lennard-Jones E/F/W on the GPU against the reference's float64 values and the oracle.

Tolerances: float64 to 1e-9 (absolute, kJ/mol and kJ/mol/nm scale); float32 forces to a
relative error of 1e-5 against float64 (||F32 - F64|| / ||F64||), energy
and virial to 1e-5 relative.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import potential, quantity, space
from nabladyn_b200.neighbors import NeighborList, NeighborPairs
from oracle import lj
from oracle import neighbors as on

pytestmark = pytest.mark.gpu

FORCE_RTOL_F32 = 1e-5


def argon_model(n, dtype, device, trainable=()):
    return potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([0.34], dtype=dtype, device=device),
        epsilon=torch.tensor([0.996], dtype=dtype, device=device),
        cutoff=1.0,
        trainable=trainable,
    )


def all_pairs(n, device):
    i, j = torch.triu_indices(n, n, offset=1, device=device)
    return NeighborPairs(torch.stack([i, j]).to(torch.int32), n, 1.0)


def relative(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_argon_float64_matches_reference(argon, cuda):
    x = torch.tensor(argon["positions"], dtype=torch.float64, device=cuda)
    cell = torch.tensor(argon["cell"], dtype=torch.float64, device=cuda)
    model = argon_model(512, torch.float64, cuda)
    energy, forces, virial = quantity.energy_force_virial(model)(x, cell, all_pairs(512, cuda))
    assert float(energy) == pytest.approx(float(argon["energy_f64"]), abs=1e-9)
    np.testing.assert_allclose(forces.cpu().numpy(), argon["forces_f64"], atol=1e-9)
    np.testing.assert_allclose(virial.cpu().numpy(), argon["virial_f64"], atol=1e-8)


def test_argon_float32_within_tolerance_of_float64(argon, cuda):
    x = torch.tensor(argon["positions"], dtype=torch.float32, device=cuda)
    cell = torch.tensor(argon["cell"], dtype=torch.float32, device=cuda)
    model = argon_model(512, torch.float32, cuda)
    neighbor_list = NeighborList(1.0, skin=0.1)
    neighbor_list.allocate(x, cell)
    energy, forces, virial = quantity.energy_force_virial(model)(x, cell, neighbor_list.tensors())
    assert energy.dtype == torch.float32
    assert relative(forces.cpu(), argon["forces_f64"]) < FORCE_RTOL_F32
    assert float(energy) == pytest.approx(float(argon["energy_f64"]), rel=1e-5)
    assert relative(virial.cpu(), argon["virial_f64"]) < 1e-5


def test_two_types_match_reference(lj_frames, cuda):
    n = lj_frames["atom_types"].shape[0]
    model = potential.lennard_jones(
        atom_types=torch.tensor(lj_frames["atom_types"], device=cuda),
        sigma=torch.tensor(lj_frames["sigma"], device=cuda),
        epsilon=torch.tensor(lj_frames["epsilon"], device=cuda),
        cutoff=float(lj_frames["cutoff"]),
    )
    evaluate = quantity.energy_force_virial(model)
    for k in range(len(lj_frames["energy"])):
        x = torch.tensor(lj_frames["positions"][k], device=cuda)
        cell = torch.tensor(lj_frames["cells"][k], device=cuda)
        neighbor_list = NeighborList(float(lj_frames["cutoff"]), skin=0.0)
        neighbor_list.allocate(x, cell)
        energy, forces, virial = evaluate(x, cell, neighbor_list.tensors())
        assert float(energy) == pytest.approx(float(lj_frames["reference_energy"][k]), abs=1e-9)
        np.testing.assert_allclose(forces.cpu().numpy(), lj_frames["reference_forces"][k],
                                   atol=1e-9)
        np.testing.assert_allclose(virial.cpu().numpy(), lj_frames["reference_virial"][k],
                                   atol=1e-8)


def test_torch_func_path_agrees_with_fused(argon, cuda):
    """The generic torch.func route through the model's autograd Function gives the same E/F/W."""
    x = torch.tensor(argon["positions"], dtype=torch.float64, device=cuda)
    cell = torch.tensor(argon["cell"], dtype=torch.float64, device=cuda)
    model = argon_model(512, torch.float64, cuda)
    pairs = all_pairs(512, cuda)
    fused = quantity.energy_force_virial(model)(x, cell, pairs)
    generic = quantity.energy_force_virial(lambda *a, **k: model(*a, **k))(x, cell, pairs)
    for a, b in zip(fused, generic):
        torch.testing.assert_close(a, b, rtol=1e-12, atol=1e-10)
    energy = model(x.requires_grad_(True), cell, pairs)
    (gradient,) = torch.autograd.grad(energy, x)
    torch.testing.assert_close(-gradient, fused[1], rtol=1e-12, atol=1e-10)


def test_strained_energy_and_parameter_gradients(argon, cuda):
    x = torch.tensor(argon["positions"], dtype=torch.float64, device=cuda)
    cell = torch.tensor(argon["cell"], dtype=torch.float64, device=cuda)
    model = argon_model(512, torch.float64, cuda, trainable=("sigma", "epsilon"))
    pairs = all_pairs(512, cuda)
    strain = torch.tensor([[1e-3, 2e-4, 0.0], [0.0, -5e-4, 1e-4], [3e-4, 0.0, 2e-4]],
                          dtype=torch.float64, device=cuda)
    energy = model(x, cell, pairs, strain=strain)
    # Oracle: deform every minimum-image vector, then the plain sum.
    wrapped = on.wrap(argon["positions"], argon["cell"])
    first, second = lj.all_pairs(512)
    d = lj.displacement(wrapped[first], wrapped[second], argon["cell"])
    e = strain.cpu().numpy()
    d = d + d @ e.T
    r2 = (d * d).sum(axis=1)
    r2 = r2[r2 < 1.0]
    p6 = (0.34**2 / r2) ** 3
    pc6 = 0.34**6
    want = float((4 * 0.996 * (p6 * p6 - p6) - 4 * 0.996 * (pc6 * pc6 - pc6)).sum())
    assert float(energy) == pytest.approx(want, abs=1e-8)
    energy = model(x, cell, pairs)
    sigma_grad, epsilon_grad = torch.autograd.grad(energy, (model.sigma, model.epsilon))
    _, _, _, dsigma, depsilon = lj.energy_force_virial(
        wrapped, argon["cell"], first, second, [0.34], [0.996], 1.0, parameter_grads=True,
    )
    np.testing.assert_allclose(sigma_grad.cpu().numpy(), dsigma, rtol=1e-10)
    np.testing.assert_allclose(epsilon_grad.cpu().numpy(), depsilon, rtol=1e-10)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_larger_system_against_oracle(cuda, dtype):
    from nabladyn_b200 import lattice

    positions, cell = lattice.fcc(12, 12 * 0.5745, 0.02, seed=8)  # 6,912 atoms
    x = torch.tensor(positions, dtype=dtype, device=cuda)
    box = torch.tensor(cell, dtype=dtype, device=cuda)
    n = x.shape[0]
    model = argon_model(n, dtype, cuda)
    neighbor_list = NeighborList(1.0, skin=0.1)
    neighbor_list.allocate(x, box)
    energy, forces, virial = quantity.energy_force_virial(model)(x, box, neighbor_list.tensors())
    wrapped = space.wrap(x.double(), box.double())[0].cpu().numpy()
    first, second, _ = on.pairs(wrapped, cell, 1.0)
    e64, f64, w64 = lj.energy_force_virial(wrapped, cell, first, second, [0.34], [0.996], 1.0)
    tolerance = FORCE_RTOL_F32 if dtype == torch.float32 else 1e-12
    assert relative(forces.cpu().double(), f64) < tolerance
    assert float(energy) == pytest.approx(e64, rel=tolerance)
    assert relative(virial.cpu().double(), w64) < tolerance
