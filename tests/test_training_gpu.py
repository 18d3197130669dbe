"""The hand-written parameter backward (dLoss/dsigma, dLoss/depsilon through E, F and W).

Checked three ways, in float64: against the reference's own gradient (its training predict and
loss under torch.func, tests/golden/lj_fit_gradient.npz) to 1e-9 relative; against central
finite differences of the loss to 1e-6 relative; and against torch double-backward through a
plain-torch restatement of the Lennard-Jones energy to 1e-9 relative, on a two-type 4,096-atom
system (the differentiation workload's shape, fewer frames).
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice, potential, space, training
from nabladyn_b200.potential import pair_index
from oracle import neighbors as on

pytestmark = pytest.mark.gpu


def two_type_model(types, sigma, epsilon, cutoff, device):
    return potential.lennard_jones(
        atom_types=torch.as_tensor(types, device=device),
        sigma=torch.as_tensor(sigma, dtype=torch.float64, device=device),
        epsilon=torch.as_tensor(epsilon, dtype=torch.float64, device=device),
        cutoff=cutoff, trainable=("sigma", "epsilon"),
    )


def all_pairs_stack(n, frames, device):
    i, j = torch.triu_indices(n, n, offset=1, device=device)
    return torch.stack([i, j]).to(torch.int32)[None].expand(frames, 2, -1).contiguous()


def our_loss_and_gradient(model, positions, cells, stack, labels, scales):
    params = {"sigma": model.sigma.detach().clone().requires_grad_(True),
              "epsilon": model.epsilon.detach().clone().requires_grad_(True)}
    predicted = training.predict(model, params, positions, cells, (stack,),
                                 ("energy", "forces", "virial"))
    value, _ = training.loss(predicted, labels, {"energy": 1.0, "forces": 1.0, "virial": 1.0},
                             scales)
    value.backward()
    return float(value.detach()), params["sigma"].grad, params["epsilon"].grad


def test_gradient_matches_reference(lj_frames, cuda):
    golden = dict(np.load("tests/golden/lj_fit_gradient.npz"))
    n = lj_frames["atom_types"].shape[0]
    model = two_type_model(lj_frames["atom_types"], golden["sigma"], golden["epsilon"],
                           float(lj_frames["cutoff"]), cuda)
    positions = torch.tensor(lj_frames["positions"], device=cuda)
    cells = torch.tensor(lj_frames["cells"], device=cuda)
    labels = {name: torch.tensor(lj_frames[name], device=cuda)
              for name in ("energy", "forces", "virial")}
    scales = dict(zip(("energy", "forces", "virial"), golden["scales"].tolist()))
    stack = all_pairs_stack(n, positions.shape[0], cuda)
    value, dsigma, depsilon = our_loss_and_gradient(model, positions, cells, stack, labels, scales)
    assert value == pytest.approx(float(golden["loss"]), rel=1e-10)
    np.testing.assert_allclose(dsigma.cpu().numpy(), golden["sigma_grad"], rtol=1e-9)
    np.testing.assert_allclose(depsilon.cpu().numpy(), golden["epsilon_grad"], rtol=1e-9)


def torch_energy(positions, cell, index, types, num_types, sigma, epsilon, cutoff, strain):
    """A plain-torch restatement of the shifted LJ energy, differentiable twice."""
    i, j = index[0].long(), index[1].long()
    d = space.strained(space._displacement_wrapped(positions[i], positions[j], cell), strain)
    r2 = d.square().sum(dim=-1)
    valid = (i != j) & (r2 < cutoff**2)
    safe = torch.where(valid, r2, torch.ones_like(r2))
    rows = pair_index(types[i], types[j], num_types)
    s, e = sigma[rows], epsilon[rows]
    p6 = (s * s / safe) ** 3
    pc6 = (s * s / cutoff**2) ** 3
    u = 4 * e * (p6 * p6 - p6) - 4 * e * (pc6 * pc6 - pc6)
    return torch.where(valid, u, torch.zeros_like(u)).sum()


def torch_double_backward(model, positions, cells, stack, labels, scales):
    sigma = model.sigma.detach().clone().requires_grad_(True)
    epsilon = model.epsilon.detach().clone().requires_grad_(True)
    energies, forces, virials = [], [], []
    for f in range(positions.shape[0]):
        x = space.wrap(positions[f], cells[f])[0].detach().requires_grad_(True)
        strain = torch.zeros((3, 3), dtype=x.dtype, device=x.device, requires_grad=True)
        e = torch_energy(x, cells[f], stack[f], model.atom_types, model.num_types, sigma,
                         epsilon, model.cutoff, strain)
        gx, gs = torch.autograd.grad(e, (x, strain), create_graph=True)
        energies.append(e)
        forces.append(-gx)
        virials.append(-gs)
    predicted = {"energy": torch.stack(energies), "forces": torch.stack(forces),
                 "virial": torch.stack(virials)}
    value, _ = training.loss(predicted, labels, {"energy": 1.0, "forces": 1.0, "virial": 1.0},
                             scales)
    dsigma, depsilon = torch.autograd.grad(value, (sigma, epsilon))
    return float(value), dsigma, depsilon


def test_gradient_matches_torch_double_backward_and_finite_differences(cuda):
    rng = np.random.default_rng(41)
    cells_per_side = 10  # 4,000 atoms at rho ~ 21, two types 50/50
    n = 4 * cells_per_side**3
    length = (n / 21.0) ** (1 / 3)
    frames = 3
    types = rng.permutation(np.arange(n) % 2).astype(np.int64)
    target_sigma, target_epsilon = [0.34, 0.32, 0.30], [0.996, 0.8, 0.6]
    start = rng.uniform(0.9, 1.1, 6)
    positions = np.stack([lattice.fcc(cells_per_side, length, 0.03, seed=50 + f)[0]
                          for f in range(frames)])
    cells = np.full((frames, 3), length)
    x = torch.tensor(positions, device=cuda)
    box = torch.tensor(cells, device=cuda)
    stack = training.pair_stack(x, box, 1.0)
    target = two_type_model(types, target_sigma, target_epsilon, 1.0, cuda)
    with torch.no_grad():
        labels = training.predict(target, {}, x, box, (stack,), ("energy", "forces", "virial"))
    labels = {k: v.detach() + 0.01 * torch.randn_like(v) for k, v in labels.items()}
    scales = training.scales(**labels)
    model = two_type_model(types, np.array(target_sigma) * start[:3],
                           np.array(target_epsilon) * start[3:], 1.0, cuda)
    value, dsigma, depsilon = our_loss_and_gradient(model, x, box, stack, labels, scales)
    reference = torch_double_backward(model, x, box, stack, labels, scales)
    assert value == pytest.approx(reference[0], rel=1e-10)
    np.testing.assert_allclose(dsigma.cpu().numpy(), reference[1].cpu().numpy(), rtol=1e-9)
    np.testing.assert_allclose(depsilon.cpu().numpy(), reference[2].cpu().numpy(), rtol=1e-9)
    # Central differences of our forward, row by row.
    for name, grad in (("sigma", dsigma), ("epsilon", depsilon)):
        base = getattr(model, name).detach()
        for row in range(3):
            h = 1e-6 * float(base[row])
            values = []
            for sign in (1, -1):
                shifted = base.clone()
                shifted[row] += sign * h
                with torch.no_grad():
                    predicted = training.predict(model, {name: shifted}, x, box, (stack,),
                                                 ("energy", "forces", "virial"))
                    values.append(float(training.loss(
                        predicted, labels, {"energy": 1.0, "forces": 1.0, "virial": 1.0},
                        scales)[0]))
            numeric = (values[0] - values[1]) / (2 * h)
            assert float(grad[row]) == pytest.approx(numeric, rel=1e-6, abs=1e-8)


def test_pair_stack_rows_are_the_oracle_pairs(cuda):
    frames = [lattice.fcc(8, 8 * 0.5745, 0.04, seed=60 + f)[0] for f in range(3)]
    cell = np.full(3, 8 * 0.5745)
    x = torch.tensor(np.stack(frames), device=cuda)
    box = torch.tensor(np.stack([cell] * 3), device=cuda)
    stack = training.pair_stack(x, box, 1.0).cpu().numpy()
    assert stack.shape[2] == training.width(stack.shape[2])
    for f in range(3):
        wrapped = space.wrap(x[f], box[f])[0].cpu().numpy()
        first, second, _ = on.pairs(wrapped, cell, 1.0)
        real = stack[f, 0] != stack[f, 1]
        np.testing.assert_array_equal(on.pair_set(stack[f, 0, real], stack[f, 1, real]),
                                      on.pair_set(first, second))
