"""The SchNet training gradient on the B200: the fused kernels with the tcgen05 tangent passes
(nd_schnet_tangent) against the float64 oracle's hand-written second-order gradient, the
reference's own loss and gradient, and the torch.func algorithm run on the same GPU.

The per-pair products take BF16 operands (FP32 accumulation) and the message sums are FP32
atomics, so the gradient carries BF16-level errors. Bounds, per parameter tensor, on
||g - g64|| / ||g64||: GRAD_TOL; on the loss, relative: LOSS_TOL.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import lattice, potential, training
from nabladyn_b200.training import _generic, _schnet_gradient
from oracle import schnet as oracle

pytestmark = pytest.mark.gpu

GRAD_TOL, LOSS_TOL = 1.5e-2, 1e-2
CHANNELS = ("energy", "forces", "virial")


def relative(ours, reference):
    reference = np.asarray(reference, dtype=np.float64)
    return float(np.linalg.norm(np.asarray(ours, dtype=np.float64) - reference)
                 / max(np.linalg.norm(reference), 1e-300))


@pytest.fixture(scope="module")
def fixture():
    golden = dict(np.load("tests/golden/schnet_343.npz"))
    fit = dict(np.load("tests/golden/schnet_fit_gradient.npz"))
    return golden, fit


def fused_gradient(cuda, golden, fit):
    n = golden["positions"].shape[0]
    model = potential.schnet(atom_types=torch.tensor(golden["atom_types"], device=cuda),
                             num_types=2, cutoff=1.2, trainable=True)
    assert _schnet_gradient.supported(model)
    first, second = np.triu_indices(n, 1)
    frames = fit["positions"].shape[0]
    stack = torch.tensor(np.stack([first, second]), dtype=torch.int32,
                         device=cuda)[None].expand(frames, 2, -1).contiguous()
    labels = {name: torch.tensor(fit[f"label:{name}"], dtype=torch.float32, device=cuda)
              for name in CHANNELS}
    scales = dict(zip(CHANNELS, fit["scales"].tolist()))
    params = {k: v.detach().clone() for k, v in model.named_parameters()}
    value, gradient = training.loss_and_gradient(
        model, params, torch.tensor(fit["positions"], dtype=torch.float32, device=cuda),
        torch.tensor(fit["cells"], dtype=torch.float32, device=cuda), (stack,), labels,
        dict.fromkeys(CHANNELS, 1.0), scales)
    return float(value), {k: v.cpu().numpy() for k, v in gradient.items()}


def oracle_gradient(golden, fit):
    n = golden["positions"].shape[0]
    first, second = np.triu_indices(n, 1)
    weights = {k[len("weight:"):]: v for k, v in golden.items() if k.startswith("weight:")}
    scales = dict(zip(CHANNELS, fit["scales"].tolist()))
    frames = fit["positions"].shape[0]
    total, gradient = 0.0, None
    for f in range(frames):
        cell = fit["cells"][f]
        x = fit["positions"][f] % cell
        e, forces, virial = oracle.energy_force_virial(x, cell, first, second,
                                                       golden["atom_types"], weights, 1.2, 50, 3)
        labels = {name: fit[f"label:{name}"][f] for name in CHANNELS}
        value, e_bar, f_bar, w_bar = oracle.loss_adjoints(
            {"energy": e, "forces": forces, "virial": virial}, labels,
            dict.fromkeys(CHANNELS, 1.0), scales, 1.0 / frames)
        total += value
        part = oracle.loss_parameter_gradient(x, cell, first, second, golden["atom_types"],
                                              weights, 1.2, 50, 3, e_bar, f_bar, w_bar)
        gradient = part if gradient is None else {k: gradient[k] + part[k] for k in part}
    return total, gradient


def test_fused_gradient_matches_oracle_and_reference(cuda, fixture):
    """343 beads, all pairs, three frames, loss over E, F and W: every parameter's gradient
    against the float64 oracle, and the four the reference's fixture holds against it."""
    golden, fit = fixture
    value, gradient = fused_gradient(cuda, golden, fit)
    expected_value, expected = oracle_gradient(golden, fit)
    assert value == pytest.approx(float(fit["loss"]), rel=LOSS_TOL)
    assert expected_value == pytest.approx(float(fit["loss"]), rel=1e-10)
    errors = {name: relative(gradient[name], expected[name]) for name in expected}
    print("relative gradient errors:", {k: f"{v:.2e}" for k, v in errors.items()})
    assert max(errors.values()) <= GRAD_TOL, errors
    for key in fit:
        if key.startswith("grad:"):
            name = key[len("grad:"):]
            assert relative(gradient[name], fit[key]) <= GRAD_TOL, name


def test_fused_gradient_repeats(cuda, fixture):
    """Two calls in a row agree to the atomics' summation order (BF16 level)."""
    golden, fit = fixture
    value_a, first = fused_gradient(cuda, golden, fit)
    value_b, second = fused_gradient(cuda, golden, fit)
    assert value_a == pytest.approx(value_b, rel=1e-3)
    for name in first:
        assert relative(second[name], first[name]) <= GRAD_TOL / 2, name


def test_fused_gradient_matches_torch_func_on_listed_pairs(cuda):
    """4,096 beads, two frames over a neighbor-list pair stack (padding columns included),
    energy and forces only: the fused gradient against the reference's torch.func algorithm
    on the same float32 model."""
    n_side, frames = 16, 2
    n = n_side**3
    length = (n / 10.0) ** (1.0 / 3.0)
    positions = torch.tensor(np.stack([
        lattice.simple_cubic(n_side, length, 0.03, seed=70 + f)[0] % length
        for f in range(frames)]), dtype=torch.float32, device=cuda)
    cells = torch.full((frames, 3), length, dtype=torch.float32, device=cuda)
    stack = training.pair_stack(positions, cells, 1.2)
    types = torch.tensor(np.random.default_rng(3).integers(0, 2, n), device=cuda)
    teacher = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, seed=1)
    model = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, trainable=True)
    predicted = training.predict(teacher, {}, positions, cells, (stack,), ("energy", "forces"))
    labels = {k: v.detach() for k, v in predicted.items()}
    scales = training.scales(**labels)
    weights = {"energy": 1.0, "forces": 1.0}
    params = {k: v.detach().clone() for k, v in model.named_parameters()}
    value, gradient = training.loss_and_gradient(model, params, positions, cells, (stack,),
                                                 labels, weights, scales)
    expected_value, expected = _generic.torch_func_loss_and_gradient(
        model, params, positions, cells, (stack,), labels, weights, scales, chunk=1)
    assert float(value) == pytest.approx(float(expected_value), rel=LOSS_TOL)
    errors = {name: relative(gradient[name].cpu().numpy(), expected[name].cpu().numpy())
              for name in expected}
    print("relative gradient errors:", {k: f"{v:.2e}" for k, v in errors.items()})
    assert max(errors.values()) <= GRAD_TOL, errors


def test_fit_on_fused_gradient(cuda, fixture):
    """training.fit with a float32 SchNet on the GPU runs on the fused gradient: four Adam
    updates over the fixture's three frames, finite losses, every trained parameter moved."""
    golden, fit = fixture
    model = potential.schnet(atom_types=torch.tensor(golden["atom_types"], device=cuda),
                             num_types=2, cutoff=1.2, trainable=True)
    before = {k: v.detach().clone() for k, v in model.named_parameters()}
    data = training.Dataset(fit["positions"].astype(np.float32), fit["cells"].astype(np.float32),
                            energy=fit["label:energy"].astype(np.float32),
                            forces=fit["label:forces"].astype(np.float32),
                            virial=fit["label:virial"].astype(np.float32))
    optimizer = torch.optim.Adam(model.parameters(), lr=1e-3)
    report = training.fit(model, data, optimizer, updates=4, batch_size=2, energy=1.0,
                          forces=1.0, virial=1.0, seed=3)
    assert report.loss.shape == (4,) and np.isfinite(report.loss).all()
    for name, value in model.named_parameters():
        assert not torch.equal(value.detach(), before[name]), name


def compare_with_torch_func(cuda, model, positions, cells, stack, labels, weights):
    scales = training.scales(**labels)
    params = {k: v.detach().clone() for k, v in model.named_parameters()}
    value, gradient = training.loss_and_gradient(model, params, positions, cells, (stack,),
                                                 labels, weights, scales)
    expected_value, expected = _generic.torch_func_loss_and_gradient(
        model, params, positions, cells, (stack,), labels, weights, scales, chunk=1)
    assert float(value) == pytest.approx(float(expected_value), rel=LOSS_TOL)
    errors = {name: relative(gradient[name].cpu().numpy(), expected[name].cpu().numpy())
              for name in expected if float(expected[name].abs().max()) > 0}
    assert max(errors.values()) <= GRAD_TOL, errors
    for name in expected:
        if float(expected[name].abs().max()) == 0:
            assert float(gradient[name].abs().max()) == 0, name


@pytest.mark.parametrize("gaussians, weights", [
    (64, {"energy": 1.0, "forces": 1.0, "virial": 1.0}),  # no spare basis column
    (50, {"energy": 1.0}),
    (50, {"forces": 2.0}),
    (50, {"virial": 0.5}),
])
def test_fused_gradient_sizes_and_channels(cuda, fixture, gaussians, weights):
    """The 343-bead frames with 64 Gaussians (the filter1 bias summed apart) and with losses
    over one channel, against the torch.func algorithm on the same float32 model."""
    golden, fit = fixture
    n = golden["positions"].shape[0]
    types = torch.tensor(golden["atom_types"], device=cuda)
    model = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, gaussians=gaussians,
                             trainable=True)
    teacher = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, gaussians=gaussians,
                               seed=1)
    positions = torch.tensor(fit["positions"], dtype=torch.float32, device=cuda)
    cells = torch.tensor(fit["cells"], dtype=torch.float32, device=cuda)
    first, second = np.triu_indices(n, 1)
    stack = torch.tensor(np.stack([first, second]), dtype=torch.int32,
                         device=cuda)[None].expand(positions.shape[0], 2, -1).contiguous()
    channels = tuple(name for name in CHANNELS if name in weights)
    predicted = training.predict(teacher, {}, positions, cells, (stack,), channels)
    labels = {k: v.detach() for k, v in predicted.items()}
    compare_with_torch_func(cuda, model, positions, cells, stack, labels, weights)


def test_fused_gradient_without_pairs(cuda):
    """Eight beads 2 nm apart in a 16 nm box: no pair within the cutoff, so only the
    embedding, the atom-wise layers and the readout carry gradient; padding columns only."""
    grid = np.stack(np.meshgrid(*[np.arange(2)] * 3, indexing="ij"), -1).reshape(-1, 3)
    positions = torch.tensor(2.0 * grid + 1.0, dtype=torch.float32, device=cuda)[None]
    cells = torch.full((1, 3), 16.0, dtype=torch.float32, device=cuda)
    first, second = np.triu_indices(8, 1)
    stack = torch.tensor(np.stack([first, second]), dtype=torch.int32, device=cuda)[None]
    types = torch.tensor([0, 1] * 4, device=cuda)
    model = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, trainable=True)
    labels = {"energy": torch.tensor([0.5], device=cuda),
              "forces": torch.zeros((1, 8, 3), device=cuda)}
    compare_with_torch_func(cuda, model, positions, cells, stack, labels,
                            {"energy": 1.0, "forces": 1.0})


def test_model_copies_after_fused_gradient(cuda, fixture):
    """The gradient's buffers and graph live beside the model: it still deep-copies, and the
    copy's gradient equals the original's to the atomics' summation order."""
    import copy

    golden, fit = fixture
    model = potential.schnet(atom_types=torch.tensor(golden["atom_types"], device=cuda),
                             num_types=2, cutoff=1.2, trainable=True)
    n = golden["positions"].shape[0]
    i, j = np.triu_indices(n, 1)
    stack = torch.tensor(np.stack([i, j]), dtype=torch.int32, device=cuda)[None].contiguous()
    positions = torch.tensor(fit["positions"][:1], dtype=torch.float32, device=cuda)
    cells = torch.tensor(fit["cells"][:1], dtype=torch.float32, device=cuda)
    labels = {"energy": torch.tensor(fit["label:energy"][:1], dtype=torch.float32, device=cuda)}
    args = (positions, cells, (stack,), labels, {"energy": 1.0}, {"energy": 1.0})
    params = {k: v.detach().clone() for k, v in model.named_parameters()}
    value, gradient = training.loss_and_gradient(model, params, *args)
    twin = copy.deepcopy(model)
    twin_params = {k: v.detach().clone() for k, v in twin.named_parameters()}
    twin_value, twin_gradient = training.loss_and_gradient(twin, twin_params, *args)
    assert float(twin_value) == pytest.approx(float(value), rel=1e-6)
    for name in gradient:
        assert relative(twin_gradient[name].cpu().numpy(),
                        gradient[name].cpu().numpy()) <= GRAD_TOL / 2, name


def test_fit_matches_torch_func_fit(cuda, fixture, monkeypatch):
    """training.fit, four plain SGD updates over the fixture's frames, on the fused gradient
    against the same fit on the reference's torch.func gradient (same start, seed and batches):
    the losses and every parameter tensor's total change agree to the gradient's bound."""
    golden, fit = fixture
    types = torch.tensor(golden["atom_types"], device=cuda)
    data = training.Dataset(fit["positions"].astype(np.float32), fit["cells"].astype(np.float32),
                            energy=fit["label:energy"].astype(np.float32),
                            forces=fit["label:forces"].astype(np.float32),
                            virial=fit["label:virial"].astype(np.float32))

    def run(fused: bool):
        model = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, trainable=True)
        start = {k: v.detach().clone() for k, v in model.named_parameters()}
        optimizer = torch.optim.SGD(model.parameters(), lr=1e-8)
        with monkeypatch.context() as patch:
            if not fused:
                patch.setattr(_schnet_gradient, "supported", lambda m: False)
            report = training.fit(model, data, optimizer, updates=4, batch_size=2, energy=1.0,
                                  forces=1.0, virial=1.0, seed=3)
        change = {k: (v.detach() - start[k]).double().cpu().numpy()
                  for k, v in model.named_parameters()}
        return report, change

    fused_report, fused_change = run(True)
    reference_report, reference_change = run(False)
    np.testing.assert_allclose(fused_report.loss, reference_report.loss, rtol=LOSS_TOL)
    errors = {name: relative(fused_change[name], reference_change[name])
              for name in reference_change}
    assert max(errors.values()) <= GRAD_TOL, errors
