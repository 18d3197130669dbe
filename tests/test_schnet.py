"""SchNet on the CPU: the float64 oracle against the reference's own numbers, the model's
seeded weights against the reference's, and the parameter block's layout.

The fixture tests/golden/schnet_343.npz holds the reference's SchNet (seed 0, 64 features,
3 blocks, 50 Gaussians, cutoff 1.2 nm) evaluated by its quantity.energy_force_virial on 343
beads, and its weights under its state-dict names.
"""

import numpy as np
import pytest
import torch

from nabladyn_b200 import potential, quantity
from nabladyn_b200.neighbors import NeighborPairs
from nabladyn_b200.potential import _schnet_kernels
from oracle import schnet as oracle

GOLDEN = "tests/golden/schnet_343.npz"


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def weights_of(golden, prefix="weight:"):
    return {k[len(prefix):]: v for k, v in golden.items() if k.startswith(prefix)}


def test_oracle_matches_reference(golden):
    n = golden["positions"].shape[0]
    first, second = np.triu_indices(n, 1)
    e, f, w = oracle.energy_force_virial(golden["positions"], golden["cell"], first, second,
                                         golden["atom_types"], weights_of(golden), 1.2, 50, 3)
    assert e == pytest.approx(float(golden["energy64"]), rel=1e-12)
    np.testing.assert_allclose(f, golden["forces64"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(w, golden["virial64"], rtol=1e-10, atol=1e-9)


def test_seeded_weights_match_reference(golden):
    types = torch.tensor(golden["atom_types"])
    model = potential.schnet(atom_types=types, num_types=2, cutoff=1.2, dtype=torch.float64)
    ours = model.state_dict()
    reference = weights_of(golden)
    assert sorted(ours) == sorted(reference)
    for name, value in reference.items():
        np.testing.assert_array_equal(ours[name].numpy(), value, err_msg=name)
    one = potential.schnet(atom_types=torch.zeros(4, dtype=torch.int64), num_types=1,
                           cutoff=1.2, dtype=torch.float64).state_dict()
    for name, value in weights_of(golden, "weight1:").items():
        np.testing.assert_array_equal(one[name].numpy(), value, err_msg=name)


def test_torch_definition_matches_reference(golden):
    """The model's own definition (the torch.func path float64 models take)."""
    n = golden["positions"].shape[0]
    model = potential.schnet(atom_types=torch.tensor(golden["atom_types"]), num_types=2,
                             cutoff=1.2, dtype=torch.float64)
    first, second = np.triu_indices(n, 1)
    pairs = NeighborPairs(torch.tensor(np.stack([first, second]), dtype=torch.int32), n, 1.2)
    e, f, w = quantity.energy_force_virial(model)(
        torch.tensor(golden["positions"]), torch.tensor(golden["cell"]), pairs)
    assert float(e) == pytest.approx(float(golden["energy64"]), rel=1e-12)
    np.testing.assert_allclose(f.numpy(), golden["forces64"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(w.numpy(), golden["virial64"], rtol=1e-10, atol=1e-9)


def test_parameter_block_layout(golden):
    model = potential.schnet(atom_types=torch.tensor(golden["atom_types"]), num_types=2,
                             cutoff=1.2)
    blob = _schnet_kernels.pack(model)
    assert blob.numel() == _schnet_kernels.weight_bytes(3, 2)
    images = blob[: 3 * 10 * 8192].view(torch.bfloat16).reshape(3, 10, 4096).float()
    w = model.blocks[1].filter2.weight.detach().to(torch.bfloat16).float()
    for row, k in ((0, 0), (5, 9), (17, 63), (63, 40)):
        offset = (row // 8) * 512 + (k // 8) * 64 + (row % 8) * 8 + k % 8
        assert images[1, 1, offset] == w[row, k]          # filter2
        assert images[1, 2, offset] == w[k, row]          # filter2^T
    b1 = model.blocks[0].filter1.weight.detach().to(torch.bfloat16).float()
    for row, k in ((3, 49), (3, 50), (63, 63)):
        offset = (row // 8) * 512 + (k // 8) * 64 + (row % 8) * 8 + k % 8
        assert images[0, 0, offset] == (b1[row, k] if k < 50 else 0.0)    # filter1
        assert images[0, 3, offset] == (b1[k, row] if row < 50 else 0.0)   # filter1^T
    assert _schnet_kernels.workspace_bytes(343, 58653, 3) > 0


def test_training_gradient_matches_reference(golden):
    """The SchNet training step (the reference's torch.func algorithm, run here in chunks of
    two frames) against the reference's own loss and gradient on three frames."""
    from nabladyn_b200 import training

    fit = dict(np.load("tests/golden/schnet_fit_gradient.npz"))
    n = golden["positions"].shape[0]
    model = potential.schnet(atom_types=torch.tensor(golden["atom_types"]), num_types=2,
                             cutoff=1.2, trainable=True, dtype=torch.float64)
    first, second = np.triu_indices(n, 1)
    stack = torch.tensor(np.stack([first, second]), dtype=torch.int32)[None].expand(3, 2, -1)
    labels = {name: torch.tensor(fit[f"label:{name}"]) for name in ("energy", "forces", "virial")}
    scales = dict(zip(("energy", "forces", "virial"), fit["scales"].tolist()))
    params = {k: v.detach().clone() for k, v in model.named_parameters()}
    value, gradient = training.loss_and_gradient(
        model, params, torch.tensor(fit["positions"]), torch.tensor(fit["cells"]),
        (stack.contiguous(),), labels, {"energy": 1.0, "forces": 1.0, "virial": 1.0}, scales,
        chunk=2)
    assert float(value) == pytest.approx(float(fit["loss"]), rel=1e-10)
    for key in fit:
        if key.startswith("grad:"):
            name = key[len("grad:"):]
            np.testing.assert_allclose(gradient[name].numpy(), fit[key], rtol=1e-8,
                                       atol=1e-8 * np.abs(fit[key]).max(), err_msg=name)


def test_oracle_parameter_gradient_matches_reference(golden):
    """The oracle's hand-written second-order parameter gradient (forward-over-reverse along
    the loss's force and virial adjoints), summed over three frames, against the reference's
    own torch.func loss and gradient."""
    fit = dict(np.load("tests/golden/schnet_fit_gradient.npz"))
    n = golden["positions"].shape[0]
    first, second = np.triu_indices(n, 1)
    weights = weights_of(golden)
    scales = dict(zip(("energy", "forces", "virial"), fit["scales"].tolist()))
    channel_weights = {"energy": 1.0, "forces": 1.0, "virial": 1.0}
    frames = fit["positions"].shape[0]
    total, gradient = 0.0, None
    for f in range(frames):
        cell = fit["cells"][f]
        x = fit["positions"][f] % cell
        e, forces, virial = oracle.energy_force_virial(x, cell, first, second,
                                                       golden["atom_types"], weights, 1.2, 50, 3)
        labels = {name: fit[f"label:{name}"][f] for name in ("energy", "forces", "virial")}
        value, e_bar, f_bar, w_bar = oracle.loss_adjoints(
            {"energy": e, "forces": forces, "virial": virial}, labels, channel_weights, scales,
            1.0 / frames)
        total += value
        part = oracle.loss_parameter_gradient(x, cell, first, second, golden["atom_types"],
                                              weights, 1.2, 50, 3, e_bar, f_bar, w_bar)
        gradient = part if gradient is None else {k: gradient[k] + part[k] for k in part}
    assert total == pytest.approx(float(fit["loss"]), rel=1e-10)
    for key in fit:
        if key.startswith("grad:"):
            name = key[len("grad:"):]
            np.testing.assert_allclose(gradient[name], fit[key], rtol=1e-8,
                                       atol=1e-8 * np.abs(fit[key]).max(), err_msg=name)


def test_atom_parameter_block_layout():
    """The FP32 atom-side parameter block the training kernels read (every block's A, D1, d1,
    D2, d2, then the readout and the embedding) has the library's size, and the gradient views
    over the same layout land on exactly those parameters."""
    from nabladyn_b200 import _native
    from nabladyn_b200.training import _schnet_gradient

    model = potential.schnet(atom_types=torch.tensor([0, 1, 1]), num_types=2, cutoff=1.2,
                             trainable=True)
    values = {name: value.detach() for name, value in model.named_parameters()}
    block = _schnet_gradient.atom_parameters(values, 3)
    assert block.numel() == _native.lib().nd_schnet_atom_parameter_floats(3, 2)
    views = _schnet_gradient.atom_gradient_views(block, 3)
    for name, view in views.items():
        assert torch.equal(view, values[name].float()), name
    covered = set(views)
    assert covered == {name for name in values if "filter" not in name}


@pytest.mark.parametrize("channels", [("energy",), ("forces",), ("virial",),
                                      ("energy", "forces", "virial")])
def test_frame_loss_adjoints_match_oracle(channels):
    """The fused gradient's per-frame loss term and its adjoints dL/dE, dL/dF, dL/dW (the
    inputs of the tangent passes) against the oracle's restatement of the reference's loss."""
    from nabladyn_b200.training import _schnet_gradient

    rng = np.random.default_rng(5)
    n = 11
    predicted = {"energy": rng.normal(), "forces": rng.normal(size=(n, 3)),
                 "virial": rng.normal(size=(3, 3))}
    labels = {"energy": rng.normal(), "forces": rng.normal(size=(n, 3)),
              "virial": rng.normal(size=(3, 3))}
    weights = {name: float(w) for name, w in zip(channels, (0.5, 2.0, 1.5))}
    scales = {"energy": 3.0, "forces": 0.7, "virial": 5.0}
    coefficient = 0.25
    device_scalar = lambda v: torch.tensor(v, dtype=torch.float64)  # noqa: E731
    value, e_bar, f_bar, w_bar = _schnet_gradient._frame_loss(
        torch.tensor(predicted["energy"], dtype=torch.float64),
        torch.tensor(predicted["forces"], dtype=torch.float32),
        torch.tensor(predicted["virial"].reshape(9), dtype=torch.float64),
        {name: torch.tensor(labels[name], dtype=torch.float64) for name in channels},
        {name: device_scalar(w) for name, w in weights.items()},
        {name: device_scalar(scales[name]) for name in channels}, device_scalar(coefficient))
    forces32 = torch.tensor(predicted["forces"], dtype=torch.float32).double().numpy()
    expected = oracle.loss_adjoints({**predicted, "forces": forces32}, labels, weights, scales,
                                    coefficient)
    assert float(value) == pytest.approx(expected[0], rel=1e-12)
    assert float(e_bar) == pytest.approx(expected[1], rel=1e-12, abs=1e-15)
    np.testing.assert_allclose(f_bar.double().numpy(), expected[2], rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(w_bar.numpy().reshape(3, 3), expected[3], rtol=1e-12, atol=1e-15)
