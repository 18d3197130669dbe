"""training.fit against the reference's own fit (tests/golden/lj_fit_run.npz, made by its
training.fit on the GPU in float64): the same batches, per-update losses to 1e-9 relative,
fitted sigma and epsilon to 1e-12 relative, and RMS errors before and after to 1e-9."""

import numpy as np
import pytest
import torch

from nabladyn_b200 import potential, training

pytestmark = pytest.mark.gpu


def test_fit_matches_reference_run(cuda):
    fit = dict(np.load("tests/golden/lj_fit_run.npz"))
    data = dict(np.load("tests/golden/lj_frames_4.npz"))
    model = potential.lennard_jones(
        atom_types=torch.tensor(data["atom_types"], device=cuda),
        sigma=torch.tensor(fit["start_sigma"], device=cuda),
        epsilon=torch.tensor(fit["start_epsilon"], device=cuda),
        cutoff=float(data["cutoff"]), trainable=("sigma", "epsilon"))
    train = training.Dataset(data["positions"], data["cells"], energy=data["energy"],
                             forces=data["forces"], virial=data["virial"])
    optimizer = torch.optim.SGD(model.parameters(), lr=1e-7)
    report = training.fit(model, train, optimizer, updates=6, batch_size=3, energy=1.0,
                          forces=1.0, virial=1.0, seed=5)
    np.testing.assert_allclose(report.loss, fit["loss"], rtol=1e-9)
    np.testing.assert_allclose(model.sigma.detach().cpu().numpy(), fit["sigma"], rtol=1e-12)
    np.testing.assert_allclose(model.epsilon.detach().cpu().numpy(), fit["epsilon"], rtol=1e-12)
    channels = ("energy", "forces", "virial")
    np.testing.assert_allclose([report.training[k][0] for k in channels], fit["before"],
                               rtol=1e-9)
    np.testing.assert_allclose([report.training[k][1] for k in channels], fit["after"],
                               rtol=1e-9)
