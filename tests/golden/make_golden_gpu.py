"""Generate the golden fixtures that need the reference's CUDA code, on a GPU machine.

The reference's training.fit builds its pair stacks with its CUDA-only NeighborList, so this
runs where a GPU is present and the reference is installed (default baseline/_ref; override
with NABLADYN_REFERENCE_PACKAGE): ``python tests/golden/make_golden_gpu.py``. Fixture:

* lj_fit_run.npz — the reference's own training.fit (float64) on the four frames of
  lj_frames_4.npz from perturbed parameters: 6 SGD updates of batch 3 (seed 5), with its
  per-update losses, the fitted sigma and epsilon, and its RMS errors before and after.
"""

import os
import sys
from pathlib import Path

import numpy as np
import torch

OUT = Path(__file__).resolve().parent
PACKAGE = Path(os.environ.get("NABLADYN_REFERENCE_PACKAGE",
                              OUT.parent.parent / "baseline" / "_ref"))
sys.path.insert(0, str(PACKAGE))

from nabladyn import potential, training  # noqa: E402

CHANNELS = ("energy", "forces", "virial")


def lj_fit_run() -> None:
    device = torch.device("cuda", 0)
    data = np.load(OUT / "lj_frames_4.npz")
    sigma = data["sigma"] * np.array([1.05, 0.97, 1.02])
    epsilon = data["epsilon"] * np.array([0.9, 1.1, 0.95])
    model = potential.lennard_jones(
        atom_types=torch.tensor(data["atom_types"], device=device),
        sigma=torch.tensor(sigma, device=device), epsilon=torch.tensor(epsilon, device=device),
        cutoff=float(data["cutoff"]), trainable=("sigma", "epsilon"))
    train = training.Dataset(data["positions"], data["cells"], energy=data["energy"],
                             forces=data["forces"], virial=data["virial"])
    optimizer = torch.optim.SGD(model.parameters(), lr=1e-7)
    report = training.fit(model, train, optimizer, updates=6, batch_size=3, energy=1.0,
                          forces=1.0, virial=1.0, seed=5)
    np.savez_compressed(
        OUT / "lj_fit_run.npz", start_sigma=sigma, start_epsilon=epsilon,
        sigma=model.sigma.detach().cpu().numpy(), epsilon=model.epsilon.detach().cpu().numpy(),
        loss=np.asarray(report.loss),
        before=np.array([report.training[k][0] for k in CHANNELS]),
        after=np.array([report.training[k][1] for k in CHANNELS]))


if __name__ == "__main__":
    lj_fit_run()
    print("wrote lj_fit_run.npz")
