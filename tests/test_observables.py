"""kinetic_energy, temperature and pressure against the reference's own values
(tests/golden/observables.npz, made by its src/nabladyn/observables.py:18-41 in float64)."""

import numpy as np
import pytest
import torch

from nabladyn_b200 import observables, units

GOLDEN = dict(np.load("tests/golden/observables.npz"))
CASES = sorted({key.split(":")[0] for key in GOLDEN})


@pytest.mark.parametrize("case", CASES)
def test_observables_match_reference(case):
    g = {key.split(":")[1]: torch.tensor(value) for key, value in GOLDEN.items()
         if key.startswith(f"{case}:")}
    n = g["velocities"].shape[0]
    kinetic = observables.kinetic_energy(g["velocities"], g["masses"])
    assert float(kinetic) == pytest.approx(float(g["kinetic"]), rel=1e-14)
    assert float(observables.temperature(kinetic, max(3 * n - 3, 1))) == pytest.approx(
        float(g["temperature"]), rel=1e-14)
    assert float(observables.pressure(kinetic, g["virial"], g["cell"])) == pytest.approx(
        float(g["pressure"]), rel=1e-14)


def test_pressure_units_and_float32():
    """Pressure in bar through units.BAR, and float32 inputs within float32 rounding."""
    g = {key.split(":")[1]: torch.tensor(value) for key, value in GOLDEN.items()
         if key.startswith("2:")}
    kinetic = observables.kinetic_energy(g["velocities"].float(), g["masses"].float())
    p32 = observables.pressure(kinetic, g["virial"].float(), g["cell"].float())
    assert p32.dtype == torch.float32
    assert float(p32) == pytest.approx(float(g["pressure"]), rel=1e-5)
    assert float(p32 / units.BAR) == pytest.approx(float(g["pressure"]) / units.BAR, rel=1e-5)
