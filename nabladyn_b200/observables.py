"""Observables of a frame: kinetic energy, temperature and pressure (nm, ps, Da, kJ/mol, K).

The formulas of src/nabladyn/observables.py:18-41.
"""

from torch import Tensor

from .units import BOLTZMANN


def kinetic_energy(velocities: Tensor, masses: Tensor) -> Tensor:
    """K = sum m v^2 / 2 in kJ/mol, for velocities [N, 3] in nm/ps and masses [N] in Da."""
    return 0.5 * (masses[:, None] * velocities.square()).sum()


def temperature(kinetic: Tensor, degrees_of_freedom: int) -> Tensor:
    """T = 2K / (g k_B) in K."""
    return 2.0 * kinetic / (degrees_of_freedom * BOLTZMANN)


def pressure(kinetic: Tensor, virial: Tensor, cell: Tensor) -> Tensor:
    """P = (2K + tr W) / (3V) in kJ/mol/nm^3; divide by ``units.BAR`` for bar."""
    return (2.0 * kinetic + virial.trace()) / (3.0 * cell.prod())


__all__ = ("kinetic_energy", "temperature", "pressure")
