"""ORACLE (test infrastructure): velocity Verlet and the Nose-Hoover chain in float64 numpy.

Restates src/nabladyn/md/_ensembles/_verlet.py:8-31 (half kick, drift + wrap),
_nve.py:39-58, _nvt.py:88-129 and _chain.py:30-83 (MTK chain of three, masses g kT tau^2,
kT tau^2, kT tau^2), with forces from oracle.lj over all pairs.
"""

from __future__ import annotations

import math

import numpy as np

from . import lj
from .neighbors import wrap

BOLTZMANN = 0.00831446261815324


def chain_half_step(kinetic, q, p, mass, degrees, kT, dt):
    """One half step of the chain; returns (factor, q, p)."""
    q, p = np.array(q, dtype=np.float64), np.array(p, dtype=np.float64)
    quarter, eighth = 0.25 * dt, 0.125 * dt

    def driving(k, energy):
        return 2.0 * energy - degrees * kT if k == 0 else p[k - 1] ** 2 / mass[k - 1] - kT

    damping = [0.0, 0.0]
    for k in (2, 1, 0):
        if k == 2:
            p[k] += quarter * driving(k, kinetic)
        else:
            p[k] = damping[k] * (damping[k] * p[k] + quarter * driving(k, kinetic))
        if k > 0:
            damping[k - 1] = math.exp(-eighth * p[k] / mass[k])
    factor = math.exp(-0.5 * dt * p[0] / mass[0])
    kinetic = kinetic * factor * factor
    q = q + 0.5 * dt * p / mass
    for k in (0, 1, 2):
        if k == 2:
            p[k] += quarter * driving(k, kinetic)
        else:
            p[k] = damping[k] * (damping[k] * p[k] + quarter * driving(k, kinetic))
    return factor, q, p


def run(positions, velocities, masses, cell, sigma, epsilon, cutoff, dt, steps,
        temperature=None, timescale=None, evaluate=None):
    """float64 NVE (or NVT when ``temperature`` is given) from a frame; returns the final frame.

    Forces are Lennard-Jones over all pairs, or ``evaluate(x) -> (energy, forces)`` of wrapped
    positions when given (any other potential's oracle).
    """
    x = wrap(np.asarray(positions, dtype=np.float64), np.asarray(cell, dtype=np.float64))
    v = np.asarray(velocities, dtype=np.float64).copy()
    m = np.asarray(masses, dtype=np.float64)
    v = v - (m[:, None] * v).sum(axis=0) / m.sum()
    n = x.shape[0]
    first, second = lj.all_pairs(n)
    if evaluate is None:
        def evaluate(frame):
            e, forces, _ = lj.energy_force_virial(frame, cell, first, second, sigma, epsilon,
                                                  cutoff)
            return e, forces
    _, f = evaluate(x)
    thermostat = temperature is not None
    if thermostat:
        kT = BOLTZMANN * temperature
        degrees = 3 * n - 3
        base = kT * timescale * timescale
        mass = np.array([degrees * base, base, base])
        q, p = np.zeros(3), np.zeros(3)
        kinetic = 0.5 * float((m[:, None] * v * v).sum())
    energy = None
    for _ in range(steps):
        if thermostat:
            factor, q, p = chain_half_step(kinetic, q, p, mass, degrees, kT, dt)
            v *= factor
            kinetic *= factor * factor
        v = v + 0.5 * dt * f / m[:, None]
        x = wrap(x + dt * v, np.asarray(cell, dtype=np.float64))
        energy, f = evaluate(x)
        v = v + 0.5 * dt * f / m[:, None]
        if thermostat:
            kinetic = 0.5 * float((m[:, None] * v * v).sum())
            factor, q, p = chain_half_step(kinetic, q, p, mass, degrees, kT, dt)
            v *= factor
            kinetic *= factor * factor
    result = {"positions": x, "velocities": v, "forces": f, "energy": energy}
    if thermostat:
        result["chain_positions"], result["chain_momenta"] = q, p
    return result
