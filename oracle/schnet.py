"""Float64 restatement of the SchNet energy, forces and virial. Test infrastructure only.

The forward pass follows src/nabladyn/potential/_schnet/_potential.py:45-120 (pair geometry,
Gaussians, cosine envelope, filter network, symmetric messages, atom-wise update) and
:190-208 (embedding, blocks, readout). The reference gets forces and virial from autograd
(src/nabladyn/quantity.py:93-117); here they come from a reverse pass written out by hand,
in the order the CUDA kernels take it, so a match with the reference's autograd numbers
pins the derivation as well as the forward arithmetic:

* readout: G = dE/dx = (sigmoid(x R1^T + e1) * R2) R1;
* each block, last first: Gh = (G D2) * sigmoid(h), Gm = Gh D1; per pair p = (a, b)
  Gf_p = Gm_a * v_b + Gm_b * v_a and Gv_b += f_p * Gm_a, Gv_a += f_p * Gm_b; G += Gv A;
* per pair and block, through the filter: dE/dr += C'(r) (Gf . f_raw)
  + sum_k [((Gf C) B2 * sigmoid(z1)) B1]_k g_k'(r);
* F_a -= dE/dr d / r, F_b += dE/dr d / r and W -= dE/dr d d^T / r.

Weights are a dict of float64 arrays under the reference's state-dict names.
"""

from __future__ import annotations

import math

import numpy as np

LN2 = math.log(2.0)


def ssp(x):
    """ln(1 + e^x) - ln 2 (src/nabladyn/potential/_schnet/_potential.py:45-47)."""
    return np.logaddexp(0.0, x) - LN2


def sigmoid(x):
    """d ssp / dx."""
    return 0.5 * (1.0 + np.tanh(0.5 * x))


def pair_geometry(positions, cell, first, second, cutoff):
    """Minimum-image d = r_first - r_second (src/nabladyn/space.py:11-19), r, validity."""
    left, right = positions[first], positions[second]
    raw = left - right
    half = 0.5 * cell
    d = (left - np.where(raw > half, cell, 0.0)) - (right - np.where(raw < -half, cell, 0.0))
    squared = (d * d).sum(axis=1)
    valid = (first != second) & (squared < cutoff * cutoff)
    r = np.sqrt(np.where(valid, squared, 1.0))
    return d, r, valid


def energy_force_virial(positions, cell, first, second, types, weights, cutoff, gaussians,
                        interactions):
    """(E, F [N, 3], W [3, 3]) of wrapped positions over the pair columns (first, second)."""
    positions = np.asarray(positions, dtype=np.float64)
    cell = np.asarray(cell, dtype=np.float64)
    first = np.asarray(first, dtype=np.int64)
    second = np.asarray(second, dtype=np.int64)
    n = positions.shape[0]
    d, r, valid = pair_geometry(positions, cell, first, second, cutoff)
    phase = math.pi / cutoff
    envelope = np.where(valid, 0.5 * (np.cos(r * phase) + 1.0), 0.0)
    slope = np.where(valid, -0.5 * phase * np.sin(r * phase), 0.0)
    width = cutoff / (gaussians - 1)
    centres = np.linspace(0.0, cutoff, gaussians)
    offset = (r[:, None] - centres) / width
    g = np.exp(-0.5 * offset * offset)
    g_slope = -g * offset / width

    x = weights["embedding"][types]
    saved = []
    for b in range(interactions):
        w = lambda name: weights[f"blocks.{b}.{name}"]  # noqa: E731
        v = x @ w("atoms.weight").T
        z1 = g @ w("filter1.weight").T + w("filter1.bias")
        f_raw = ssp(z1) @ w("filter2.weight").T + w("filter2.bias")
        f = f_raw * envelope[:, None]
        m = np.zeros_like(x)
        np.add.at(m, first, f * v[second])
        np.add.at(m, second, f * v[first])
        h = m @ w("update1.weight").T + w("update1.bias")
        saved.append((v, z1, f_raw, f, h))
        x = x + ssp(h) @ w("update2.weight").T + w("update2.bias")
    y = x @ weights["readout1.weight"].T + weights["readout1.bias"]
    energy = float((ssp(y) @ weights["readout2.weight"].T + weights["readout2.bias"]).sum())

    grad = (sigmoid(y) * weights["readout2.weight"][0]) @ weights["readout1.weight"]
    dedr = np.zeros(r.shape[0])
    for b in reversed(range(interactions)):
        w = lambda name: weights[f"blocks.{b}.{name}"]  # noqa: E731
        v, z1, f_raw, f, h = saved[b]
        grad_h = (grad @ w("update2.weight")) * sigmoid(h)
        grad_m = grad_h @ w("update1.weight")
        grad_f = grad_m[first] * v[second] + grad_m[second] * v[first]
        grad_v = np.zeros_like(grad)
        np.add.at(grad_v, second, f * grad_m[first])
        np.add.at(grad_v, first, f * grad_m[second])
        grad = grad + grad_v @ w("atoms.weight")
        q = ((grad_f * envelope[:, None]) @ w("filter2.weight")) * sigmoid(z1)
        dedr += slope * (grad_f * f_raw).sum(axis=1) + ((q @ w("filter1.weight")) * g_slope).sum(axis=1)
    dedr = np.where(valid, dedr, 0.0)
    unit = d * (dedr / r)[:, None]
    forces = np.zeros((n, 3))
    np.add.at(forces, first, -unit)
    np.add.at(forces, second, unit)
    virial = -(unit[:, :, None] * d[:, None, :]).sum(axis=0)
    return energy, forces, virial


__all__ = ("ssp", "sigmoid", "pair_geometry", "energy_force_virial")
