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

The parameter gradient of a training loss over E, F and W (src/nabladyn/training/_fit.py:
245-271 takes it with torch.func through a double backward) is written out too
(``loss_parameter_gradient``): forward-over-reverse, the forward pass carrying beside each
value its derivative along the loss's force and virial adjoints, then one reverse pass over
both streams.

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




def loss_parameter_gradient(positions, cell, first, second, types, weights, cutoff, gaussians,
                            interactions, e_bar, f_bar, w_bar):
    """d/dtheta of  e_bar E + sum_i f_bar_i . F_i + w_bar : W  (one frame), by hand.

    With F = -dE/dr and W = -dE/d(strain), the last two terms are -D_u E along u = (f_bar on the
    atoms, w_bar on the strain): per pair the distance moves at
    rdot = d.(f_bar_a - f_bar_b) / r + d^T w_bar d / r, so the objective is
    Phi = e_bar E - Edot with Edot the derivative of E along rdot. The forward pass carries a
    tangent beside every value (g', C', ssp' and the chain through both GEMMs of every filter
    and atom-wise layer), and a reverse pass over both streams gives dPhi/dtheta. Returns a
    dict of arrays under the state-dict names.
    """
    positions = np.asarray(positions, dtype=np.float64)
    cell = np.asarray(cell, dtype=np.float64)
    first = np.asarray(first, dtype=np.int64)
    second = np.asarray(second, dtype=np.int64)
    f_bar = np.asarray(f_bar, dtype=np.float64)
    w_bar = np.asarray(w_bar, dtype=np.float64)
    d, r, valid = pair_geometry(positions, cell, first, second, cutoff)
    rdot = ((d * (f_bar[first] - f_bar[second])).sum(axis=1)
            + np.einsum("pa,ab,pb->p", d, w_bar, d)) / r
    rdot = np.where(valid, rdot, 0.0)
    phase = math.pi / cutoff
    envelope = np.where(valid, 0.5 * (np.cos(r * phase) + 1.0), 0.0)
    slope = np.where(valid, -0.5 * phase * np.sin(r * phase), 0.0)
    width = cutoff / (gaussians - 1)
    centres = np.linspace(0.0, cutoff, gaussians)
    offset = (r[:, None] - centres) / width
    g = np.exp(-0.5 * offset * offset)
    g_dot = -g * offset / width * rdot[:, None]
    c_dot = slope * rdot

    def sig(x):
        return sigmoid(x)

    def dsig(x):
        s = sigmoid(x)
        return s * (1.0 - s)

    n = positions.shape[0]
    x = weights["embedding"][types]
    x_dot = np.zeros_like(x)
    saved = []
    for b in range(interactions):
        w = lambda name: weights[f"blocks.{b}.{name}"]  # noqa: E731
        v, v_dot = x @ w("atoms.weight").T, x_dot @ w("atoms.weight").T
        z = g @ w("filter1.weight").T + w("filter1.bias")
        z_dot = g_dot @ w("filter1.weight").T
        s, s_dot = ssp(z), sig(z) * z_dot
        u = s @ w("filter2.weight").T + w("filter2.bias")
        u_dot = s_dot @ w("filter2.weight").T
        f = u * envelope[:, None]
        f_dot = u_dot * envelope[:, None] + u * c_dot[:, None]
        m, m_dot = np.zeros_like(x), np.zeros_like(x)
        np.add.at(m, first, f * v[second])
        np.add.at(m, second, f * v[first])
        np.add.at(m_dot, first, f_dot * v[second] + f * v_dot[second])
        np.add.at(m_dot, second, f_dot * v[first] + f * v_dot[first])
        h = m @ w("update1.weight").T + w("update1.bias")
        h_dot = m_dot @ w("update1.weight").T
        saved.append((x, x_dot, v, v_dot, z, z_dot, s, s_dot, u, u_dot, f, f_dot, m, m_dot, h,
                      h_dot))
        x = x + ssp(h) @ w("update2.weight").T + w("update2.bias")
        x_dot = x_dot + (sig(h) * h_dot) @ w("update2.weight").T
    r1, e1 = weights["readout1.weight"], weights["readout1.bias"]
    r2 = weights["readout2.weight"][0]
    y, y_dot = x @ r1.T + e1, x_dot @ r1.T
    grads = {name: np.zeros_like(value) for name, value in weights.items()}
    # Phi = e_bar sum(ssp(y) r2 + e2) - sum((sig(y) y_dot) r2)
    y_bar = e_bar * sig(y) * r2 - dsig(y) * y_dot * r2
    y_dot_bar = -sig(y) * r2
    grads["readout2.weight"][0] = (e_bar * ssp(y) - sig(y) * y_dot).sum(axis=0)
    grads["readout2.bias"][0] = e_bar * n
    grads["readout1.weight"] = y_bar.T @ x + y_dot_bar.T @ x_dot
    grads["readout1.bias"] = y_bar.sum(axis=0)
    x_bar, x_dot_bar = y_bar @ r1, y_dot_bar @ r1
    for b in reversed(range(interactions)):
        name = lambda k: f"blocks.{b}.{k}"  # noqa: E731
        w = lambda k: weights[name(k)]  # noqa: E731
        (x, x_dot, v, v_dot, z, z_dot, s, s_dot, u, u_dot, f, f_dot, m, m_dot, h,
         h_dot) = saved[b]
        d2 = w("update2.weight")
        ssp_bar, q_bar = x_bar @ d2, x_dot_bar @ d2
        grads[name("update2.weight")] += x_bar.T @ ssp(h) + x_dot_bar.T @ (sig(h) * h_dot)
        grads[name("update2.bias")] += x_bar.sum(axis=0)
        h_bar = ssp_bar * sig(h) + q_bar * h_dot * dsig(h)
        h_dot_bar = q_bar * sig(h)
        d1 = w("update1.weight")
        m_bar, m_dot_bar = h_bar @ d1, h_dot_bar @ d1
        grads[name("update1.weight")] += h_bar.T @ m + h_dot_bar.T @ m_dot
        grads[name("update1.bias")] += h_bar.sum(axis=0)
        # the messages, both streams
        f_bar_p = (m_bar[first] * v[second] + m_bar[second] * v[first]
                   + m_dot_bar[first] * v_dot[second] + m_dot_bar[second] * v_dot[first])
        f_dot_bar = m_dot_bar[first] * v[second] + m_dot_bar[second] * v[first]
        v_bar, v_dot_bar = np.zeros_like(v), np.zeros_like(v)
        np.add.at(v_bar, second, f * m_bar[first] + f_dot * m_dot_bar[first])
        np.add.at(v_bar, first, f * m_bar[second] + f_dot * m_dot_bar[second])
        np.add.at(v_dot_bar, second, f * m_dot_bar[first])
        np.add.at(v_dot_bar, first, f * m_dot_bar[second])
        a = w("atoms.weight")
        grads[name("atoms.weight")] += v_bar.T @ x + v_dot_bar.T @ x_dot
        x_bar = x_bar + v_bar @ a
        x_dot_bar = x_dot_bar + v_dot_bar @ a
        # the filter network, both streams
        u_bar = f_bar_p * envelope[:, None] + f_dot_bar * c_dot[:, None]
        u_dot_bar = f_dot_bar * envelope[:, None]
        b2 = w("filter2.weight")
        s_bar, s_dot_bar = u_bar @ b2, u_dot_bar @ b2
        grads[name("filter2.weight")] += u_bar.T @ s + u_dot_bar.T @ s_dot
        grads[name("filter2.bias")] += u_bar.sum(axis=0)
        z_bar = s_bar * sig(z) + s_dot_bar * z_dot * dsig(z)
        z_dot_bar = s_dot_bar * sig(z)
        grads[name("filter1.weight")] += z_bar.T @ g + z_dot_bar.T @ g_dot
        grads[name("filter1.bias")] += z_bar.sum(axis=0)
    np.add.at(grads["embedding"], np.asarray(types, dtype=np.int64), x_bar)
    return grads


def loss_adjoints(predicted, labels, weights, scales, coefficient):
    """One frame's loss term and its adjoints (dL/dE, dL/dF [N, 3], dL/dW [3, 3]).

    The loss of src/nabladyn/training/_loss.py:105-125: per weighted channel, the frame's mean
    of ((X - X*) / s)^2 over its components, times the frame's coefficient and the channel's
    weight. ``predicted`` and ``labels`` map "energy", "forces", "virial" to arrays.
    """
    value = 0.0
    adjoints = {}
    for name in ("energy", "forces", "virial"):
        x = np.asarray(predicted[name], dtype=np.float64)
        if name not in weights:
            adjoints[name] = np.zeros_like(x)
            continue
        error = (x - np.asarray(labels[name], dtype=np.float64)) / scales[name]
        value += coefficient * weights[name] * float(np.mean(error * error))
        adjoints[name] = coefficient * weights[name] * 2.0 * error / scales[name] / error.size
    return value, float(adjoints["energy"]), adjoints["forces"], adjoints["virial"]


__all__ = ("ssp", "sigmoid", "pair_geometry", "energy_force_virial", "loss_parameter_gradient",
           "loss_adjoints")
