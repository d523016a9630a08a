"""Structured discrete-velocity tables of the S2 path (the reference's mod_VelocityTables.f90).

The reference ships two half-range Gauss-Hermite rules, half16 and half32 (8 and 16 positive
nodes, mirrored), and builds the 2-D table from a raw rule in FillVelocity
(mod_VelocityTables.f90:31-122): u_e = sqrt(2) x, w_e = sqrt(2) exp(x^2) w, both times the
velocity scale, then the tensor product k = i + (j-1) n.  The batched and refined cases also need
24^2 and 48^2 tables, which the reference does not ship.  This module generates any half-range rule
(weight exp(-x^2) on [0, inf), n positive nodes) from its moments: Gautschi's Chebyshev algorithm gives
the recurrence coefficients at 100 significant digits, and the Golub-Welsch eigen-decomposition of the
Jacobi matrix gives the nodes and weights, rounded to FP64 once at the end.  For n = 8 and n = 16 the
result matches the reference's half16 / half32 tables to the last printed digit (tests).
"""
import math

import numpy as np


def half_range_gauss_hermite(n, dps=100):
    """n-point Gauss rule for the weight exp(-x^2) on [0, inf): (nodes, weights), ascending FP64."""
    import mpmath as mp
    with mp.workdps(dps):
        nm = 2 * n
        # moments mu_k = Gamma((k + 1) / 2) / 2
        mu = [mp.gamma(mp.mpf(k + 1) / 2) / 2 for k in range(nm)]
        alpha = [mp.mpf(0)] * n
        beta = [mp.mpf(0)] * n
        # Chebyshev algorithm (ordinary moments): sigma_{k,l} rows
        sig_prev = [mp.mpf(0)] * nm          # sigma_{-1,l}
        sig = list(mu)                       # sigma_{0,l}
        alpha[0] = mu[1] / mu[0]
        beta[0] = mu[0]
        for k in range(1, n):
            new = [mp.mpf(0)] * nm
            for l in range(k, nm - k):
                new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
            alpha[k] = new[k + 1] / new[k] - sig[k] / sig[k - 1]
            beta[k] = new[k] / sig[k - 1]
            sig_prev, sig = sig, new
        J = mp.matrix(n, n)
        for k in range(n):
            J[k, k] = alpha[k]
            if k + 1 < n:
                J[k, k + 1] = J[k + 1, k] = mp.sqrt(beta[k + 1])
        ev, V = mp.eigsy(J)
        order = sorted(range(n), key=lambda i: ev[i])
        nodes = [float(ev[i]) for i in order]
        weights = [float(beta[0] * V[0, i] ** 2) for i in order]
    return np.array(nodes), np.array(weights)


def raw_rule(n_per_side):
    """The mirrored raw rule of a halfN table: 2 n nodes ascending and their weights."""
    x, w = half_range_gauss_hermite(n_per_side)
    return np.concatenate([-x[::-1], x]), np.concatenate([w[::-1], w])


def fill_velocity(raw_node, raw_weight, scale=2.0):
    """FillVelocity (mod_VelocityTables.f90:97-120) in FP64: (u, v, w) of the tensor table."""
    raw_node = np.asarray(raw_node, dtype=np.float64)
    raw_weight = np.asarray(raw_weight, dtype=np.float64)
    ue = math.sqrt(2.0) * raw_node
    we = math.sqrt(2.0) * np.exp(raw_node * raw_node) * raw_weight
    if scale != 1.0:
        ue = scale * ue
        we = scale * we
    n = len(raw_node)
    u = np.tile(ue, n)            # k = i + (j-1) n: i fastest
    v = np.repeat(ue, n)
    w = np.tile(we, n) * np.repeat(we, n)   # weight(k) = we(i) * we(j)
    return u, v, w


def structured_table(n_per_axis, scale=2.0):
    """The (n_per_axis)^2 table of a half-range rule with n_per_axis / 2 positive nodes."""
    if n_per_axis % 2:
        raise ValueError("the half-range tables have an even node count per axis")
    node, weight = raw_rule(n_per_axis // 2)
    return fill_velocity(node, weight, scale)
