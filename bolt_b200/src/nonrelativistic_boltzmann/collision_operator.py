"""BGK relaxation to the local Maxwellian
(bolt/src/nonrelativistic_boltzmann/collision_operator.py:16-128)."""

import math

import torch


def f0(v1, v2, v3, n, T, v1_bulk, v2_bulk, v3_bulk, params):
    m = params.mass
    k = params.boltzmann_constant
    if params.p_dim == 3:
        return n * (m / (2 * math.pi * k * T)) ** (3 / 2) \
            * torch.exp(-m * (v1 - v1_bulk) ** 2 / (2 * k * T)) \
            * torch.exp(-m * (v2 - v2_bulk) ** 2 / (2 * k * T)) \
            * torch.exp(-m * (v3 - v3_bulk) ** 2 / (2 * k * T))
    if params.p_dim == 2:
        return n * (m / (2 * math.pi * k * T)) \
            * torch.exp(-m * (v1 - v1_bulk) ** 2 / (2 * k * T)) \
            * torch.exp(-m * (v2 - v2_bulk) ** 2 / (2 * k * T))
    return n * torch.sqrt(m / (2 * math.pi * k * T)) \
        * torch.exp(-m * (v1 - v1_bulk) ** 2 / (2 * k * T))


def BGK(f, t, q1, q2, v1, v2, v3, moments, params, flag=False):
    n = moments('density', f)
    m = params.mass
    eps = 1e-30
    v1_bulk = moments('mom_v1_bulk', f) / (n + eps)
    v2_bulk = moments('mom_v2_bulk', f) / (n + eps)
    v3_bulk = moments('mom_v3_bulk', f) / (n + eps)
    T = (1 / params.p_dim) * (2 * moments('energy', f) * m
                              - n * m * v1_bulk ** 2
                              - n * m * v2_bulk ** 2
                              - n * m * v3_bulk ** 2) / (n + eps) + eps
    f_MB = f0(v1, v2, v3, n, T, v1_bulk, v2_bulk, v3_bulk, params)
    tau = params.tau(q1, q2, v1, v2, v3)
    if not flag:
        return -(f - f_MB) / tau
    return f_MB
