"""Linear Landau damping through the electrostatic path (the FFT Poisson
solve at every df/dt, fft.py:9-78) -- the physics the reference's
landau_damping/linear example checks against linear theory.

1D1V, q1 in [0, 4 pi) periodic (k = 0.5 in Debye units), 32 cells; p1 in
[-8, 8] with 128 cells; electrons (charge -1, m = 1, T = 1) with
f0 = (1 + 0.01 cos(k q1)) Maxwellian, collisionless; WENO5 + upwind, RK4,
dt = 0.02, 750 steps (t = 15).  The electric field energy W(t) = sum E1^2
oscillates at 2 omega and decays at 2 gamma; the linear dispersion relation
gives omega = 1.4156, gamma = -0.1533 for k = 0.5.  The fitted gamma (log W
at its successive maxima) is within 2 % of theory and omega (from the
spacing of the maxima) within 1 %, in FP64 and in FP32 (FP64 moments); the
FP64 run reproduces the numpy oracle's W(t) over the first 50 steps to 1e-10.
"""

import math

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout

pytestmark = pytest.mark.gpu

K = 0.5
L = 2 * math.pi / K
GAMMA, OMEGA = -0.1533, 1.4156

SPEC = C.make(N_q1=32, N_q2=1, N_p1=128, N_p2=1, N_p3=1, q1_end=L,
              p1_start=[-8.0], p1_end=[8.0], p2_start=[-0.5], p2_end=[0.5],
              p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=1,
              source_enabled=False, fields_enabled=True, fields_type='electrostatic',
              fields_solver='fft', integrator='RK4', dt=0.02, steps=750,
              init=dict(amp=0.01, k1=1.0 / L, k2=0))


def _energy_history(precision, steps):
    nls = make_solver(SPEC, precision)
    g = SPEC['N_ghost']
    W = []
    for _ in range(steps):
        nls.strang_timestep(SPEC['dt'])
        E1 = nls.fields_solver.cell_centered_EM_fields[0, 0, g:-g, g]
        W.append(float((E1.double() ** 2).sum()))
    return nls, np.array(W)


def _fit(W):
    t = SPEC['dt'] * (1 + np.arange(len(W)))
    pk = [i for i in range(1, len(W) - 1) if W[i] > W[i - 1] and W[i] >= W[i + 1]]
    assert len(pk) >= 5, pk
    gamma = np.polyfit(t[pk], np.log(W[pk]), 1)[0] / 2
    omega = math.pi / np.mean(np.diff(t[pk]))
    return gamma, omega


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_landau_damping_rate_and_frequency(precision):
    _, W = _energy_history(precision, SPEC['steps'])
    gamma, omega = _fit(W)
    assert abs(gamma - GAMMA) < 0.02 * abs(GAMMA), gamma
    assert abs(omega - OMEGA) < 0.01 * OMEGA, omega


def test_landau_field_energy_matches_oracle():
    from oracle.bolt_oracle import Oracle
    steps = 50
    nls, W = _energy_history('fp64', 0)
    o = Oracle(SPEC, to_layout(nls.f, SPEC))
    g = SPEC['N_ghost']
    Wg, Wo = [], []
    for _ in range(steps):
        nls.strang_timestep(SPEC['dt'])
        o.step(SPEC['dt'])
        Wg.append(float((nls.fields_solver.cell_centered_EM_fields[0, 0, g:-g, g].double() ** 2).sum()))
        Wo.append(float((o.fields.cell[0][g, g:-g] ** 2).sum()))
    Wg, Wo = np.array(Wg), np.array(Wo)
    assert np.max(np.abs(Wg - Wo) / Wo) < 1e-10
