"""The C/OpenMP restatement (oracle/bolt_oracle_c.c) that bench.py times as the
CPU baseline and as the reference arm, pinned to the numpy oracle and to the
reference-generated fixtures.  CPU only.

It covers the fields-off periodic path: WENO5, minmod, PPM and
piecewise-constant faces, BGK on and off, RK2 (fvm_operator.py:6-35) and RK4
(integrators.py:15-28).  Its RK4 combine adds the stages one at a time, which
differs from the reference's (k1 + 2k2 + 2k3 + k4)/6 in the last bits only, so
the two restatements agree to 1e-14 normwise and the fixtures to 1e-12."""

import numpy as np
import pytest

import cases as C
from _util import load_golden, rel, interior, check_compact
from oracle import c_oracle
from oracle.bolt_oracle import Oracle

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')


def _spec(recon, bgk, integrator):
    return C.make(N_q1=10, N_q2=6, N_p1=8, N_p2=6, N_p3=4, recon_q=recon, recon_p=recon,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  source_enabled=bgk, tau=0.02, dt=1e-3, steps=2, integrator=integrator,
                  init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=7, u=[0.3, -0.2, 0.1],
                            T=[1.0, 1.3, 0.8]))


@pytest.mark.parametrize('integrator', ['RK2', 'RK4'])
@pytest.mark.parametrize('bgk', [True, False])
@pytest.mark.parametrize('recon', ['weno5', 'minmod', 'ppm', 'piecewise-constant'])
def test_c_restatement_matches_numpy_oracle(recon, bgk, integrator):
    spec = _spec(recon, bgk, integrator)
    f0 = C.initial_f(spec)
    o = Oracle(spec, f0.copy())
    f = np.ascontiguousarray(f0.copy())
    for _ in range(spec['steps']):
        o.step(spec['dt'])
        c_oracle.rk_step(f, spec, spec['dt'], integrator=int(integrator[2]))
    g = spec['N_ghost']
    assert rel(interior(f, g), interior(o.f, g)) < 1e-14


def test_c_restatement_two_species():
    spec = C.make(N_q1=8, N_q2=8, N_p1=8, N_p2=4, N_p3=4,
                  p1_start=[-5.0, -3.0], p1_end=[5.0, 3.0], p2_start=[-5.0, -3.0],
                  p2_end=[5.0, 3.0], p3_start=[-5.0, -3.0], p3_end=[5.0, 3.0],
                  mass=[1.0, 4.0], charge=[0.0, 0.0], p_dim=3, tau=0.01, dt=1e-3,
                  integrator='RK4', init=dict(amp=0.1, k1=1, k2=2, u=[0.2, -0.1, 0.05]))
    f0 = C.initial_f(spec)
    o = Oracle(spec, f0.copy())
    f = np.ascontiguousarray(f0.copy())
    for _ in range(2):
        o.step(spec['dt'])
        c_oracle.rk_step(f, spec, spec['dt'], integrator=4)
    assert rel(interior(f, 3), interior(o.f, 3)) < 1e-14


@pytest.mark.parametrize('name', ['c1_1d1v_weno5_rk2', 'c1_1d1v_weno5_rk4_llf',
                                  'c3_2d3v_weno5_rk4_small'])
def test_c_restatement_matches_reference_fixture(name):
    """Config 1 of the benchmark set (64 x 128, WENO5, RK2, 100 steps) and the
    RK4 fixtures, stepped by the C restatement from the reference's own
    halo-refreshed initial state."""
    spec = C.CASES[name]
    G = load_golden(name)
    f = np.ascontiguousarray(G['f0_refreshed'].copy())
    integ = 4 if spec['integrator'] == 'RK4' else 2
    for _ in range(spec['steps']):
        c_oracle.rk_step(f, spec, spec['dt'], integrator=integ)
    g = spec['N_ghost']
    assert rel(interior(f, g), G['f_final']) < 1e-12


def test_c_restatement_matches_reference_at_24c3():
    """The bench's velocity grid (24^3) from the compact reference fixture."""
    name = 'c3_2d3v_weno5_rk4_p24'
    spec = C.COMPACT_CASES[name]
    G = load_golden(name)
    f = np.ascontiguousarray(C.periodic_wrap(C.compact_f0(G), spec))
    for _ in range(spec['steps']):
        c_oracle.rk_step(f, spec, spec['dt'], integrator=4)
    o = Oracle(spec, f)
    g = spec['N_ghost']
    m = {k: interior(o.moments(k), g) for k in MOMENTS}
    check_compact(spec, G, interior(f, g), m)
