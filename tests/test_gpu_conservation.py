"""Conservation audit and long-run FP32 accuracy of the CUDA path.

* Collisionless, fields off, periodic: the finite-volume flux form telescopes,
  so total mass, momentum and energy (moments summed over the interior q-cells)
  are conserved to round-off: 1e-13 relative in FP64, 2e-6 in FP32 (f stored
  in FP32) after 20 RK4 steps.
* With BGK the truncated velocity grid (|p| <= 6) makes the discrete
  Maxwellian leak a little mass; the leak equals the oracle's to 1e-13.
* FP32 f with FP64 moments against the FP64 form of the same kernels after
  1000 RK4 steps of the 2D3V BGK workload (24^3 velocity grid, 32x32 q-grid):
  density and energy within 1e-5 relative L2.
"""

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout, moments_layout
from _util import interior, rel

pytestmark = pytest.mark.gpu

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')


def _spec(**kw):
    base = dict(N_q1=16, N_q2=16, N_p1=8, N_p2=8, N_p3=8,
                p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
                p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
                tau=0.05, dt=1e-3, steps=20, integrator='RK4',
                riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                init=dict(amp=0.1, k1=1, k2=1, u=[0.3, -0.2, 0.1], T=[1.0, 1.3, 0.8]))
    base.update(kw)
    return C.make(**base)


def _totals(nls, spec):
    """Interior sums of the five moments (times the q-cell area)."""
    g = spec['N_ghost']
    area = (1.0 / spec['N_q1']) * (1.0 / spec['N_q2'])
    return np.array([interior(moments_layout(nls.compute_moments(k)), g).sum() * area
                     for k in MOMENTS])


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-13), ('fp32', 2e-6)])
def test_collisionless_periodic_conserves_mass_momentum_energy(precision, tol):
    spec = _spec(source_enabled=False)
    nls = make_solver(spec, precision)
    t0 = _totals(nls, spec)
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    t1 = _totals(nls, spec)
    scale = np.array([t0[0], t0[0], t0[0], t0[0], t0[4]])     # momenta scaled by the mass
    change = np.abs(t1 - t0) / scale
    assert change.max() < tol, dict(zip(MOMENTS, change))


def test_bgk_mass_leak_matches_oracle():
    from oracle.bolt_oracle import Oracle
    spec = _spec(N_q1=8, N_q2=8, tau=0.01, steps=10)
    nls = make_solver(spec, 'fp64')
    o = Oracle(spec, to_layout(nls.f, spec))
    g = spec['N_ghost']
    m0 = interior(o.moments('density'), g).sum()
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
        o.step(spec['dt'])
    leak_gpu = interior(moments_layout(nls.compute_moments('density')), g).sum() - m0
    leak_oracle = interior(o.moments('density'), g).sum() - m0
    assert abs(leak_gpu - leak_oracle) < 1e-13 * abs(m0), (leak_gpu, leak_oracle)


def test_fp32_vs_fp64_after_1000_steps():
    spec = C.make(N_q1=32, N_q2=32, N_p1=24, N_p2=24, N_p3=24,
                  p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
                  p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=1e-3, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.05, k1=1, k2=1))
    out = {}
    for precision in ('fp64', 'fp32'):
        nls = make_solver(spec, precision)
        for _ in range(1000):
            nls.strang_timestep(spec['dt'])
        g = spec['N_ghost']
        out[precision] = {k: interior(moments_layout(nls.compute_moments(k)), g)
                          for k in ('density', 'energy')}
        del nls
        torch.cuda.empty_cache()
    errs = {k: rel(out['fp32'][k], out['fp64'][k]) for k in ('density', 'energy')}
    print('fp32 vs fp64 after 1000 steps, 32x32 x 24^3:', errs)
    assert max(errs.values()) < 1e-5, errs


def test_fp32_vs_fp64_after_1000_steps_full_workload():
    """The 128x128 x 24^3 bench workload itself (226M cells, ~55 s of GPU time
    for the FP64 run): density and energy of FP32 f with FP64 moments within
    1e-5 relative L2 of the FP64 form after 1000 RK4 steps."""
    spec = C.make(N_q1=128, N_q2=128, N_p1=24, N_p2=24, N_p3=24,
                  p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
                  p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=1e-3, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.05, k1=1, k2=1))
    out = {}
    for precision in ('fp64', 'fp32'):
        nls = make_solver(spec, precision)
        for _ in range(1000):
            nls.strang_timestep(spec['dt'])
        g = spec['N_ghost']
        out[precision] = {k: interior(moments_layout(nls.compute_moments(k)), g)
                          for k in ('density', 'energy')}
        del nls
        torch.cuda.empty_cache()
    errs = {k: rel(out['fp32'][k], out['fp64'][k]) for k in ('density', 'energy')}
    print('fp32 vs fp64 after 1000 steps, 128x128 x 24^3:', errs)
    assert max(errs.values()) < 1e-5, errs
