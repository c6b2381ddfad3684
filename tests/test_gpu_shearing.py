"""Shearing-box boundaries (boundaries.py:6-145) through the CUDA path.

The reference resamples each ghost strip with ArrayFire's approx2
(BICUBIC_SPLINE), a third-party kernel that cannot run here; the strips are
restated as the one-dimensional Catmull-Rom cubic along the sheared axis
(oracle/bolt_oracle.py, Oracle._shear_strip), so parity with the reference is
unpinned at that boundary.  Checked here: the reference's own known-answer
test (test_shearing_boundaries/test_shear.py: ghost strips equal the shifted
initial data with O(N^-3) error) on the CUDA ghost pass, and whole RK4 runs
against the oracle (FP64 1e-12, FP32 2e-6, FP64 throughput form 1e-10)."""

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout, moments_layout
from _util import rel, interior, moment_errors
from test_oracle_golden import shear_spec, shear_errors

pytestmark = pytest.mark.gpu

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')


@pytest.mark.parametrize('axis', [1, 2])
def test_shearing_box_kat_third_order(axis):
    """After the halo refresh at time t the CUDA ghost strips (FP64) equal the
    initial data shifted by -/+ q omega L t, with error O(N^-3) (slope within
    0.3 of -3 over N = 32 .. 512)."""
    Ns = [32, 64, 128, 256, 512]
    errs = []
    for N in Ns:
        spec = shear_spec(N, axis)
        nls = make_solver(spec, 'fp64')
        g = spec['N_ghost']
        e = 0.0
        for t in np.linspace(0.11, 0.89, 7):
            nls.time_elapsed = t
            nls._communicate_f()
            out = to_layout(nls.f, spec)[..., 0, 0, 0, 0]

            def strip(side):
                if axis == 1:
                    return out[g:N + g, :g] if side == 'lo' else out[g:N + g, N + g:]
                return (out[:g, g:N + g] if side == 'lo' else out[N + g:, g:N + g]).T
            e += shear_errors(spec, strip, t, axis)
        errs.append(e)
        nls.synchronize()
    slope = np.polyfit(np.log10(Ns), np.log10(errs), 1)[0]
    assert abs(slope + 3) < 0.3, (errs, slope)


@pytest.mark.parametrize('precision,tol', [('fp32', 1e-6), ('fp64', 1e-14)])
@pytest.mark.parametrize('axis', [1, 2])
def test_shearing_box_strips_vs_oracle(axis, precision, tol):
    """The CUDA ghost strips at several times against the oracle's, from the
    same f (in FP32 the strips are resampled in FP64 from FP32 values and
    rounded once)."""
    from oracle.bolt_oracle import Oracle
    spec = shear_spec(64, axis)
    nls = make_solver(spec, precision)
    o = Oracle(spec, to_layout(nls.f, spec))
    for t in (0.0, 0.23, 0.61, 1.7, 12.345):
        nls.time_elapsed = o.time_elapsed = t
        nls._communicate_f()
        e = rel(to_layout(nls.f, spec), o.refresh(o.f))
        assert e < tol, (t, e)
    nls.synchronize()


def _run_spec(axis):
    bc = dict(bc_q1='shearing-box', bc_q2='periodic') if axis == 1 else \
        dict(bc_q1='periodic', bc_q2='shearing-box')
    return C.make(N_q1=16, N_q2=16, N_p1=8, N_p2=8, N_p3=4,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=2e-3, steps=4, integrator='RK4', shear_q=1.5, shear_omega=2.0,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=9, u=[0.2, -0.1, 0.05]), **bc)


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-12), ('fp32', 2e-6), ('fp64-fast', 1e-10)])
@pytest.mark.parametrize('axis', [1, 2])
def test_shearing_box_run_vs_oracle(axis, precision, tol):
    """Four RK4 steps with a shearing-box axis (the strips sheared to each
    step's start time) against the oracle from the same initial state: f and
    the five moments."""
    from oracle.bolt_oracle import Oracle
    spec = _run_spec(axis)
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    o = Oracle(spec, to_layout(nls.f, spec))
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
        o.step(spec['dt'])
    torch.cuda.synchronize()
    if precision != 'fp64':
        assert nls.paired_launch_count() == 4 * spec['steps']
    e = rel(interior(to_layout(nls.f, spec), g), interior(o.f, g))
    assert e < tol, e
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    errs = moment_errors(m, {k: interior(o.moments(k), g) for k in MOMENTS})
    assert max(errs.values()) < tol, errs
    # the ghost strips of the final state at the final time
    nls._communicate_f()
    o_ghost = o.refresh(o.f)
    assert rel(to_layout(nls.f, spec), o_ghost) < tol
    nls.synchronize()
