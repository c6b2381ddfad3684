"""The reference's own known-answer and convergence tests, run through the CUDA
path (the oracle versions of the first three are in test_oracle_golden.py):

* velocity moments of a drifting Maxwellian against their closed forms
  (test_compute_moments.py:76-144);
* periodic ghost cells equal to the analytic periodic function
  (test_apply_boundary_conditions.py:131-145, test_communicate.py:168-182);
* the temporal order of the RK2 and RK4 steppers (test_time_integrators.py:26-70
  asserts the slope of log error vs log dt within 0.2 of 2 and 4 on a scalar
  ODE), measured here on the WENO5 FVM update itself against a run with a 64x
  smaller dt, within 0.3;
* FDTD second-order convergence of a vacuum mode set up through
  initialize_A3_B3 (test_fdtd_explicit.py:120-220, mode 1: slope within 0.2
  of -2), over exactly one period;
* the discrete divergence of B from initialize_A3_B3 vanishes
  (test_check_maxwells_contraints.py:96) and stays zero under the FDTD update;
* the TM mode driven by a current J3, through evolve_electrodynamic_fields
  (test_fdtd_explicit_with_currents.py:97-159: slope within 0.25 of -2), set
  up on the Yee positions of fields.py's initialisation;
* the FFT Poisson solve of rho = -sin(2 pi q1 + 4 pi q2) on 1024^2 cells
  against its closed form to 1e-14 (test_fft_poisson.py:55-80), both the
  initial solve and the per-df/dt solve of the electrostatic path.
"""

import math

import numpy as np
import pytest
import torch

import cases as C
from _modules import build_modules, make_solver, to_layout

pytestmark = pytest.mark.gpu


def _interior_q(a, g):
    """(..., Nq1g, Nq2g) -> interior cells."""
    return a[..., g:a.shape[-2] - g, g:a.shape[-1] - g]


def test_moment_kat():
    spec = C.make(N_q1=16, N_q2=16, N_p1=32, N_p2=32, N_p3=32,
                  p1_start=[-10.0], p1_end=[10.0], p2_start=[-10.0], p2_end=[10.0],
                  p3_start=[-10.0], p3_end=[10.0], mass=[1.0], charge=[0.0], p_dim=3)
    nls = make_solver(spec, 'fp64')
    q1, q2 = nls.q1_center, nls.q2_center                        # (1, 1, Nq1g, Nq2g)
    p1, p2, p3 = nls.p1_center, nls.p2_center, nls.p3_center     # (Np, Ns, 1, 1)
    rho = 1 + 0.01 * torch.sin(2 * math.pi * q1 + 4 * math.pi * q2)
    T = 1 + 0.01 * torch.cos(2 * math.pi * q1 + 4 * math.pi * q2)
    pb = 0.01 * torch.exp(-10 * q1 ** 2 - 10 * q2 ** 2)
    f = rho * (1 / (2 * math.pi * T)) ** 1.5 * torch.exp(-(p1 - pb) ** 2 / (2 * T)) \
        * torch.exp(-(p2 - pb) ** 2 / (2 * T)) * torch.exp(-(p3 - pb) ** 2 / (2 * T))
    nls.f = f
    g = spec['N_ghost']
    err = lambda name, ref: float(torch.mean(torch.abs(
        _interior_q(nls.compute_moments(name), g) - _interior_q(ref, g))))
    assert err('density', rho) < 1e-13
    assert err('energy', 1.5 * rho * T + 1.5 * rho * pb ** 2) < 1e-13
    for name in ('mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk'):
        assert err(name, rho * pb) < 1e-13


@pytest.mark.parametrize('precision,tol', [('fp64', 5e-14), ('fp32', 1e-6)])
def test_periodic_ghost_fill_kat(precision, tol):
    spec = C.make(N_q1=32, N_q2=16, N_p1=2, N_p2=1, N_p3=1,
                  p1_start=[-1.0], p1_end=[1.0], p2_start=[-0.5], p2_end=[0.5],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1)
    nls = make_solver(spec, precision)
    g = spec['N_ghost']
    expected = torch.sin(2 * math.pi * nls.q1_center + 4 * math.pi * nls.q2_center)
    f = torch.zeros_like(nls.f, dtype=torch.float64)
    f[..., g:-g, g:-g] = _interior_q(expected, g)
    nls.f = f                                    # ghosts zero until the fill
    nls._communicate_f()                         # as the reference's test calls it
    nls._apply_bcs_f()
    torch.cuda.synchronize()
    got = nls.f.double()
    assert float((got - expected.expand_as(got)).abs().max()) < tol


def _advect_1d1v(integrator, dt, t_end):
    spec = C.make(N_q1=32, N_q2=1, N_p1=32, N_p2=1, N_p3=1,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-0.5], p2_end=[0.5],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
                  source_enabled=False, integrator=integrator,
                  init=dict(amp=0.01, k1=1, k2=0))
    nls = make_solver(spec, 'fp64')
    n = int(round(t_end / dt))
    assert abs(n * dt - t_end) < 1e-12
    for _ in range(n):
        nls.strang_timestep(dt)
    return to_layout(nls.f, spec)[3:-3, 3:-3]


@pytest.mark.parametrize('integrator,order', [('RK2', 2), ('RK4', 4)])
def test_rk_temporal_order(integrator, order):
    """Collisionless 1D1V advection (WENO5, |v| <= 5, dq1 = 1/32): the same
    grid stepped with dt, dt/2, dt/4 (CFL 0.5, 0.25, 0.125) against dt/64."""
    dt0, t_end = 1.0 / 320, 0.1
    ref = _advect_1d1v(integrator, dt0 / 64, t_end)
    dts = [dt0, dt0 / 2, dt0 / 4]
    errs = [np.abs(_advect_1d1v(integrator, dt, t_end) - ref).max() for dt in dts]
    slope = np.polyfit(np.log10(dts), np.log10(errs), 1)[0]
    assert abs(slope - order) < 0.3, (errs, slope)


def _fdtd_mode1_solver(N, dt, a3b3, init_E=None):
    """2D2V with charge 0 (vacuum Maxwell), fields from initialize_E and
    initialize_A3_B3."""
    spec = C.make(N_q1=N, N_q2=N, N_p1=4, N_p2=4, N_p3=1,
                  p1_start=[-1.0], p1_end=[1.0], p2_start=[-1.0], p2_end=[1.0],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=2,
                  recon_q='minmod', recon_p='minmod', source_enabled=False,
                  fields_enabled=True, fields_initialize='user-defined')
    from bolt_b200.physical_system import physical_system
    from bolt_b200.nonlinear_solver import nonlinear_solver
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    dom, bc, params, initialize = build_modules(spec, 'fp64', None)
    params.dt = dt
    initialize.initialize_A3_B3 = a3b3
    if init_E is not None:
        initialize.initialize_E = init_E
    elif a3b3 is _mode1_A3_B3:
        initialize.initialize_E = _mode1_E
    else:
        initialize.initialize_E = lambda q1, q2, p: (0 * q1, 0 * q1, 0 * q1)
    return nonlinear_solver(physical_system(dom, bc, params, initialize, adv, col.BGK, mom))


def _mode1_E(q1, q2, params):
    # initialize_fdtd_mode1.py: E3 of the (2 pi, 4 pi) vacuum mode
    return (0 * q1, 0 * q1,
            -6 * math.pi * math.sqrt(5 / 9) * torch.cos(2 * math.pi * q1 + 4 * math.pi * q2))


def _mode1_A3_B3(q1, q2, params):
    # A3 at t = -dt/2 (B lives half a step behind E)
    s = 0.5 * math.sqrt(5 / 9) * params.dt
    return (torch.sin(2 * math.pi * (q1 - s) + 4 * math.pi * (q2 - s)), 0 * q1)


def _yee(nls):
    return nls.fields_solver.yee_grid_EM_fields[:, 0].double()      # (6, Nq1g, Nq2g)


def test_fdtd_mode_converges_second_order():
    period = 1 / math.sqrt(5)              # omega = 2 pi sqrt(5) for k = (2 pi, 4 pi)
    Ns = [32, 64, 128]
    errs = {3: [], 4: [], 2: []}
    for N in Ns:
        n = math.ceil(period * 2 * N)      # dt <= dq / 2, as the reference's test
        dt = period / n
        nls = _fdtd_mode1_solver(N, dt, _mode1_A3_B3)
        y0 = _yee(nls).clone()
        for _ in range(n):
            nls.strang_timestep(dt)
        y1 = _yee(nls)
        g = nls.N_ghost
        for c in errs:
            errs[c].append(float(torch.mean(torch.abs(_interior_q(y1[c] - y0[c], g)))))
    for c, e in errs.items():
        slope = np.polyfit(np.log10(Ns), np.log10(e), 1)[0]
        assert abs(slope + 2) < 0.2, (c, e, slope)


def test_div_b_vanishes():
    def a3b3(q1, q2, params):
        # initialize_check_maxwells_contraints.py
        return (torch.sin(2 * math.pi * q1 + 4 * math.pi * q2), 1e-5 * q1 ** 0)
    N = 32
    nls = _fdtd_mode1_solver(N, 1 / (2 * N), a3b3)
    g = nls.N_ghost
    dq1 = dq2 = 1.0 / N

    def div_b():
        y = _yee(nls)
        B1, B2 = y[3], y[4]                # (Nq1g, Nq2g): q1 is dim 0 here
        d = (B1 - torch.roll(B1, 1, dims=0)) / dq1 + (B2 - torch.roll(B2, 1, dims=1)) / dq2
        api = nls.fields_solver.compute_divB()[0, 0]
        assert torch.equal(api, d)
        return float(torch.mean(torch.abs(_interior_q(d, g))))
    assert div_b() < 1e-14 * (4 * math.pi / dq1)
    for _ in range(20):
        nls.strang_timestep(1 / (2 * N))
    assert div_b() < 1e-14 * (4 * math.pi / dq1)


def test_fdtd_tm_mode_with_currents_converges_second_order():
    """The driven TM mode of test_fdtd_explicit_with_currents.py:97-159:
    A3 = sin(phi), B1 = dA3/dq2, B2 = -dA3/dq1, E3 = 6 pi cos(phi),
    J3 = -16 pi^2 sin(phi), phi = 2 pi q1 + 4 pi q2 - 6 pi t, one drive period.
    The fields sit on the Yee positions of fields.py's initialisation (E3 and
    A3 at the cell centre, J3 with E3); the reference's test file places every
    component at the left-bottom corner instead, and imports a module path
    (bolt.lib.nonlinear_solver) absent from its tree."""
    Ns = [32, 64, 128]
    errs = {3: [], 4: [], 2: []}
    for N in Ns:
        dt = (1.0 / N) / 2
        tm_E = lambda q1, q2, p: (0 * q1, 0 * q1,
                                  6 * math.pi * torch.cos(2 * math.pi * q1 + 4 * math.pi * q2))
        # B half a step ahead of E (B^{n+1/2} with E^n)
        tm_A3_B3 = lambda q1, q2, p: (torch.sin(2 * math.pi * (q1 - 0.5 * dt)
                                                + 4 * math.pi * (q2 - 0.5 * dt)), 0 * q1)
        nls = _fdtd_mode1_solver(N, dt, tm_A3_B3, tm_E)
        q1, q2 = nls.q1_center, nls.q2_center
        y0 = _yee(nls).clone()
        n = 2 * N                                               # t = 1: one drive period
        for k in range(1, n + 1):
            t = k * dt - 0.5 * dt                               # currents at n + 1/2
            J3 = -16 * math.pi ** 2 * torch.sin(2 * math.pi * (q1 - t) + 4 * math.pi * (q2 - t))
            nls.fields_solver.evolve_electrodynamic_fields(0, 0, J3, dt)
        y1 = _yee(nls)
        g = nls.N_ghost
        for c in errs:
            errs[c].append(float(torch.mean(torch.abs(_interior_q(y1[c] - y0[c], g)))))
    for c, e in errs.items():
        slope = np.polyfit(np.log10(Ns), np.log10(e), 1)[0]
        assert abs(slope + 2) < 0.25, (c, e, slope)


def test_fft_poisson_kat():
    """One p-cell of width 1, so the density is f itself; charge 1 and
    n = 2 - sin(2 pi q1 + 4 pi q2) give rho - mean(rho) = -sin(...)."""
    N = 1024
    spec = C.make(N_q1=N, N_q2=N, N_p1=1, N_p2=1, N_p3=1,
                  p1_start=[-0.5], p1_end=[0.5], p2_start=[-0.5], p2_end=[0.5],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[1.0], p_dim=1,
                  source_enabled=False, fields_enabled=True, fields_type='electrostatic',
                  fields_solver='fft', fields_initialize='fft')
    nls = make_solver(spec, 'fp64')
    q1, q2 = nls.q1_center, nls.q2_center
    theta = 2 * math.pi * q1 + 4 * math.pi * q2
    g = spec['N_ghost']
    E1x = (0.1 / math.pi) * torch.cos(theta)
    E2x = (0.2 / math.pi) * torch.cos(theta)

    def errors():
        c = nls.fields_solver.cell_centered_EM_fields
        return (float(torch.mean(torch.abs(_interior_q(c[0:1] - E1x, g)))),
                float(torch.mean(torch.abs(_interior_q(c[1:2] - E2x, g)))))
    nls.f = (2 - torch.sin(theta)).expand_as(nls.f)
    nls.df_dt()                                  # the electrostatic solve of the CUDA path
    e1, e2 = errors()
    assert e1 < 1e-14 and e2 < 1e-14, (e1, e2)
    # the solve at construction, from the initial f of the same density
    def init_f(q1, q2, p1, p2, p3, params):
        return (2 - torch.sin(2 * math.pi * q1 + 4 * math.pi * q2)) * p1 ** 0
    from bolt_b200.physical_system import physical_system
    from bolt_b200.nonlinear_solver import nonlinear_solver
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    dom, bc, params, initialize = build_modules(spec, 'fp64', None)
    initialize.initialize_f = init_f
    nls = nonlinear_solver(physical_system(dom, bc, params, initialize, adv, col.BGK, mom))
    e1, e2 = errors()
    assert e1 < 1e-14 and e2 < 1e-14, (e1, e2)
