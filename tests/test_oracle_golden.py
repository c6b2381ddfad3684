"""The oracle against fixtures produced by the unmodified Bolt source
(tests/golden/make_golden.py) and against the analytic known-answer tests of
Bolt's own unit tests.  CPU only."""

import numpy as np
import pytest

import cases as C
from _util import load_golden, rel, interior, moment_errors, check_compact
from oracle.bolt_oracle import Oracle, Grid, moment

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')


@pytest.mark.parametrize('name', C.ASL_NAMES)
def test_oracle_asl_matches_reference(name):
    """Semi-Lagrangian q-advection split with the BGK source (Strang, Lie,
    SWSS, Jia; instantaneous and collisionless variants; periodic and mirror
    walls; a characteristic crossing 1.7 cells per step; with electrostatic
    fields split again with the FVM in p) against the
    reference's own operators run over the numpy stand-ins, whose approx2 is
    the Catmull-Rom restatement the oracle shares (so the interpolation itself
    is unpinned; everything around it -- back-tracing, ghost refresh, source
    RK2, splitting -- is pinned): f and moments to 1e-13."""
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    f0 = C.initial_f(spec)
    assert rel(interior(f0, g), G['f0']) < 1e-14
    o = Oracle(spec, f0)
    assert rel(o.refresh(o.f), G['f0_refreshed']) < 1e-14
    for _ in range(spec['steps']):
        o.split_step(spec['dt'])
    assert rel(interior(o.f, g), G['f_final']) < 1e-13
    if spec['fields_enabled']:
        assert rel(o.fields.cell, G['fields_cell']) < 1e-11
    m = {k: interior(o.moments(k), g) for k in MOMENTS}
    errs = moment_errors(m, {k: G['mom_' + k] for k in MOMENTS})
    assert max(errs.values()) < 1e-13, errs
    assert abs(o.time_elapsed - float(G['time_elapsed'])) < 1e-15


def test_catmull_rom_interpolation_known_answers():
    """The interpolation restated for approx2(BICUBIC_SPLINE): exact on
    quadratics between interior samples (a Catmull-Rom spline reproduces
    them), the samples themselves at integer positions, 0 off the grid."""
    from oracle.bolt_oracle import interp2_catmull_rom
    n2, n1 = 9, 11
    j, i = np.meshgrid(np.arange(n2), np.arange(n1), indexing='ij')
    a = (1.0 + 0.5 * i - 0.25 * j + 0.125 * i * j)[:, :, None]
    x = (i + 0.37)[:, :, None]
    y = (j - 0.61)[:, :, None]
    got = interp2_catmull_rom(a, x, y)[:, :, 0]
    want = 1.0 + 0.5 * x[:, :, 0] - 0.25 * y[:, :, 0] + 0.125 * x[:, :, 0] * y[:, :, 0]
    inner = (slice(2, n2 - 1), slice(1, n1 - 3))
    assert np.abs(got[inner] - want[inner]).max() < 1e-13
    assert np.array_equal(interp2_catmull_rom(a, i[:, :, None] + 0.0, j[:, :, None] + 0.0), a)
    assert got[0, 0] == 0.0 and got[-1, -1] == 0.0          # y < 0; x > n1 - 1


@pytest.mark.parametrize('name', C.FVM_NAMES)
def test_oracle_matches_reference(name):
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    f0 = C.initial_f(spec)
    assert rel(interior(f0, g), G['f0']) < 1e-14
    user = C.field_functions(spec['field_init'], np.sin, np.cos) \
        if spec.get('field_init') else None
    o = Oracle(spec, f0, field_functions=user)
    o.dirichlet = C.dirichlet_values(spec)
    fr = o.refresh(o.f)
    assert rel(fr, G['f0_refreshed']) < 1e-14
    o.dt = spec['dt']
    at = getattr(o, 'at_n', None)
    d = o.dfdt(fr)
    if at is not None:
        o.at_n = at
    assert rel(interior(d, g), G['dfdt0']) < 1e-12
    if spec['fields_enabled']:
        assert rel(o.fields.cell, G['fields_cell0']) < 1e-11
        assert rel(o.fields.yee, G['fields_yee0']) < 1e-11
    for _ in range(spec['steps']):
        o.step(spec['dt'])
    assert rel(interior(o.f, g), G['f_final']) < 1e-12
    m = {k: interior(o.moments(k), g) for k in MOMENTS}
    errs = moment_errors(m, {k: G['mom_' + k] for k in MOMENTS})
    assert max(errs.values()) < 1e-12, errs
    if spec['fields_enabled']:
        assert rel(o.fields.cell, G['fields_cell']) < 1e-11
        assert rel(o.fields.yee, G['fields_yee']) < 1e-11
    assert abs(o.time_elapsed - float(G['time_elapsed'])) < 1e-15


def test_oracle_matches_reference_at_24c3():
    """The compact fixture of the bench's velocity grid (8x8 q x 24^3 p, WENO5,
    BGK, RK4): f0 rebuilt from the stored factors, df/dt of the refreshed
    state and f after three steps (in full at the stored q-cells, as per-q-cell
    velocity sums everywhere), and the moments."""
    name = 'c3_2d3v_weno5_rk4_p24'
    spec = C.COMPACT_CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    f0 = C.compact_f0(G)
    assert rel(interior(C.initial_f(spec), g), interior(f0, g)) < 1e-14
    o = Oracle(spec, C.periodic_wrap(f0, spec))
    o.dt = spec['dt']
    d = interior(o.dfdt(o.refresh(o.f)), g)
    for _ in range(spec['steps']):
        o.step(spec['dt'])
    m = {k: interior(o.moments(k), g) for k in MOMENTS}
    check_compact(spec, G, interior(o.f, g), m, dfdt0=d)


def test_moment_kat():
    """test_compute_moments.py:76-144: drifting Maxwellian on a 32^3 p-grid
    over [-10,10]^3, 16^2 q-grid; mean abs error < 1e-13 for n, E, momenta."""
    spec = C.make(N_q1=16, N_q2=16, N_p1=32, N_p2=32, N_p3=32, N_ghost=0,
                  p1_start=[-10.0], p1_end=[10.0], p2_start=[-10.0], p2_end=[10.0],
                  p3_start=[-10.0], p3_end=[10.0], mass=[1.0], charge=[0.0], p_dim=3)
    gr = Grid(spec)
    q1, q2 = gr.q1_center, gr.q2_center
    rho = 1 + 0.01 * np.sin(2 * np.pi * q1 + 4 * np.pi * q2)
    T = 1 + 0.01 * np.cos(2 * np.pi * q1 + 4 * np.pi * q2)
    pb = 0.01 * np.exp(-10 * q1 ** 2 - 10 * q2 ** 2)
    e = lambda a: a[:, :, None, None, None, None]
    p1, p2, p3 = gr.p1c[None, None], gr.p2c[None, None], gr.p3c[None, None]
    f = e(rho) * (1 / (2 * np.pi * e(T))) ** 1.5 * np.exp(-(p1 - e(pb)) ** 2 / (2 * e(T))) \
        * np.exp(-(p2 - e(pb)) ** 2 / (2 * e(T))) * np.exp(-(p3 - e(pb)) ** 2 / (2 * e(T)))
    n = moment(gr, f, 'density')[..., 0]
    E = moment(gr, f, 'energy')[..., 0]
    assert np.mean(np.abs(n - rho)) < 1e-13
    assert np.mean(np.abs(E - (1.5 * rho * T + 1.5 * rho * pb ** 2))) < 1e-13
    for name in ('mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk'):
        assert np.mean(np.abs(moment(gr, f, name)[..., 0] - rho * pb)) < 1e-13


def test_periodic_ghost_fill_kat():
    """test_apply_boundary_conditions.py:131-145 / test_communicate.py:168-182:
    periodic ghosts equal the analytic periodic function to < 5e-14."""
    spec = C.make(N_q1=32, N_q2=16, N_p1=2, N_p2=1, N_p3=1, N_ghost=3,
                  p1_start=[-1.0], p1_end=[1.0], p2_start=[-0.5], p2_end=[0.5],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1)
    o = Oracle(spec, np.zeros(Grid(spec).fshape))
    gr = o.g
    expected = np.sin(2 * np.pi * gr.q1_center + 4 * np.pi * gr.q2_center)
    f = np.zeros(gr.fshape)
    f[3:-3, 3:-3] = expected[3:-3, 3:-3, None, None, None, None]
    out = o.refresh(f)
    assert np.max(np.abs(out - expected[:, :, None, None, None, None])) < 5e-14


def test_rk_orders():
    """test_time_integrators.py:26-70: df/dt = f integrated to t = 1, slope of
    log(error) vs log(N) within 0.2 of -2 (RK2) and -4 (RK4), using the
    oracle's stage formulas."""
    def rk2(x, dt):
        x_half = x + x * (dt / 2)
        return x + x_half * dt

    def rk4(x, dt):
        k1 = x; k2 = x + 0.5 * k1 * dt; k3 = x + 0.5 * k2 * dt; k4 = x + k3 * dt
        return x + ((k1 + 2 * k2 + 2 * k3 + k4) / 6) * dt
    for fn, order, ns in ((rk2, 2, 10 ** np.arange(4)), (rk4, 4, 10 ** np.arange(3))):
        err = []
        for n in ns:
            x = 1.0
            for _ in range(n):
                x = fn(x, 1.0 / n)
            err.append(abs(x - np.e))
        slope = np.polyfit(np.log10(ns), np.log10(err), 1)[0]
        assert abs(slope + order) < 0.2


def test_reference_restart_files_parse():
    """The PETSc binary Vecs the reference dumped (tests/golden/dumps) read back
    with the solver's reader and are re-written byte-for-byte by its writer."""
    import os
    import tempfile
    from bolt_b200.nonlinear_solver import _read_petsc_vec, _write_petsc_vec
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'dumps')
    state = np.load(os.path.join(d, 'c3_2d3v_weno5_rk4_small_state.npz'))
    vals = _read_petsc_vec(os.path.join(d, 'c3_2d3v_weno5_rk4_small_f.bin'))
    assert np.array_equal(vals, state['f'].reshape(-1))
    with tempfile.TemporaryDirectory() as t:
        _write_petsc_vec(os.path.join(t, 'x.bin'), vals)
        a = open(os.path.join(t, 'x.bin'), 'rb').read()
        b = open(os.path.join(d, 'c3_2d3v_weno5_rk4_small_f.bin'), 'rb').read()
        assert a == b


def test_fdtd_tm_mode_with_currents_second_order():
    """test_fdtd_explicit_with_currents.py:97-159 on the oracle's FDTD: the TM
    mode driven by J3 = -16 pi^2 sin(phi), set up on the Yee positions of
    fields.py's initialisation (E3, A3 and J3 at the cell centre, B from A3
    by backward differences), returns to its initial state after one drive
    period with error O(N^-2) (slope within 0.25 of -2)."""
    import math
    Ns = [32, 64, 128]
    errs = {2: [], 3: [], 4: []}
    for N in Ns:
        dt = 0.5 / N
        spec = C.make(N_q1=N, N_q2=N, N_p1=4, N_p2=4, N_p3=1, p1_start=[-1.0], p1_end=[1.0],
                      p2_start=[-1.0], p2_end=[1.0], p3_start=[-0.5], p3_end=[0.5],
                      mass=[1.0], charge=[0.0], p_dim=2, source_enabled=False,
                      fields_enabled=True, fields_initialize='user-defined')
        tp = 2 * math.pi
        user = {'initialize_E': lambda q1, q2, p: (0 * q1, 0 * q1,
                                                   3 * tp * np.cos(tp * q1 + 2 * tp * q2)),
                'initialize_A3_B3': lambda q1, q2, p: (
                    np.sin(tp * (q1 - 0.5 * dt) + 2 * tp * (q2 - 0.5 * dt)), 0 * q1)}
        o = Oracle(spec, np.ones(Grid(spec).fshape), field_functions=user)
        y0 = o.fields.yee.copy()
        q1, q2 = o.g.q1_center, o.g.q2_center
        for k in range(1, 2 * N + 1):
            t = (k - 0.5) * dt
            J3 = -4 * tp ** 2 * np.sin(tp * (q1 - t) + 2 * tp * (q2 - t))
            o.fields.evolve(0 * q1, 0 * q1, J3, dt)
        for c in errs:
            errs[c].append(np.mean(np.abs(interior(o.fields.yee[c] - y0[c], 3))))
    for c, e in errs.items():
        slope = np.polyfit(np.log10(Ns), np.log10(e), 1)[0]
        assert abs(slope + 2) < 0.25, (c, e, slope)


def shear_spec(N, axis):
    """The reference's shearing-box known-answer setup
    (test_shearing_boundaries/test_shear.py:22-88): N x N q-grid on [0, 1]^2,
    one p-cell, density 1 + 0.01 sin-like wave along the sheared axis
    (here 1 + 0.01 cos(2 pi q)), q = omega = 1; the other axis periodic."""
    bc = dict(bc_q1='shearing-box', bc_q2='periodic') if axis == 1 else \
        dict(bc_q1='periodic', bc_q2='shearing-box')
    k = dict(k1=0, k2=1) if axis == 1 else dict(k1=1, k2=0)
    return C.make(N_q1=N, N_q2=N, N_p1=1, N_p2=1, N_p3=1, p1_start=[-0.5], p1_end=[0.5],
                  p2_start=[-0.5], p2_end=[0.5], p3_start=[-0.5], p3_end=[0.5], mass=[1.0],
                  charge=[0.0], p_dim=3, shear_q=1.0, shear_omega=1.0,
                  init=dict(amp=0.01, **k), **bc)


def shear_errors(spec, fghost_fn, t, axis):
    """Mean |ghost - exact| over both strips' interior rows (columns): the
    exact values are the initial density at the sheared, wrapped positions."""
    g = spec['N_ghost']
    N = spec['N_q1']
    centres = (np.arange(-g, N + g) + 0.5) / N
    vel = float(C.maxwellian_p(spec, 0, 0.0, 0.0, 0.0))    # the single p-cell's factor
    err = 0.0
    for side, sgn in (('lo', -1), ('hi', +1)):
        pos = np.mod(centres + sgn * t, 1.0)
        exact = (1 + 0.01 * np.cos(2 * np.pi * pos)) * vel
        got = fghost_fn(side)                     # (N_rows of the strip, N_g)
        err += np.mean(np.abs(got - exact[g:N + g, None]))
    return err


@pytest.mark.parametrize('axis', [1, 2])
def test_shearing_box_kat_third_order(axis):
    """boundaries.py:6-145 on the oracle: after the halo refresh at time t the
    ghost strips equal the initial data shifted by -/+ q omega L t along the
    other axis, with error O(N^-3) (slope of log error vs log N within 0.3 of
    -3, as test_shear.py asserts) for N = 32 .. 512.  The error constant
    depends on where the shift falls within a cell, so each N sums the errors
    of seven shifts spread over the period (test_shear.py draws one at
    random)."""
    Ns = [32, 64, 128, 256, 512]
    errs = []
    for N in Ns:
        spec = shear_spec(N, axis)
        o = Oracle(spec, C.initial_f(spec))
        g = spec['N_ghost']
        e = 0.0
        for t in np.linspace(0.11, 0.89, 7):
            o.time_elapsed = t
            out = o.refresh(o.f)[..., 0, 0, 0, 0]     # (Nq2g, Nq1g)

            def strip(side):
                if axis == 1:
                    return out[g:N + g, :g] if side == 'lo' else out[g:N + g, N + g:]
                return (out[:g, g:N + g] if side == 'lo' else out[N + g:, g:N + g]).T
            e += shear_errors(spec, strip, t, axis)
        errs.append(e)
    slope = np.polyfit(np.log10(Ns), np.log10(errs), 1)[0]
    assert abs(slope + 3) < 0.3, (errs, slope)
