"""print_performance_timings (performance_timings.py:9-165): with
performance_test_flag=True the solver times every step and every launch group
with CUDA events.  The parts (ghost pass, moments, q-stage, p-stage, field
solve) lie inside the step's own events, so they sum to no more than the
timestep total; the table ends with Spatial Zone Cycles/s."""

import pytest

import cases as C
from _modules import build_modules

pytestmark = pytest.mark.gpu


def _solver(spec, precision):
    from bolt_b200.physical_system import physical_system
    from bolt_b200.nonlinear_solver import nonlinear_solver
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    dom, bc, params, ini = build_modules(spec, precision)
    return nonlinear_solver(physical_system(dom, bc, params, ini, adv, col.BGK, mom),
                            performance_test_flag=True)


@pytest.mark.parametrize('name,precision', [('c3_2d3v_weno5_rk4_small', 'fp32'),
                                            ('c2_2d2v_fdtd_rk4_small', 'fp64'),
                                            ('dirichlet_2d2v_minmod', 'fp64')])
def test_component_timings(name, precision, capsys):
    spec = C.CASES[name]
    nls = _solver(spec, precision)
    n = 4
    for _ in range(n):
        nls.strang_timestep(spec['dt'])
    t = nls.performance_timings()
    assert t['timestep'] > 0 and t['q-stage'] > 0
    assert all(v >= 0 for v in t.values())
    parts = sum(v for k, v in t.items() if k != 'timestep')
    assert parts <= t['timestep'] * 1.02 + 1e-5, t
    if spec['fields_enabled']:
        assert t['p-stage'] > 0 and t['fields'] > 0
    else:
        assert t['p-stage'] == 0 and t['fields'] == 0
    if spec['bc_q1'] == 'dirichlet':
        assert t['ghosts'] > 0
    nls.strang_timestep(spec['dt'])
    nls.print_performance_timings(n + 1)
    out = capsys.readouterr().out
    assert 'TIMESTEP' in out and 'Spatial Zone Cycles/s' in out
    nls.synchronize()
