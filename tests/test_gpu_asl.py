"""The advective semi-Lagrangian (ASL) method in q on the GPU
(bolt_asl_advect_q / bolt_asl_source through nonlinear_solver's splitting
timesteps; with electrostatic fields split again with bolt_fvm_p_step, the
FVM in p) against the reference's own ASL operators
(asl_operators.py:20-83, operator_splitting_methods.py) run over the numpy
stand-ins (tests/golden/make_golden.py), whose approx2 is the Catmull-Rom
restatement the CUDA kernel also follows.  Driven from the fixture's
halo-refreshed initial state, f and the moments after the case's steps:
FP64 1e-12, FP32 2e-6; the electrostatic fields FP64 1e-10, FP32 1e-3 (the
FFT solve of a density with 1e-2 noise, which FP32 f resolves to ~1e-4)."""

import numpy as np
import pytest
import torch

import bolt_b200._native as N
import cases as C
from _modules import make_solver, to_layout, moments_layout
from _util import load_golden, rel, interior, moment_errors

pytestmark = pytest.mark.gpu

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')


def _af(a):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.reshape(t.shape[0], t.shape[1], t.shape[2], -1).permute(3, 2, 1, 0)


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-12), ('fp32', 2e-6),
                                           ('fp64-fast', 1e-12)])
@pytest.mark.parametrize('name', C.ASL_NAMES)
def test_asl_matches_reference(name, precision, tol):
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    nls.f = _af(G['f0_refreshed']).to('cuda')
    step = getattr(nls, spec['splitting'] + '_timestep')
    launches = nls.launch_count()
    for _ in range(spec['steps']):
        step(spec['dt'])
    torch.cuda.synchronize()
    assert nls.launch_count() > launches              # the CUDA kernels ran
    e = rel(interior(to_layout(nls.f, spec), g), G['f_final'])
    assert e < tol, e
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    errs = moment_errors(m, {k: G['mom_' + k] for k in MOMENTS})
    assert max(errs.values()) < tol, errs
    if spec['fields_enabled']:
        cell = nls.fields_solver.cell_centered_EM_fields[:, 0].permute(0, 2, 1).cpu().numpy()
        e = rel(cell, G['fields_cell'])
        assert e < (1e-10 if precision != 'fp32' else 1e-3), ('fields', e)
    assert abs(nls.time_elapsed - float(G['time_elapsed'])) < 1e-12
    nls.synchronize()


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
@pytest.mark.parametrize('scheme', ['strang', 'lie'])
def test_asl_buffer_passing_step_equals_in_place_operators(scheme, precision):
    """The Strang and Lie steps hand f between the operators through the
    context's work buffer (bolt_asl_advect_q_to / bolt_asl_source_to, no copy
    back); the in-place operators composed by hand (bolt_asl_advect_q /
    bolt_asl_source, each writing f) give the same f bit for bit."""
    spec = dict(C.CASES['asl_2d2v_lie'])
    spec['splitting'] = scheme
    a = make_solver(spec, precision)
    b = make_solver(spec, precision)
    b.f = a.f.clone()
    dt = spec['dt']
    for _ in range(3):
        getattr(a, scheme + '_timestep')(dt)
        if scheme == 'strang':
            b._op_advect_q(0.5 * dt)
            b._op_solve_src(dt)
            b._op_advect_q(0.5 * dt)
        else:
            b._op_advect_q(dt)
            b._op_solve_src(dt)
    torch.cuda.synchronize()
    g = spec['N_ghost']
    fa, fb = interior(to_layout(a.f, spec), g), interior(to_layout(b.f, spec), g)
    assert np.array_equal(fa, fb)
    # the buffer forms refuse aliasing they cannot honour
    fp, w = a._fstore.data_ptr(), a._work_buffer()
    assert a._lib.bolt_asl_advect_q_to(a._ctx, fp, fp, float(dt), a._stream()) == N.BOLT_ERR_ARG
    assert a._lib.bolt_asl_source_to(a._ctx, w, fp, w, float(dt), 0,
                                     a._stream()) == N.BOLT_ERR_ARG
    a.synchronize()
    b.synchronize()


def test_asl_advection_of_a_linear_profile_is_exact():
    """Collisionless, one velocity: a profile linear in q1 over the interior
    of a mirror-free periodic grid is carried by exactly p1 dt (the
    Catmull-Rom cubic reproduces it) wherever the feet stay in the interior."""
    spec = C.make(N_q1=32, N_q2=1, N_p1=1, N_p2=1, N_p3=1,
                  p1_start=[0.45], p1_end=[0.55], p2_start=[-0.5], p2_end=[0.5],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
                  solver_q='ASL', splitting='lie', source_enabled=False, tau=1.0,
                  dt=0.01, steps=1)
    nls = make_solver(spec, 'fp64')
    g = spec['N_ghost']
    q1 = nls.q1_center                                  # (1, 1, Nq1g, Nq2g)
    nls.f = (2.0 + 3.0 * q1).expand_as(nls.f).clone()
    nls.lie_timestep(spec['dt'])
    got = nls.f[0, 0, :, g].double()
    want = 2.0 + 3.0 * (q1[0, 0, :, g].double() - 0.5 * spec['dt'])
    inner = slice(g + 2, 32 + g - 2)
    assert float((got[inner] - want[inner]).abs().max()) < 1e-13


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_asl_nan_raises_solver_diverging(precision):
    """A NaN written into f from the host reaches the interpolation and the
    source; their kernels raise the divergence flag, and the timestep raises
    SystemExit('Solver Diverging!') (timestep.py:28-38)."""
    spec = C.CASES['asl_2d2v_lie']
    nls = make_solver(spec, precision)
    nls.lie_timestep(spec['dt'])
    torch.cuda.synchronize()
    nls.check_divergence()                          # a clean step leaves no flag
    f = nls.f.clone()
    g = spec['N_ghost']
    f[3, 0, g + 5, g + 4] = float('nan')
    nls.f = f
    with pytest.raises(SystemExit, match='Solver Diverging!'):
        for _ in range(3):
            nls.lie_timestep(spec['dt'])
            torch.cuda.synchronize()
    nls.synchronize()
