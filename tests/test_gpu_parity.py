"""CUDA path vs the golden fixtures of the reference run and vs the oracle.

FP64: df/dt, f after the case's steps, moments and fields within 1e-12
normwise relative (the bar stated for the reference's FP64 path).
FP32 (f and stencils in FP32, moments/Maxwellian in FP64): 2e-6 normwise on
f after the steps and 1e-5 on df/dt."""

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout, moments_layout
from _util import load_golden, rel, interior, moment_errors

pytestmark = pytest.mark.gpu

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')
NAMES = sorted(C.CASES)


def _check_case(name, precision, tol_dfdt, tol_f, tol_mom):
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    f0 = to_layout(nls.f, spec)
    assert rel(interior(f0, g), G['f0']) < (1e-14 if precision == 'fp64' else 1e-7)
    if spec['fields_enabled']:
        cell = nls.fields_solver.cell_centered_EM_fields[:, 0].permute(0, 2, 1).cpu().numpy()
        assert rel(cell, G['fields_cell0']) < 1e-11
    nls.dt = spec['dt']
    d = to_layout(nls.df_dt(), spec)
    if spec['fields_enabled']:
        nls.fields_solver.at_n = True
    e = rel(interior(d, g), G['dfdt0'])
    assert e < tol_dfdt, ('dfdt', e)
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    torch.cuda.synchronize()
    e = rel(interior(to_layout(nls.f, spec), g), G['f_final'])
    assert e < tol_f, ('f', e)
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    errs = moment_errors(m, {k: G['mom_' + k] for k in MOMENTS})
    assert max(errs.values()) < tol_mom, errs
    if spec['fields_enabled'] and precision == 'fp64':
        cell = nls.fields_solver.cell_centered_EM_fields[:, 0].permute(0, 2, 1).cpu().numpy()
        assert rel(cell, G['fields_cell']) < 1e-10
    assert abs(nls.time_elapsed - float(G['time_elapsed'])) < 1e-12
    nls.synchronize()


@pytest.mark.parametrize('name', NAMES)
def test_fp64_matches_reference(name):
    _check_case(name, 'fp64', 1e-12, 1e-12, 1e-12)


@pytest.mark.parametrize('name', ['c1_1d1v_weno5_rk2', 'c3_2d3v_weno5_rk4_small',
                                  'c2_2d2v_fdtd_rk4_small', 'minmod_2d2v_fields_bgk',
                                  'ppm_2d2v_fields_bgk', 'dirichlet_1d1v_weno5'])
def test_fp32_close_to_reference(name):
    _check_case(name, 'fp32', 1e-4, 2e-6, 2e-6)
