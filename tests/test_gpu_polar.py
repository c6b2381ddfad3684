"""The polar2D p-space grid (params.p_space_grid = 'polar2D'; p1 the radius,
p2 the angle over a full turn) on the CUDA path.

Parity with the reference fixtures of the polar2D cases runs with the other
cases (test_gpu_parity.py, test_gpu_asl.py).  These tests pin the two rules
the grid changes one at a time:
  * every moment carries the factor initial_mu (compute_moments.py:48-53):
    the polar2D moments of an f equal initial_mu times the cartesian moments
    of the same f on the same grid, exactly (one FP64 product);
  * a mirror edge reflects the angle (boundaries.py:313-413): theta -> -theta
    at q2 edges, theta -> pi - theta at q1 edges, checked cell by cell
    against the oracle's halo refresh;
and the configuration the path refuses: a q1 mirror edge with an odd N_p2
(the reference splits the angle range in two halves)."""

import copy

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout, moments_layout
from _util import rel
from oracle.bolt_oracle import Oracle

NAME = 'polar2d_mirror_2d2v_rk4'
MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy', 'energy_q1',
           'q_q2')


@pytest.mark.gpu
def test_polar_moments_are_initial_mu_times_cartesian():
    spec = C.CASES[NAME]
    polar = make_solver(spec)
    cart_spec = copy.deepcopy(spec)
    cart_spec['p_space_grid'] = 'cartesian'
    cart = make_solver(cart_spec)
    mu = spec['initial_mu']
    for name in MOMENTS:
        a = moments_layout(polar.compute_moments(name, f=polar.f))
        b = moments_layout(cart.compute_moments(name, f=polar.f))
        assert np.array_equal(a, mu * b), name


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['polar2d_mirror_2d2v_rk4',
                                  'polar2d_mirror_dirichlet_minmod_rk2'])
def test_polar_mirror_halo_matches_oracle(name):
    # the oracle refreshes the solver's own f, so mirror ghosts (pure copies)
    # must agree bit for bit; Dirichlet inflow values are evaluated by torch
    # in the solver and by numpy in the oracle (1e-14)
    spec = C.CASES[name]
    nls = make_solver(spec)
    o = Oracle(spec, to_layout(nls.f, spec))
    if 'dirichlet' in spec:
        o.dirichlet = C.dirichlet_values(spec)
    nls._communicate_f()
    nls._apply_bcs_f()
    got = to_layout(nls.f, spec)
    want = o.refresh(o.f)
    if 'dirichlet' in spec:
        assert rel(got, want) < 1e-14
    else:
        assert np.array_equal(got, want), rel(got, want)


@pytest.mark.gpu
def test_polar_refuses_odd_angle_count_at_q1_mirror():
    spec = copy.deepcopy(C.CASES[NAME])
    spec['N_p2'] = 7
    with pytest.raises(Exception) as e:
        make_solver(spec)
    assert 'unsupported' in str(e.value)
    # an odd angle count is fine with q2 mirrors only (no halves to split)
    spec['bc_q1'] = 'periodic'
    nls = make_solver(spec)
    torch.cuda.synchronize()
    assert nls.f.shape[1] == 1
