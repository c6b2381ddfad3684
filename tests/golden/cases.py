"""Seeded synthetic cases for parity tests.

Each case is a plain dict (the "spec") naming the grid, boundary conditions,
physics switches and initial condition.  The same spec drives
  * the Bolt reference run over numpy stand-ins (make_golden.py, this container only),
  * the numpy oracle (oracle/bolt_oracle.py),
  * the CUDA path through bolt_b200's physical_system / nonlinear_solver API.

Initial conditions (evaluated at cell centres, ghost cells included):
  n(q)  = base * (1 + amp * cos(2 pi k1 q1) * cos(2 pi k2 q2)) * (1 + noise * xi(q))
  f     = n * prod_{d < p_dim} sqrt(m / (2 pi k T_d)) exp(-m (p_d - u_d)^2 / (2 k T_d))
xi is N(0,1) per interior q-cell from numpy.random.default_rng(seed), extended
periodically into the ghost cells.
"""

import copy
import numpy as np

BASE = dict(
    q1_start=0.0, q1_end=1.0, q2_start=0.0, q2_end=1.0,
    N_ghost=3, bc_q1='periodic', bc_q2='periodic',
    boltzmann_constant=1.0, eps=1.0, mu=1.0,
    recon_q='weno5', recon_p='weno5',
    riemann_q='upwind-flux', riemann_p='upwind-flux',
    source_enabled=True, fields_enabled=False,
    fields_type='electrodynamic', fields_initialize='fft', fields_solver='fdtd',
    integrator='RK2', tau=0.01,
    init=dict(base=1.0, amp=0.0, k1=1, k2=0, noise=0.0, seed=0,
              T=[1.0, 1.0, 1.0], u=[0.0, 0.0, 0.0]),
)


def make(**kw):
    s = copy.deepcopy(BASE)
    init = kw.pop('init', {})
    s.update(kw)
    s['init'].update(init)
    return s


CASES = {
    # 1D1V BGK relaxation 64 x 128, WENO5, RK2, dt=1e-4, 100 steps
    'c1_1d1v_weno5_rk2': make(
        N_q1=64, N_q2=1, N_p1=128, N_p2=1, N_p3=1,
        p1_start=[-10.0], p1_end=[10.0], p2_start=[-0.5], p2_end=[0.5],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
        tau=0.01, dt=1e-4, steps=100,
        init=dict(amp=0.01, k1=1, k2=0)),
    # same, RK4 (restated integrators.RK4 around df_dt_fvm), LLF
    'c1_1d1v_weno5_rk4_llf': make(
        N_q1=64, N_q2=1, N_p1=128, N_p2=1, N_p3=1,
        p1_start=[-10.0], p1_end=[10.0], p2_start=[-0.5], p2_end=[0.5],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
        tau=0.01, dt=1e-4, steps=20, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.01, k1=1, k2=0)),
    # reduced 2D3V throughput case: BGK tau=0.05, WENO5, RK4
    'c3_2d3v_weno5_rk4_small': make(
        N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=8,
        p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
        p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
        tau=0.05, dt=1e-3, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.05, k1=1, k2=1)),
    # reduced 2D2V electromagnetic FDTD case, collisionless, RK2 (reference scheme)
    'c2_2d2v_fdtd_rk2_small': make(
        N_q1=8, N_q2=8, N_p1=16, N_p2=16, N_p3=1,
        p1_start=[-8.0], p1_end=[8.0], p2_start=[-8.0], p2_end=[8.0],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
        source_enabled=False, fields_enabled=True, dt=5e-4, steps=4,
        init=dict(T=[2.0, 1.0, 1.0], noise=1e-3, seed=0)),
    # same with RK4: fields advance once per step in stage 2
    'c2_2d2v_fdtd_rk4_small': make(
        N_q1=8, N_q2=8, N_p1=16, N_p2=16, N_p3=1,
        p1_start=[-8.0], p1_end=[8.0], p2_start=[-8.0], p2_end=[8.0],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
        source_enabled=False, fields_enabled=True, dt=5e-4, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(T=[2.0, 1.0, 1.0], noise=1e-3, seed=0)),
    # minmod in q and p, fields and BGK together
    'minmod_2d2v_fields_bgk': make(
        N_q1=8, N_q2=6, N_p1=10, N_p2=8, N_p3=1,
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
        recon_q='minmod', recon_p='minmod', fields_enabled=True, tau=0.1,
        dt=1e-3, steps=3, init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=3,
                                     u=[0.3, -0.2, 0.0])),
    # PPM in q and p
    'ppm_2d2v_fields_bgk': make(
        N_q1=8, N_q2=6, N_p1=10, N_p2=8, N_p3=1,
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
        recon_q='ppm', recon_p='ppm', fields_enabled=True, tau=0.1,
        dt=1e-3, steps=3, init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=4,
                                     u=[0.3, -0.2, 0.0])),
    # piecewise-constant, 2D3V with fields (exercises the p3 axis)
    'pc_2d3v_fields': make(
        N_q1=6, N_q2=4, N_p1=6, N_p2=6, N_p3=4,
        p1_start=[-4.0], p1_end=[4.0], p2_start=[-4.0], p2_end=[4.0],
        p3_start=[-4.0], p3_end=[4.0], mass=[1.0], charge=[-1.0], p_dim=3,
        recon_q='piecewise-constant', recon_p='piecewise-constant',
        fields_enabled=True, tau=0.2, dt=1e-3, steps=2,
        init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=5, u=[0.2, 0.1, -0.1])),
    # Dirichlet inflow along q1, WENO5, BGK, RK2
    'dirichlet_1d1v_weno5': make(
        N_q1=16, N_q2=1, N_p1=32, N_p2=1, N_p3=1,
        p1_start=[-6.0], p1_end=[6.0], p2_start=[-0.5], p2_end=[0.5],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
        bc_q1='dirichlet', tau=0.05, dt=2e-3, steps=5,
        dirichlet=dict(left=dict(base=1.5, T=[1.0, 1.0, 1.0], u=[0.5, 0, 0]),
                       right=dict(base=0.5, T=[2.0, 1.0, 1.0], u=[-0.5, 0, 0])),
        init=dict(amp=0.1, k1=1, k2=0)),
    # Dirichlet on both q axes, 2D2V, minmod, collisionless
    'dirichlet_2d2v_minmod': make(
        N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=1,
        p1_start=[-4.0], p1_end=[4.0], p2_start=[-4.0], p2_end=[4.0],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=2,
        bc_q1='dirichlet', bc_q2='dirichlet', recon_q='minmod', recon_p='minmod',
        source_enabled=False, dt=2e-3, steps=3,
        dirichlet=dict(left=dict(base=1.2, T=[1.0, 1.0, 1.0], u=[0.3, 0.1, 0]),
                       right=dict(base=0.8, T=[1.0, 1.0, 1.0], u=[-0.3, 0, 0]),
                       bottom=dict(base=1.1, T=[1.0, 1.0, 1.0], u=[0.0, 0.4, 0]),
                       top=dict(base=0.9, T=[1.0, 1.0, 1.0], u=[0.0, -0.4, 0])),
        init=dict(amp=0.1, k1=1, k2=1)),
    # mirror walls on both q axes (boundaries.py:226-301), a drifting,
    # anisotropic 2D2V gas reflecting off them, WENO5, BGK, RK2
    'mirror_2d2v_weno5': make(
        N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=1,
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=2,
        bc_q1='mirror', bc_q2='mirror', tau=0.05, dt=2e-3, steps=4,
        init=dict(amp=0.1, k1=1, k2=1, u=[0.4, -0.3, 0.0], T=[1.0, 1.5, 1.0])),
    # mirror + Dirichlet inflow along q1, periodic q2, 2D3V, LLF, RK4
    'mirror_dirichlet_2d3v_rk4': make(
        N_q1=8, N_q2=8, N_p1=8, N_p2=4, N_p3=4,
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
        bc_q1='mirror+dirichlet', tau=0.05, dt=2e-3, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        dirichlet=dict(left=dict(base=1.3, T=[1.0, 1.0, 1.0], u=[0.5, 0.1, 0]),
                       right=dict(base=0.7, T=[1.5, 1.0, 1.0], u=[-0.4, 0, 0])),
        init=dict(amp=0.1, k1=1, k2=2, u=[-0.2, 0.3, 0.1])),
    # electrostatic fields re-solved by FFT at every df/dt (Vlasov-Poisson):
    # Landau damping as the reference's landau_damping/linear example sets it
    # up (uniform along a 3-cell q2, minmod, upwind, collisionless), RK2
    'es_1d1v_landau_rk2': make(
        N_q1=32, N_q2=3, N_p1=48, N_p2=1, N_p3=1, recon_q='minmod', recon_p='minmod',
        p1_start=[-6.0], p1_end=[6.0], p2_start=[-0.5], p2_end=[0.5],
        p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=1,
        source_enabled=False, fields_enabled=True,
        fields_type='electrostatic', fields_solver='fft', dt=2e-3, steps=5,
        init=dict(amp=0.05, k1=1, k2=0)),
    # 2D2V electrostatic with BGK, two species, LLF, RK4
    'es_2d2v_two_species_rk4': make(
        N_q1=8, N_q2=6, N_p1=8, N_p2=8, N_p3=1,
        p1_start=[-5.0, -2.0], p1_end=[5.0, 2.0], p2_start=[-5.0, -2.0], p2_end=[5.0, 2.0],
        p3_start=[-0.5, -0.5], p3_end=[0.5, 0.5], mass=[1.0, 6.0], charge=[-1.0, 0.5],
        p_dim=2, fields_enabled=True, fields_type='electrostatic', fields_solver='fft',
        tau=0.1, dt=1e-3, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=11, u=[0.2, -0.1, 0.0])),
    # two species with different masses, charges and p-ranges, fields + BGK
    'two_species_2d2v_fields': make(
        N_q1=6, N_q2=4, N_p1=8, N_p2=6, N_p3=1,
        p1_start=[-5.0, -3.0], p1_end=[5.0, 3.0], p2_start=[-5.0, -3.0], p2_end=[5.0, 3.0],
        p3_start=[-0.5, -0.5], p3_end=[0.5, 0.5], mass=[1.0, 4.0], charge=[-1.0, 1.0],
        p_dim=2, fields_enabled=True, tau=0.1, dt=1e-3, steps=2,
        init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=6, T=[1.0, 1.5, 1.0])),
}

# a wider ghost zone than the stencil needs (the reference's halo tests draw
# N_ghost from 3..4: test_communicate.py, test_apply_boundary_conditions.py)
CASES['c3_2d3v_weno5_rk4_ghost4'] = make(
    N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=8, N_ghost=4,
    p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
    p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
    tau=0.05, dt=1e-3, steps=3, integrator='RK4',
    riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
    init=dict(amp=0.05, k1=1, k2=1, noise=1e-3, seed=4, u=[0.1, -0.2, 0.05]))

# The headline velocity grid, 24^3 p-cells per q-cell, on one 8x8 q-tile (the
# smallest grid the paired FP32 kernel takes): 13,824 p-cells are 432 chunks
# of 32, so most chunks start inside a p1 row and a p-split's first chunk at
# any p1 offset that is a multiple of 8.  Its f (0.9M cells) is too large to
# store whole, so make_golden.py writes a compact fixture (see compact()).
COMPACT_CASES = {
    'c3_2d3v_weno5_rk4_p24': make(
        N_q1=8, N_q2=8, N_p1=24, N_p2=24, N_p3=24,
        p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
        p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
        tau=0.05, dt=1e-3, steps=3, integrator='RK4', compact=True,
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.05, k1=1, k2=1)),
}
# interior (q2, q1) cells whose df/dt and f_final a compact fixture holds in full
COMPACT_SEL = ((0, 0), (7, 7), (2, 5), (5, 2))


def compact_f0(fx):
    """f0 with ghost cells from a compact fixture's factors: n_q[q2, q1] times
    v_p[p3, p2, p1], the single multiplication initialize_f ends with."""
    n, v = fx['n_q'], fx['v_p']
    return n[:, :, None, None, None, None] * v[None, None, None]


def periodic_wrap(a, spec):
    """The interior of a (Nq2g, Nq1g, ...) array with its ghost cells refilled
    periodically (communicate_f on a periodic grid)."""
    g = spec['N_ghost']
    inner = a[g:a.shape[0] - g, g:a.shape[1] - g]
    j = (np.arange(a.shape[0]) - g) % inner.shape[0]
    i = (np.arange(a.shape[1]) - g) % inner.shape[1]
    return inner[j][:, i]


def qcell_sums(spec, a):
    """Per q-cell and species velocity sums of an interior (Nq2, Nq1, Ns, Np3,
    Np2, Np1) array x: [sum x, sum v1 x, sum v2 x, sum v3 x, sum |v|^2 x,
    sum x^2] over p (no p-cell measure), shape (Nq2, Nq1, Ns, 6)."""
    out = np.empty(a.shape[:3] + (6,))
    for s in range(a.shape[2]):
        p1, p2, p3 = _pgrid(spec, s)
        x = a[:, :, s]
        sm = lambda y: y.sum(axis=(2, 3, 4))
        out[:, :, s, 0] = sm(x)
        out[:, :, s, 1] = sm(x * p1)
        out[:, :, s, 2] = sm(x * p2)
        out[:, :, s, 3] = sm(x * p3)
        out[:, :, s, 4] = sm(x * (p1 ** 2 + p2 ** 2 + p3 ** 2))
        out[:, :, s, 5] = sm(x * x)
    return out


# user-defined initial fields (fields.py:280-420): each form of the initialize
# module's field functions, FDTD-coupled 2D2V, reference scheme (RK2)
_FIELD_INIT_BASE = dict(
    N_q1=8, N_q2=6, N_p1=8, N_p2=6, N_p3=1,
    p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
    p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0],
    p_dim=2, fields_enabled=True, tau=0.1, dt=1e-3, steps=2,
    init=dict(amp=0.05, k1=1, k2=1, T=[1.0, 1.2, 1.0]))
for _name, _init, _form in (
        ('fields_user_E_B', 'user-defined', 'E_B'),
        ('fields_user_Aphi_A', 'user-defined', 'Aphi_A'),
        ('fields_user_E_A3B3', 'user-defined', 'E_A3B3'),
        ('fields_fft_user_B', 'fft + user-defined magnetic fields', 'B')):
    CASES[_name] = make(fields_initialize=_init, field_init=_form,
                        **copy.deepcopy(_FIELD_INIT_BASE))

# 2D3V with user-defined E and B: every field component nonzero, so each of
# the three p-flux divergences (term_to_return) is pinned
CASES['fields_user_E_B_2d3v'] = make(
    N_q1=6, N_q2=4, N_p1=6, N_p2=6, N_p3=4,
    p1_start=[-4.0], p1_end=[4.0], p2_start=[-4.0], p2_end=[4.0],
    p3_start=[-4.0], p3_end=[4.0], mass=[1.0], charge=[-1.0], p_dim=3,
    fields_enabled=True, fields_initialize='user-defined', field_init='E_B',
    tau=0.1, dt=1e-3, steps=2,
    init=dict(amp=0.05, k1=1, k2=1, T=[1.0, 1.2, 0.9], u=[0.1, -0.1, 0.2]))


# Advective semi-Lagrangian (ASL) in q (solver_method_in_q = 'ASL', fields
# off): the step splits q-advection (back-traced characteristics, bicubic
# interpolation) and the BGK source (RK2) by the named scheme
# (timestep.py, operator_splitting_methods.py, asl_operators.py:20-83)
_ASL_1D = dict(N_q1=64, N_q2=1, N_p1=64, N_p2=1, N_p3=1,
               p1_start=[-6.0], p1_end=[6.0], p2_start=[-0.5], p2_end=[0.5],
               p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
               solver_q='ASL', tau=0.05, dt=2e-3, steps=10,
               init=dict(amp=0.05, k1=1, k2=0, u=[0.2, 0.0, 0.0]))
_ASL_2D = dict(N_q1=16, N_q2=12, N_p1=10, N_p2=8, N_p3=1,
               p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
               p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=2,
               solver_q='ASL', tau=0.1, dt=5e-3, steps=5,
               init=dict(amp=0.1, k1=1, k2=1, u=[0.3, -0.2, 0.0], T=[1.0, 1.5, 1.0]))
CASES['asl_1d1v_strang'] = make(splitting='strang', **copy.deepcopy(_ASL_1D))
CASES['asl_1d1v_cfl17_lie'] = make(splitting='lie', **dict(copy.deepcopy(_ASL_1D),
                                                             dt=4.4e-3, steps=6))
CASES['asl_1d1v_instant_strang'] = make(splitting='strang', instantaneous=True,
                                        **copy.deepcopy(_ASL_1D))
CASES['asl_2d2v_lie'] = make(splitting='lie', **copy.deepcopy(_ASL_2D))
CASES['asl_2d2v_swss'] = make(splitting='swss', **copy.deepcopy(_ASL_2D))
CASES['asl_2d2v_jia'] = make(splitting='jia', **copy.deepcopy(_ASL_2D))
CASES['asl_2d2v_free_strang'] = make(splitting='strang', source_enabled=False,
                                     **copy.deepcopy(_ASL_2D))
CASES['asl_2d2v_mirror_strang'] = make(splitting='strang', bc_q1='mirror',
                                       **copy.deepcopy(_ASL_2D))
CASES['asl_2d3v_strang'] = make(
    N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=4,
    p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
    p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
    solver_q='ASL', splitting='strang', tau=0.05, dt=4e-3, steps=3,
    init=dict(amp=0.1, k1=1, k2=1, u=[0.2, -0.1, 0.05]))


# ASL in q with electrostatic fields and the FVM in p: the splitting of
# (op_advect_q, op_solve_src) and op_fvm, whose df/dt is then the p-part with
# the FFT field solve of its argument (timestep.py:134-148, df_dt_fvm.py:56-99)
CASES['asl_es_1d1v_strang'] = make(
    N_q1=32, N_q2=3, N_p1=48, N_p2=1, N_p3=1, recon_p='minmod',
    p1_start=[-6.0], p1_end=[6.0], p2_start=[-0.5], p2_end=[0.5],
    p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=1,
    solver_q='ASL', splitting='strang', source_enabled=False, fields_enabled=True,
    fields_type='electrostatic', fields_solver='fft', dt=2e-3, steps=5,
    init=dict(amp=0.05, k1=1, k2=0))
CASES['asl_es_2d2v_lie_rk4'] = make(
    N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=1,
    p1_start=[-5.0, -2.0], p1_end=[5.0, 2.0], p2_start=[-5.0, -2.0], p2_end=[5.0, 2.0],
    p3_start=[-0.5, -0.5], p3_end=[0.5, 0.5], mass=[1.0, 6.0], charge=[-1.0, 0.5],
    p_dim=2, solver_q='ASL', splitting='lie', fields_enabled=True,
    fields_type='electrostatic', fields_solver='fft', tau=0.1, dt=2e-3, steps=3,
    integrator='RK4', riemann_p='lax-friedrichs',
    init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=11, u=[0.2, -0.1, 0.0]))

# polar2D p-grid (p1 the radius, p2 the angle over a full turn): every moment
# scaled by initial_mu (compute_moments.py:48-53), mirror edges reflecting the
# angle (boundaries.py:313-413): both q axes mirrored, RK4, WENO5; a q1
# Dirichlet-inflow left edge (every radius moves inwards there) with the mirror
# on the right, minmod, RK2; and the semi-Lagrangian q-step between mirrors
_POLAR = dict(N_q1=8, N_q2=8, N_p1=8, N_p2=8, N_p3=1,
              p1_start=[0.0], p1_end=[4.0], p2_start=[-np.pi], p2_end=[np.pi],
              p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=2,
              p_space_grid='polar2D', initial_mu=0.7)
CASES['polar2d_mirror_2d2v_rk4'] = make(
    bc_q1='mirror', bc_q2='mirror', tau=0.05, dt=2e-3, steps=3, integrator='RK4',
    init=dict(amp=0.1, k1=1, k2=1, u=[1.5, 0.3, 0.0], T=[1.0, 0.8, 1.0]),
    **copy.deepcopy(_POLAR))
CASES['polar2d_mirror_dirichlet_minmod_rk2'] = make(
    bc_q1='mirror+dirichlet', recon_q='minmod', recon_p='minmod', tau=0.05, dt=2e-3,
    steps=3, dirichlet=dict(left=dict(base=1.2, T=[1.0, 1.0, 1.0], u=[1.0, 0.2, 0]),
                            right=dict(base=0.8, T=[1.2, 1.0, 1.0], u=[2.0, -0.1, 0])),
    init=dict(amp=0.1, k1=1, k2=2, u=[1.2, -0.2, 0.0], T=[1.0, 1.2, 1.0]),
    **copy.deepcopy(_POLAR))
# with fields: the charge density and the currents carry the factor too
# (df_dt_fvm.py:213-242), FDTD from the FFT initial solve, and the
# electrostatic FFT solve at every df/dt
CASES['polar2d_fdtd_2d2v_rk4'] = make(
    fields_enabled=True, tau=0.05, dt=1e-3, steps=3, integrator='RK4',
    init=dict(amp=0.1, k1=1, k2=1, noise=1e-2, seed=5, u=[1.5, 0.3, 0.0], T=[1.0, 0.8, 1.0]),
    **dict(copy.deepcopy(_POLAR), initial_mu=1.3, charge=[-1.0]))
CASES['polar2d_es_2d2v_rk2'] = make(
    fields_enabled=True, fields_type='electrostatic', fields_solver='fft',
    source_enabled=False, dt=1e-3, steps=3,
    init=dict(amp=0.1, k1=1, k2=0, u=[1.5, 0.3, 0.0], T=[1.0, 0.8, 1.0]),
    **dict(copy.deepcopy(_POLAR), initial_mu=1.3, charge=[-1.0]))
CASES['asl_polar2d_mirror_strang'] = make(
    solver_q='ASL', splitting='strang', bc_q1='mirror', bc_q2='mirror', tau=0.1, dt=5e-3,
    steps=3, init=dict(amp=0.1, k1=1, k2=1, u=[1.5, 0.3, 0.0], T=[1.0, 0.8, 1.0]),
    **copy.deepcopy(_POLAR))

# the finite-volume cases and the semi-Lagrangian ones
FVM_NAMES = sorted(n for n, s in CASES.items() if s.get('solver_q', 'FVM') == 'FVM')
ASL_NAMES = sorted(n for n, s in CASES.items() if s.get('solver_q', 'FVM') == 'ASL')


def field_functions(form, sin, cos):
    """The initialize-module field functions of the 'field_init' cases, written
    against a math namespace (numpy, torch, or the ArrayFire stand-in):
    E_B -> initialize_E, initialize_B; Aphi_A -> initialize_A_phi,
    initialize_A; E_A3B3 -> initialize_E, initialize_A3_B3; B -> initialize_B."""
    tp = 2 * np.pi

    def initialize_E(q1, q2, params):
        return (0.1 * sin(tp * q2), 0.05 * cos(tp * q1), 0.02 * sin(tp * (q1 + q2)))

    def initialize_B(q1, q2, params):
        return (0.03 * cos(tp * q2), 0.04 * sin(tp * q1), 0.5 + 0.02 * cos(tp * (q1 - q2)))

    def initialize_A_phi(q1, q2, params):
        return (0.02 * cos(tp * q2), 0.02 * sin(tp * q1), 0.03 * sin(tp * (q1 + q2)),
                0.01 * cos(tp * q1) * cos(tp * q2))

    def initialize_A(q1, q2, params):
        return (0.015 * sin(tp * q2), 0.025 * cos(tp * q1), 0.03 * cos(tp * (q1 + 2 * q2)))

    def initialize_A3_B3(q1, q2, params):
        return (0.03 * sin(tp * (q1 + 2 * q2)), 0.4 + 0.01 * cos(tp * q1))

    table = {'E_B': (initialize_E, initialize_B),
             'Aphi_A': (initialize_A_phi, initialize_A),
             'E_A3B3': (initialize_E, initialize_A3_B3),
             'B': (initialize_B,)}
    return {fn.__name__: fn for fn in table[form]}


# ---------------------------------------------------------------------------
def _noise(spec, Nq1g, Nq2g):
    ini = spec['init']
    Ng = spec['N_ghost']
    if not ini.get('noise'):
        return np.zeros((Nq2g, Nq1g))
    rng = np.random.default_rng(ini.get('seed', 0))
    xi = rng.standard_normal((spec['N_q2'], spec['N_q1']))
    j = (np.arange(Nq2g) - Ng) % spec['N_q2']
    i = (np.arange(Nq1g) - Ng) % spec['N_q1']
    return xi[j][:, i]


def density_q(spec, q1, q2, noise_grid, ini=None):
    ini = spec['init'] if ini is None else ini
    n = ini.get('base', 1.0) * (1 + ini.get('amp', 0.0)
                                * np.cos(2 * np.pi * ini.get('k1', 1) * q1)
                                * np.cos(2 * np.pi * ini.get('k2', 0) * q2))
    return n * (1 + ini.get('noise', 0.0) * noise_grid)


def maxwellian_p(spec, s, p1, p2, p3, ini=None):
    """Velocity factor of species s (array over p)."""
    ini = spec['init'] if ini is None else ini
    m = spec['mass'][s]
    k = spec['boltzmann_constant']
    T = ini.get('T', [1.0, 1.0, 1.0])
    u = ini.get('u', [0.0, 0.0, 0.0])
    out = 1.0
    for d, p in enumerate((p1, p2, p3)[:spec['p_dim']]):
        out = out * np.sqrt(m / (2 * np.pi * k * T[d])) * np.exp(-m * (p - u[d]) ** 2 / (2 * k * T[d]))
    return out


def _grids(spec):
    Ng = spec['N_ghost']
    Nq1g, Nq2g = spec['N_q1'] + 2 * Ng, spec['N_q2'] + 2 * Ng
    dq1 = (spec['q1_end'] - spec['q1_start']) / spec['N_q1']
    dq2 = (spec['q2_end'] - spec['q2_start']) / spec['N_q2']
    q1 = spec['q1_start'] + (np.arange(-Ng, spec['N_q1'] + Ng) + 0.5) * dq1
    q2 = spec['q2_start'] + (np.arange(-Ng, spec['N_q2'] + Ng) + 0.5) * dq2
    return Nq1g, Nq2g, q1[None, :], q2[:, None]


def _pgrid(spec, s):
    out = []
    for d in (1, 2, 3):
        N = spec['N_p%d' % d]
        a, b = spec['p%d_start' % d][s], spec['p%d_end' % d][s]
        out.append(a + (0.5 + np.arange(N)) * ((b - a) / N))
    p1, p2, p3 = out
    return p1[None, None, :], p2[None, :, None], p3[:, None, None]


def initial_f(spec, ini=None):
    """f0 in the (Nq2g, Nq1g, Ns, Np3, Np2, Np1) layout, FP64."""
    Nq1g, Nq2g, q1, q2 = _grids(spec)
    ns = len(spec['mass'])
    noise = _noise(spec, Nq1g, Nq2g)
    n = density_q(spec, q1, q2, noise, ini)
    f = np.empty((Nq2g, Nq1g, ns, spec['N_p3'], spec['N_p2'], spec['N_p1']))
    for s in range(ns):
        p1, p2, p3 = _pgrid(spec, s)
        f[:, :, s] = n[:, :, None, None, None] * maxwellian_p(spec, s, p1, p2, p3, ini)[None, None]
    return f


def dirichlet_values(spec):
    """Boundary functions f_left/right/bottom/top as full f-shaped arrays."""
    out = {}
    for side, ini in spec.get('dirichlet', {}).items():
        d = dict(base=1.0, amp=0.0, k1=1, k2=0, noise=0.0)
        d.update(ini)
        out[side] = initial_f(spec, d)
    return out


def tau_value(spec):
    return spec['tau']
