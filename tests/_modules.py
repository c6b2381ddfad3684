"""Config modules (domain, boundary_conditions, params, initialize) for the
bolt_b200 API, built from a case spec of tests/golden/cases.py.  The user
callbacks are written against torch, the way a Bolt user's ArrayFire
callbacks would be ported."""

import math
import types

import numpy as np
import torch

import cases as C


def build_modules(spec, precision='fp64', integrator=None):
    dom = types.ModuleType('domain')
    for k in ('q1_start', 'q1_end', 'q2_start', 'q2_end', 'N_q1', 'N_q2',
              'N_p1', 'N_p2', 'N_p3', 'N_ghost'):
        setattr(dom, k, spec[k])
    for k in ('p1_start', 'p1_end', 'p2_start', 'p2_end', 'p3_start', 'p3_end'):
        setattr(dom, k, list(spec[k]))
    Nq1g = spec['N_q1'] + 2 * spec['N_ghost']
    Nq2g = spec['N_q2'] + 2 * spec['N_ghost']
    noise = torch.from_numpy(C._noise(spec, Nq1g, Nq2g).T.copy()).reshape(1, 1, Nq1g, Nq2g)

    def make_f(ini):
        def fn(q1, q2, p1, p2, p3, params):
            m = params.mass
            k = params.boltzmann_constant
            n = ini.get('base', 1.0) * (1 + ini.get('amp', 0.0)
                                        * torch.cos(2 * np.pi * ini.get('k1', 1) * q1)
                                        * torch.cos(2 * np.pi * ini.get('k2', 0) * q2))
            if ini.get('noise', 0.0):
                n = n * (1 + ini['noise'] * noise.to(q1.device))
            T = ini.get('T', [1.0, 1.0, 1.0])
            u = ini.get('u', [0.0, 0.0, 0.0])
            out = 1.0
            for d, p in enumerate((p1, p2, p3)[:params.p_dim]):
                out = out * torch.sqrt(m / (2 * np.pi * k * T[d])) \
                    * torch.exp(-m * (p - u[d]) ** 2 / (2 * k * T[d]))
            return n * out
        return fn

    defaults = dict(base=1.0, amp=0.0, k1=1, k2=0, noise=0.0)
    ini = dict(defaults)
    ini.update(spec['init'])
    initialize = types.ModuleType('initialize')
    initialize.initialize_f = make_f(ini)
    if spec.get('field_init'):
        for k, fn in C.field_functions(spec['field_init'], torch.sin, torch.cos).items():
            setattr(initialize, k, fn)

    bc = types.ModuleType('boundary_conditions')
    bc.in_q1_left = bc.in_q1_right = spec['bc_q1']
    bc.in_q2_bottom = bc.in_q2_top = spec['bc_q2']
    for side, dini in spec.get('dirichlet', {}).items():
        d = dict(defaults)
        d.update(dini)
        fn = make_f(d)

        def fb(f, t, q1, q2, p1, p2, p3, params, fn=fn):
            return fn(q1, q2, p1, p2, p3, params)
        setattr(bc, 'f_' + side, fb)

    params = types.ModuleType('params')
    params.fields_type = spec['fields_type']
    params.fields_initialize = spec['fields_initialize']
    params.fields_solver = spec['fields_solver']
    params.solver_method_in_q = spec.get('solver_q', 'FVM')
    params.solver_method_in_p = 'FVM'
    params.reconstruction_method_in_q = spec['recon_q']
    params.reconstruction_method_in_p = spec['recon_p']
    params.riemann_solver_in_q = spec['riemann_q']
    params.riemann_solver_in_p = spec['riemann_p']
    params.p_dim = spec['p_dim']
    params.num_devices = 1
    params.mass = list(spec['mass'])
    params.charge = list(spec['charge'])
    params.boltzmann_constant = spec['boltzmann_constant']
    params.fields_enabled = spec['fields_enabled']
    params.source_enabled = spec['source_enabled']
    params.instantaneous_collisions = bool(spec.get('instantaneous', False))
    params.hybrid_model_enabled = False
    params.eps = spec['eps']
    params.mu = spec['mu']
    params.p_space_grid = spec.get('p_space_grid', 'cartesian')
    params.initial_mu = spec.get('initial_mu', 1.0)
    params.time_integrator = integrator or spec['integrator']
    params.precision = precision
    # shearing-box rate q omega (boundaries.py:17-18)
    params.q = spec.get('shear_q', 0.0)
    params.omega = spec.get('shear_omega', 0.0)
    tau = spec['tau']

    def tau_fn(q1, q2, p1, p2, p3):
        return tau * p1 ** 0 * q1 ** 0
    params.tau = tau_fn
    return dom, bc, params, initialize


def make_solver(spec, precision='fp64', integrator=None):
    from bolt_b200.physical_system import physical_system
    from bolt_b200.nonlinear_solver import nonlinear_solver
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    dom, bc, params, initialize = build_modules(spec, precision, integrator)
    system = physical_system(dom, bc, params, initialize, adv, col.BGK, mom)
    return nonlinear_solver(system)


def to_layout(af_tensor, spec):
    """AF-ordered (Np, Ns, Nq1g, Nq2g) tensor -> numpy (q2, q1, s, p3, p2, p1)."""
    a = af_tensor.detach().to(torch.float64).cpu().permute(3, 2, 1, 0).contiguous().numpy()
    return a.reshape(a.shape[:3] + (spec['N_p3'], spec['N_p2'], spec['N_p1']))


def moments_layout(m):
    """(1, Ns, Nq1g, Nq2g) -> (Nq2g, Nq1g, Ns)."""
    return m[0].detach().cpu().permute(2, 1, 0).numpy()
