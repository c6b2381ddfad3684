"""Generate golden fixtures by running the UNMODIFIED Bolt reference source.

Usage (where a read-only copy of the reference project is present):
    python tests/golden/make_golden.py /path/to/reference [case ...]
    BOLT_REFERENCE_DIR=/path/to/reference python tests/golden/make_golden.py [case ...]

The reference's runtime stack (arrayfire, petsc4py, mpi4py, prettytable) is not
installable offline, so single-process numpy stand-ins from tests/golden/refshim
are put first on sys.path.  Three gaps in the reference are restated here as
thin wrappers, exactly as the oracle restates them:
  * WENO5 is refused by a guard in reconstruct.py:39-41; the wrapper calls the
    reference's own reconstruct_weno5 (weno5.py:4) for 'weno5'.
  * Only an RK2 stepper exists for the FVM (fvm_operator.py:6-35); for
    integrator 'RK4' the wrapper composes the reference's df_dt_fvm with the
    stages of integrators.py:15-28 and the halo/BC refresh of
    fvm_operator.py before each stage.  With electrodynamic fields it sets the
    fields solver's time-level flag so the fields advance once per step, in
    stage 2.
  * riemann_solver_in_q/p are ignored by the reference (riemann.py:46-49 is
    always upwind); LLF cases therefore run the upwind flux here, which is the
    same mathematical flux (the oracle evaluates the LLF formula).

Writes tests/golden/<case>.npz with arrays in the (q2, q1, s, p3, p2, p1)
layout; f0, dfdt0 (and, with fields, dfdt0_p1..p3: the term_to_return
p-flux divergences), f_final and the moments hold interior cells only,
f0_refreshed (the initial state after the halo/BC refresh) and the field arrays
hold ghost cells too.  Only this script reads the reference; the fixtures travel.
"""

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'refshim'))
sys.path.insert(0, HERE)

import cases as C  # noqa: E402


def af_to_layout(a, spec):
    """Reference logical (Np, Ns, Nq1g, Nq2g) -> (Nq2g, Nq1g, Ns, Np3, Np2, Np1)."""
    arr = np.asarray(a)
    arr = arr.reshape(arr.shape + (1,) * (4 - arr.ndim))
    t = np.transpose(arr, (3, 2, 1, 0))
    return t.reshape(t.shape[:3] + (spec['N_p3'], spec['N_p2'], spec['N_p1'])).copy()


def q_to_layout(a):
    """(1, Ns, Nq1g, Nq2g) moment -> (Nq2g, Nq1g, Ns)."""
    arr = np.asarray(a)
    arr = arr.reshape(arr.shape + (1,) * (4 - arr.ndim))
    return np.transpose(arr[0], (2, 1, 0)).copy()


def build_modules(spec, af, record=None):
    """Config modules of a case; with a dict `record`, initialize_f also leaves
    its q-factor n and p-factor out there (f0 = n * out, one multiplication
    per cell)."""
    dom = types.ModuleType('domain')
    for k in ('q1_start', 'q1_end', 'q2_start', 'q2_end', 'N_q1', 'N_q2',
              'N_p1', 'N_p2', 'N_p3', 'N_ghost'):
        setattr(dom, k, spec[k])
    for k in ('p1_start', 'p1_end', 'p2_start', 'p2_end', 'p3_start', 'p3_end'):
        setattr(dom, k, list(spec[k]))

    Nq1g = spec['N_q1'] + 2 * spec['N_ghost']
    Nq2g = spec['N_q2'] + 2 * spec['N_ghost']
    noise = C._noise(spec, Nq1g, Nq2g)            # (Nq2g, Nq1g)
    noise_af = af.Array._wrap(noise.T[None, None])  # (1, 1, Nq1g, Nq2g)

    def make_f(ini, record=None):
        def fn(q1, q2, p1, p2, p3, params):
            m = params.mass
            k = params.boltzmann_constant
            n = ini.get('base', 1.0) * (1 + ini.get('amp', 0.0)
                                        * af.cos(2 * np.pi * ini.get('k1', 1) * q1)
                                        * af.cos(2 * np.pi * ini.get('k2', 0) * q2))
            n = n * (1 + ini.get('noise', 0.0) * noise_af)
            T = ini.get('T', [1.0, 1.0, 1.0])
            u = ini.get('u', [0.0, 0.0, 0.0])
            out = 1.0
            for d, p in enumerate((p1, p2, p3)[:params.p_dim]):
                out = out * af.sqrt(m / (2 * np.pi * k * T[d])) \
                    * af.exp(-m * (p - u[d]) ** 2 / (2 * k * T[d]))
            if record is not None:
                record['n'], record['out'] = n, out
            return n * out
        return fn

    init_defaults = dict(base=1.0, amp=0.0, k1=1, k2=0, noise=0.0)
    ini = dict(init_defaults)
    ini.update(spec['init'])
    initialize = types.ModuleType('initialize')
    initialize.initialize_f = make_f(ini, record)
    if spec.get('field_init'):
        for k, fn in C.field_functions(spec['field_init'], af.sin, af.cos).items():
            setattr(initialize, k, fn)

    bc = types.ModuleType('boundary_conditions')
    bc.in_q1_left = bc.in_q1_right = spec['bc_q1']
    bc.in_q2_bottom = bc.in_q2_top = spec['bc_q2']
    for side, dini in spec.get('dirichlet', {}).items():
        d = dict(init_defaults)
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
    params.time_integrator = spec['integrator']
    tau = spec['tau']

    def tau_fn(q1, q2, p1, p2, p3):
        return tau * p1 ** 0 * q1 ** 0
    params.tau = tau_fn
    return dom, bc, params, initialize


def patch_reference():
    import arrayfire as af
    from bolt.lib.nonlinear.finite_volume import df_dt_fvm as dmod
    from bolt.lib.nonlinear.finite_volume import fvm_operator as fmod
    from bolt.lib.nonlinear.finite_volume.reconstruction.minmod import reconstruct_minmod
    from bolt.lib.nonlinear.finite_volume.reconstruction.ppm import reconstruct_ppm
    from bolt.lib.nonlinear.finite_volume.reconstruction.weno5 import reconstruct_weno5

    def reconstruct(self, input_array, axis, method):
        if method == 'piecewise-constant':
            return input_array, input_array
        if method == 'minmod':
            return reconstruct_minmod(input_array, axis)
        if method == 'ppm':
            return reconstruct_ppm(input_array, axis)
        if method == 'weno5':
            return reconstruct_weno5(input_array, axis)
        raise NotImplementedError(method)
    dmod.reconstruct = reconstruct

    rk2 = fmod.timestep_fvm
    df_dt_fvm = dmod.df_dt_fvm

    def timestep(self, dt):
        if getattr(self.physical_system.params, 'time_integrator', 'RK2') != 'RK4':
            return rk2(self, dt)
        fs = getattr(self, 'fields_solver', None)
        fe = self.physical_system.params.fields_enabled and \
            self.physical_system.params.fields_type == 'electrodynamic'

        def stage(x, evolve):
            self.f = x
            self._communicate_f()
            self._apply_bcs_f()
            if fe:
                fs.at_n = not evolve
            return self.f, df_dt_fvm(self.f, self)

        f_initial, k1 = stage(self.f, False)
        _, k2 = stage(f_initial + 0.5 * k1 * dt, True)
        _, k3 = stage(f_initial + 0.5 * k2 * dt, False)
        _, k4 = stage(f_initial + k3 * dt, False)
        self.f = f_initial + ((k1 + 2 * k2 + 2 * k3 + k4) / 6) * dt
        af.eval(self.f)
    fmod.timestep_fvm = timestep
    return df_dt_fvm


def run_case(name, spec):
    import arrayfire as af
    from bolt.lib.physical_system import physical_system
    from bolt.lib.nonlinear.nonlinear_solver import nonlinear_solver
    import bolt.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt.src.nonrelativistic_boltzmann.moments as mom

    df_dt_fvm = patch_reference()
    # the constructor's device-bandwidth probe (bandwidth_test.py:13-34) only
    # prints a number; skip its 100 x 268 MB numpy additions
    import bolt.lib.nonlinear.nonlinear_solver as nsmod
    nsmod.bandwidth_test = lambda n_evals: 0.0
    record = {}
    dom, bc, params, initialize = build_modules(spec, af, record)
    system = physical_system(dom, bc, params, initialize, adv, col.BGK, mom)
    nls = nonlinear_solver(system)
    out = {}
    out['f0'] = interior(af_to_layout(nls.f, spec), spec)
    if spec.get('compact'):
        out['n_q'], out['v_p'] = init_factors(record, spec, out['f0'])
    # df/dt of the halo-refreshed initial state (fields at their initial level)
    f_save = nls.f
    nls._communicate_f()
    nls._apply_bcs_f()
    out['f0_refreshed'] = af_to_layout(nls.f, spec)
    nls.dt = spec['dt']
    if spec['fields_enabled']:
        at_n = nls.fields_solver.at_n
    if spec.get('solver_q', 'FVM') == 'FVM':
        out['dfdt0'] = interior(af_to_layout(df_dt_fvm(nls.f, nls), spec), spec)
    if spec['fields_enabled']:
        # the single p-flux divergences of the same state (term_to_return,
        # df_dt_fvm.py:325-335), each from the same field time level
        for k in (1, 2, 3):
            nls.fields_solver.at_n = at_n
            term = df_dt_fvm(nls.f, nls, term_to_return='d_flux_p%d_dp%d' % (k, k))
            out['dfdt0_p%d' % k] = interior(af_to_layout(term, spec), spec)
        nls.fields_solver.at_n = at_n
        out['fields_cell0'] = np.transpose(np.asarray(nls.fields_solver.cell_centered_EM_fields)
                                           .reshape(6, 1, Nq(spec, 1), Nq(spec, 2))[:, 0], (0, 2, 1))
        out['fields_yee0'] = np.transpose(np.asarray(nls.fields_solver.yee_grid_EM_fields)
                                          .reshape(6, 1, Nq(spec, 1), Nq(spec, 2))[:, 0], (0, 2, 1))
    nls.f = f_save
    # the splitting scheme (all four are the same step for FVM in q and p)
    step = getattr(nls, spec.get('splitting', 'strang') + '_timestep')
    for _ in range(spec['steps']):
        step(spec['dt'])
    out['f_final'] = interior(af_to_layout(nls.f, spec), spec)
    for mname in ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy'):
        out['mom_' + mname] = interior(q_to_layout(nls.compute_moments(mname)), spec)
    if spec['fields_enabled']:
        out['fields_cell'] = np.transpose(np.asarray(nls.fields_solver.cell_centered_EM_fields)
                                          .reshape(6, 1, Nq(spec, 1), Nq(spec, 2))[:, 0], (0, 2, 1))
        out['fields_yee'] = np.transpose(np.asarray(nls.fields_solver.yee_grid_EM_fields)
                                         .reshape(6, 1, Nq(spec, 1), Nq(spec, 2))[:, 0], (0, 2, 1))
    out['time_elapsed'] = np.array(nls.time_elapsed)
    return compact(out, spec) if spec.get('compact') else out


def init_factors(record, spec, f0):
    """initialize_f's factors in the fixture layout: n_q (Nq2g, Nq1g) and v_p
    (Np3, Np2, Np1), checked to rebuild the reference's f0 bit for bit."""
    n = np.asarray(record['n'])
    n = n.reshape(n.shape + (1,) * (4 - n.ndim))[0, 0].T.copy()
    v = np.asarray(record['out']).reshape(spec['N_p3'], spec['N_p2'], spec['N_p1']).copy()
    assert np.array_equal(interior(C.compact_f0({'n_q': n, 'v_p': v}), spec), f0)
    return n, v


def compact(out, spec):
    """A compact fixture for a case whose f is too large to store: the factors
    of f0, the halo-refreshed f0 checked to be its periodic wrap, df/dt and
    f_final in full at the q-cells C.COMPACT_SEL and as per-q-cell velocity
    sums (C.qcell_sums) everywhere, and the moments."""
    full = C.compact_f0(out)
    assert np.array_equal(out.pop('f0_refreshed'), C.periodic_wrap(full, spec))
    out.pop('f0')
    sel = np.array(C.COMPACT_SEL)
    for k in ('dfdt0', 'f_final'):
        a = out.pop(k)
        out[k + '_sel'] = a[sel[:, 0], sel[:, 1]].copy()
        out[k + '_qsum'] = C.qcell_sums(spec, a)
    return out


def interior(a, spec):
    g = spec['N_ghost']
    return a[g:a.shape[0] - g, g:a.shape[1] - g].copy()


def Nq(spec, d):
    return spec['N_q%d' % d] + 2 * spec['N_ghost']


def reference_dir(argv):
    """The reference project's root: the first argument that is a directory,
    else $BOLT_REFERENCE_DIR; the remaining arguments are case names."""
    ref = os.environ.get('BOLT_REFERENCE_DIR')
    names = []
    for a in argv:
        if os.path.isdir(a):
            ref = a
        else:
            names.append(a)
    if not ref or not os.path.isdir(os.path.join(ref, 'bolt')):
        raise SystemExit('give the reference project root (containing bolt/) as an argument '
                         'or in BOLT_REFERENCE_DIR')
    return ref, names


def main(argv):
    ref, names = reference_dir(argv)
    sys.path.insert(1, ref)
    names = names or sorted(C.CASES) + sorted(C.COMPACT_CASES)
    for name in names:
        spec = C.CASES[name] if name in C.CASES else C.COMPACT_CASES[name]
        out = run_case(name, spec)
        np.savez_compressed(os.path.join(HERE, name + '.npz'), **out)
        print('wrote', name, {k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    main(sys.argv[1:])
