"""CUDA path vs the golden fixtures of the reference run (and the oracle).

The GPU is driven from the fixture's exact initial state (f after the halo
refresh, and the initial fields), because df/dt of data with 1e-3 noise is
ill-conditioned: WENO5's smoothness indicators cancel catastrophically, so a
one-ulp difference in f0 (torch vs numpy exp) moves df/dt by ~1e-10.  The
solver's own initialisation is checked separately against the fixture.

Tolerances (normwise relative):
  FP64: df/dt, f after the case's steps, moments: 1e-12; fields 1e-10.
  FP32 (f and stencils FP32, moments/Maxwellian FP64): df/dt 1e-3 (flux
  differences cancel, amplifying FP32 rounding by ~1/(k dq)), f after the
  steps 2e-6, moments 2e-6, initial fields 1e-3 (the FFT solve is driven by
  density noise of 1e-3..1e-2, or by the near-cancelling charge densities of
  two species, which FP32 storage of f resolves to ~1e-4..5e-4)."""

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout, moments_layout
from _util import load_golden, rel, interior, moment_errors, check_compact

pytestmark = pytest.mark.gpu

MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')
NAMES = C.FVM_NAMES
TOL = {'fp64': dict(f0=1e-14, fields0=1e-11, dfdt=1e-12, f=1e-12, mom=1e-12, fields=1e-10),
       'fp32': dict(f0=1e-7, fields0=1e-3, dfdt=1e-3, f=2e-6, mom=2e-6, fields=1e-4),
       # FP64 throughput form: the paired kernel with FMA contraction and
       # Newton-refined reciprocals (df/dt alone keeps the reference order)
       'fp64-fast': dict(f0=1e-14, fields0=1e-11, dfdt=1e-12, f=1e-10, mom=1e-10,
                         fields=1e-10)}


def af_from_layout(a):
    """numpy (q2, q1, s, p3, p2, p1) -> torch AF-ordered (Np, Ns, Nq1g, Nq2g)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    t = t.reshape(t.shape[0], t.shape[1], t.shape[2], -1)
    return t.permute(3, 2, 1, 0)


def fields_af(a):
    """(6, Nq2g, Nq1g) -> (6, 1, Nq1g, Nq2g)."""
    return torch.from_numpy(np.ascontiguousarray(a)).permute(0, 2, 1).unsqueeze(1)


def cell_of(nls):
    return nls.fields_solver.cell_centered_EM_fields[:, 0].permute(0, 2, 1).cpu().numpy()


def yee_of(nls):
    return nls.fields_solver.yee_grid_EM_fields[:, 0].permute(0, 2, 1).cpu().numpy()


def _check_case(name, precision):
    tol = TOL[precision]
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    # the solver's own initialisation
    assert rel(interior(to_layout(nls.f, spec), g), G['f0']) < tol['f0']
    if spec['fields_enabled']:
        assert rel(cell_of(nls), G['fields_cell0']) < tol['fields0']
        assert rel(yee_of(nls), G['fields_yee0']) < tol['fields0']
    # drive from the fixture's state
    nls.f = af_from_layout(G['f0_refreshed']).to('cuda')
    if spec['fields_enabled']:
        nls.fields_solver.cell_centered_EM_fields = fields_af(G['fields_cell0'])
        nls.fields_solver.yee_grid_EM_fields = fields_af(G['fields_yee0'])
    nls.dt = spec['dt']
    d = to_layout(nls.df_dt(), spec)
    if spec['fields_enabled']:
        nls.fields_solver.at_n = True
    e = rel(interior(d, g), G['dfdt0'])
    assert e < tol['dfdt'], ('dfdt', e)
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    torch.cuda.synchronize()
    e = rel(interior(to_layout(nls.f, spec), g), G['f_final'])
    assert e < tol['f'], ('f', e)
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    errs = moment_errors(m, {k: G['mom_' + k] for k in MOMENTS})
    assert max(errs.values()) < tol['mom'], errs
    if spec['fields_enabled']:
        e = rel(cell_of(nls), G['fields_cell'])
        assert e < tol['fields'], ('fields', e)
    assert abs(nls.time_elapsed - float(G['time_elapsed'])) < 1e-12
    nls.synchronize()


@pytest.mark.parametrize('name', NAMES)
def test_fp64_matches_reference(name):
    _check_case(name, 'fp64')


@pytest.mark.parametrize('name', ['c1_1d1v_weno5_rk2', 'c1_1d1v_weno5_rk4_llf',
                                  'c3_2d3v_weno5_rk4_small', 'c2_2d2v_fdtd_rk4_small',
                                  'minmod_2d2v_fields_bgk', 'ppm_2d2v_fields_bgk',
                                  'dirichlet_1d1v_weno5', 'two_species_2d2v_fields',
                                  'mirror_2d2v_weno5', 'mirror_dirichlet_2d3v_rk4',
                                  'dirichlet_2d2v_minmod', 'pc_2d3v_fields',
                                  'es_1d1v_landau_rk2', 'es_2d2v_two_species_rk4',
                                  'fields_user_Aphi_A', 'fields_fft_user_B',
                                  'c3_2d3v_weno5_rk4_ghost4'])
def test_fp32_close_to_reference(name):
    _check_case(name, 'fp32')


@pytest.mark.parametrize('name', ['c3_2d3v_weno5_rk4_small', 'c3_2d3v_weno5_rk4_ghost4',
                                  'mirror_dirichlet_2d3v_rk4'])
def test_fp64_fast_close_to_reference(name):
    """The FP64 throughput form (paired kernel, FMA, Newton reciprocals) on
    the reference fixtures whose grids it takes: f and moments to 1e-10."""
    _check_case(name, 'fp64-fast')


def test_evolve_electrodynamic_fields_matches_oracle():
    """fields_solver.evolve_electrodynamic_fields with the caller's currents
    (per species, summed as af.sum(J, 1)) against the oracle's restatement of
    fields.py:568-647, three updates from the fixture's fields; compute_divE
    against its definition (fields.py:35-46)."""
    from oracle.bolt_oracle import Oracle, _periodic_fill, _sh
    name = 'fields_user_E_B'
    spec = C.CASES[name]
    G = load_golden(name)
    nls = make_solver(spec, 'fp64')
    o = Oracle(spec, C.initial_f(spec),
               field_functions=C.field_functions(spec['field_init'], np.sin, np.cos))
    nls.fields_solver.cell_centered_EM_fields = fields_af(G['fields_cell0'])
    nls.fields_solver.yee_grid_EM_fields = fields_af(G['fields_yee0'])
    o.fields.cell, o.fields.yee = G['fields_cell0'].copy(), G['fields_yee0'].copy()
    rng = np.random.default_rng(5)
    shape = o.fields.yee.shape[1:]                              # (Nq2g, Nq1g)
    for _ in range(3):
        J = rng.standard_normal((3, 2) + shape) * 0.1          # 2 per-species parts
        Jaf = [torch.from_numpy(np.ascontiguousarray(J[c].transpose(0, 2, 1)))[None]
               for c in range(3)]                               # (1, 2, Nq1g, Nq2g)
        nls.fields_solver.evolve_electrodynamic_fields(*Jaf, 2e-3)
        o.fields.evolve(J[0].sum(0), J[1].sum(0), J[2].sum(0), 2e-3)
    assert rel(yee_of(nls), o.fields.yee) < 1e-13
    assert rel(cell_of(nls), o.fields.cell) < 1e-13
    assert nls.fields_solver.time_elapsed == pytest.approx(6e-3)
    y = _periodic_fill(o.g, o.fields.yee)
    divE = (_sh(y[0], -1, 0) - y[0]) / o.g.dq1 + (_sh(y[1], 0, -1) - y[1]) / o.g.dq2
    got = nls.fields_solver.compute_divE()[0, 0].T.cpu().numpy()
    assert rel(got, divE) < 1e-12


PARTIAL = C.make(N_q1=12, N_q2=10, N_p1=8, N_p2=6, N_p3=4,
                 p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                 p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                 tau=0.05, dt=1e-3, steps=3, integrator='RK4',
                 riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                 init=dict(amp=0.1, k1=1, k2=1, u=[0.2, -0.1, 0.05]))


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-12), ('fp32', 2e-6)])
def test_partial_tiles_and_chunks_vs_oracle(precision, tol):
    """q-extents that are not multiples of the 8x8 tile and Np = 192 (six
    full chunks of 32 for the FP32 paired kernel's fast path, partial tiles
    at the right/top edges): CUDA vs the oracle from the same initial f."""
    from oracle.bolt_oracle import Oracle
    spec = PARTIAL
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    f0 = to_layout(nls.f, spec)          # the state actually on the GPU
    o = Oracle(spec, f0)
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
        o.step(spec['dt'])
    e = rel(interior(to_layout(nls.f, spec), g), interior(o.f, g))
    assert e < tol, e


# Several 8x8 q-tiles, N_p1 a multiple of 8 and N_p = 256 (eight chunks of 32):
# these run the FP32 paired kernel (TMA halo/base loads and out1/out2 stores,
# FP32 exp tables, grouped FP64 moments); the FP64 runs take the scalar kernel.
PAIR_CASES = {
    'pair_periodic_two_species': C.make(
        N_q1=24, N_q2=16, N_p1=8, N_p2=8, N_p3=4,
        p1_start=[-5.0, -3.0], p1_end=[5.0, 3.0], p2_start=[-5.0, -3.0], p2_end=[5.0, 3.0],
        p3_start=[-5.0, -3.0], p3_end=[5.0, 3.0], mass=[1.0, 4.0], charge=[0.0, 0.0],
        p_dim=3, tau=0.004, dt=1e-3, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.1, k1=1, k2=2, u=[0.2, -0.1, 0.05], T=[1.0, 1.5, 0.8])),
    'pair_dirichlet_rk2': C.make(
        N_q1=16, N_q2=16, N_p1=16, N_p2=4, N_p3=4,
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
        bc_q1='dirichlet', bc_q2='dirichlet', tau=0.05, dt=1e-3, steps=3,
        dirichlet=dict(left=dict(base=1.2, T=[1.0, 1.0, 1.0], u=[0.3, 0.1, 0]),
                       right=dict(base=0.8, T=[1.0, 1.0, 1.0], u=[-0.3, 0, 0]),
                       bottom=dict(base=1.1, T=[1.0, 1.0, 1.0], u=[0.0, 0.4, 0]),
                       top=dict(base=0.9, T=[1.0, 1.0, 1.0], u=[0.0, -0.4, 0])),
        init=dict(amp=0.1, k1=1, k2=1)),
    'pair_minmod_rk4': C.make(
        N_q1=24, N_q2=16, N_p1=8, N_p2=8, N_p3=4, recon_q='minmod', recon_p='minmod',
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
        tau=0.02, dt=1e-3, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.1, k1=1, k2=2, u=[0.3, -0.2, 0.05], T=[1.0, 1.4, 0.8])),
    'pair_ppm_rk2': C.make(
        N_q1=16, N_q2=24, N_p1=8, N_p2=4, N_p3=4, recon_q='ppm', recon_p='ppm',
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
        tau=0.03, dt=1e-3, steps=3, integrator='RK2',
        init=dict(amp=0.1, k1=2, k2=1, u=[-0.3, 0.2, 0.1])),
    'pair_mirror_rk4': C.make(
        N_q1=16, N_q2=24, N_p1=8, N_p2=4, N_p3=4,
        p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
        p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
        bc_q1='mirror', bc_q2='mirror', tau=0.02, dt=1e-3, steps=3, integrator='RK4',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
        init=dict(amp=0.1, k1=1, k2=1, u=[0.5, -0.4, 0.1], T=[1.0, 1.3, 0.9])),
}


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-12), ('fp32', 2e-6), ('fp64-fast', 1e-12)])
@pytest.mark.parametrize('name', sorted(PAIR_CASES))
def test_paired_kernel_cases_vs_oracle(name, precision, tol):
    """Multi-tile grids that meet the paired kernel's shape conditions, periodic
    (two species, RK4) and Dirichlet (RK2): f and the five moments after three
    steps vs the oracle started from the state on the GPU.  The periodic case
    relaxes stiffly (dt/tau = 0.25, anisotropic temperature), so errors in the
    stage moments that feed the Maxwellian reach f almost undamped."""
    from oracle.bolt_oracle import Oracle
    spec = PAIR_CASES[name]
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    o = Oracle(spec, to_layout(nls.f, spec))
    if 'dirichlet' in spec:
        o.dirichlet = C.dirichlet_values(spec)
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
        o.step(spec['dt'])
    e = rel(interior(to_layout(nls.f, spec), g), interior(o.f, g))
    assert e < tol, e
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    ref = {k: interior(o.moments(k), g) for k in MOMENTS}
    errs = moment_errors(m, ref)
    assert max(errs.values()) < tol, errs


@pytest.mark.parametrize('recon', ['weno5', 'minmod', 'ppm', 'piecewise-constant'])
def test_paired_kernel_matches_scalar_kernel(monkeypatch, recon):
    """The paired FP32 kernel against the scalar FP32 kernel (BOLT_NO_PAIR) on
    a 32x32 x 24^3 Maxwellian with a density wave, two RK4 steps: same
    arithmetic type, different operation order, so they agree to a few FP32
    ulps."""
    spec = C.make(N_q1=32, N_q2=32, N_p1=24, N_p2=24, N_p3=24, recon_q=recon, recon_p=recon,
                  p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
                  p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=1e-3, steps=2, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.05, k1=1, k2=1, u=[0.1, -0.2, 0.05]))
    out = {}
    for mode in ('pair', 'scalar'):
        if mode == 'scalar':
            monkeypatch.setenv('BOLT_NO_PAIR', '1')
        nls = make_solver(spec, 'fp32')
        for _ in range(spec['steps']):
            nls.strang_timestep(spec['dt'])
        out[mode] = (to_layout(nls.f, spec),
                     {k: moments_layout(nls.compute_moments(k)) for k in MOMENTS})
        del nls
    g = spec['N_ghost']
    e = rel(interior(out['pair'][0], g), interior(out['scalar'][0], g))
    assert e < 1e-6, e
    errs = moment_errors({k: interior(v, g) for k, v in out['pair'][1].items()},
                         {k: interior(v, g) for k, v in out['scalar'][1].items()})
    assert max(errs.values()) < 1e-6, errs


# ---------------------------------------------------------------------------
# The headline velocity grid: 24^3 p-cells per q-cell (432 chunks of 32 p, so
# a chunk, and a p-split's first chunk, can start inside a p1 row)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize('precision', ['fp64', 'fp32', 'fp64-fast'])
def test_reference_at_headline_velocity_grid(precision):
    """8x8 q x 24^3 p, WENO5 + LLF, BGK, RK4, 3 steps, from the compact
    reference fixture: df/dt of the refreshed initial state and f after the
    steps, in full at the fixture's q-cells and as per-q-cell velocity sums
    everywhere, and the five moments.  FP32 steps run the paired kernel."""
    name = 'c3_2d3v_weno5_rk4_p24'
    spec = C.COMPACT_CASES[name]
    G = load_golden(name)
    tol = TOL[precision]
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    f0 = C.compact_f0(G)
    assert rel(interior(to_layout(nls.f, spec), g), interior(f0, g)) < tol['f0']
    nls.f = af_from_layout(C.periodic_wrap(f0, spec)).to('cuda')
    nls.dt = spec['dt']
    d = interior(to_layout(nls.df_dt(), spec), g)
    pair0 = nls.paired_launch_count()
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    torch.cuda.synchronize()
    if precision != 'fp64':
        assert nls.paired_launch_count() - pair0 == 4 * spec['steps']
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    check_compact(spec, G, interior(to_layout(nls.f, spec), g), m, dfdt0=d,
                  tol_f=tol['f'], tol_dfdt=tol['dfdt'], tol_mom=tol['mom'])
    assert abs(nls.time_elapsed - float(G['time_elapsed'])) < 1e-12
    nls.synchronize()


HEADLINE_P_MULTI = C.make(
    N_q1=16, N_q2=16, N_p1=24, N_p2=24, N_p3=24,
    p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
    p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
    tau=0.05, dt=1e-3, steps=2, integrator='RK4',
    riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
    init=dict(amp=0.05, k1=1, k2=1, noise=1e-3, seed=2, u=[0.1, -0.2, 0.05]))


@pytest.fixture(scope='module')
def headline_multi_ref():
    """The C restatement's two RK4 steps of HEADLINE_P_MULTI from the FP64
    solver's initial state (the restatement is pinned to the numpy oracle and
    the fixtures by tests/test_c_oracle.py)."""
    from oracle import c_oracle
    from oracle.bolt_oracle import Oracle
    spec = HEADLINE_P_MULTI
    f = np.ascontiguousarray(to_layout(make_solver(spec, 'fp64').f, spec))
    f0 = f.copy()
    for _ in range(spec['steps']):
        c_oracle.rk_step(f, spec, spec['dt'], integrator=4)
    o = Oracle(spec, f)
    g = spec['N_ghost']
    return f0, interior(f, g), {k: interior(o.moments(k), g) for k in MOMENTS}


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-12), ('fp32', 2e-6), ('fp64-fast', 1e-10)])
@pytest.mark.parametrize('cps', [None, 432, 54, 7, 5])
def test_headline_velocity_grid_multi_tile_vs_oracle(monkeypatch, headline_multi_ref, precision,
                                                     tol, cps):
    """16x16 q (four 8x8 tiles) x 24^3 p with density noise, two RK4 steps,
    under the automatic p-split and under fixed splits of 432 (one split), 54,
    7 and 5 chunks per CTA (a split's first p lies at p1 offset 0, 8 or 16 of
    a row): f and the moments against the C restatement from the same state."""
    spec = HEADLINE_P_MULTI
    if cps is not None:
        monkeypatch.setenv('BOLT_CHUNKS_PER_SPLIT', str(cps))
    f0, ref_f, ref_m = headline_multi_ref
    nls = make_solver(spec, precision)
    nsplit, got_cps = nls.split_info()
    if cps is not None:
        assert got_cps == cps and nsplit == -(-432 // cps)
    nls.f = af_from_layout(f0).to('cuda')
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    torch.cuda.synchronize()
    if precision != 'fp64':
        assert nls.paired_launch_count() == 4 * spec['steps']
    g = spec['N_ghost']
    e = rel(interior(to_layout(nls.f, spec), g), ref_f)
    assert e < tol, e
    m = {k: interior(moments_layout(nls.compute_moments(k)), g) for k in MOMENTS}
    errs = moment_errors(m, ref_m)
    assert max(errs.values()) < tol, errs
    nls.synchronize()


# ---------------------------------------------------------------------------
# df_dt_fvm's term_to_return (df_dt_fvm.py:325-339): one p-flux divergence
# ---------------------------------------------------------------------------
TERM_CASES = ['c2_2d2v_fdtd_rk2_small', 'es_2d2v_two_species_rk4', 'fields_user_E_B_2d3v',
              'pc_2d3v_fields', 'minmod_2d2v_fields_bgk', 'ppm_2d2v_fields_bgk']


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
@pytest.mark.parametrize('name', TERM_CASES)
def test_term_to_return_matches_reference(name, precision):
    """d_flux_p{1,2,3}_dp{1,2,3} of the fixture's refreshed initial state and
    fields against the reference's df_dt_fvm(..., term_to_return=...); a term
    the reference gives as exactly zero (a single-cell axis, or C_p3 = 0 with
    no E3 or B) must be exactly zero here too."""
    tol = TOL[precision]
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    nls = make_solver(spec, precision)
    nls.f = af_from_layout(G['f0_refreshed']).to('cuda')
    nls.fields_solver.cell_centered_EM_fields = fields_af(G['fields_cell0'])
    nls.fields_solver.yee_grid_EM_fields = fields_af(G['fields_yee0'])
    nls.dt = spec['dt']
    at_n = nls.fields_solver.at_n
    for k in (1, 2, 3):
        nls.fields_solver.at_n = at_n
        d = interior(to_layout(nls.df_dt(term_to_return='d_flux_p%d_dp%d' % (k, k)), spec), g)
        ref = G['dfdt0_p%d' % k]
        if not np.any(ref):
            assert not np.any(d), (k, float(np.abs(d).max()))
        else:
            e = rel(d, ref)
            assert e < tol['dfdt'], (k, e)
    nls.synchronize()


def test_term_to_return_needs_fields():
    spec = C.CASES['c3_2d3v_weno5_rk4_small']
    nls = make_solver(spec, 'fp64')
    with pytest.raises(ValueError):
        nls.df_dt(term_to_return='d_flux_p1_dp1')
    # any other value returns the whole df/dt, as in the reference
    G = load_golden('c3_2d3v_weno5_rk4_small')
    nls.f = af_from_layout(G['f0_refreshed']).to('cuda')
    d = to_layout(nls.df_dt(term_to_return='all'), spec)
    g = spec['N_ghost']
    assert rel(interior(d, g), G['dfdt0']) < 1e-12


@pytest.mark.parametrize('recon', ['weno5', 'minmod', 'ppm', 'piecewise-constant'])
def test_fp64_fast_matches_reference_order_on_a_discontinuity(recon):
    """FP64 throughput form against the reference-order FP64 kernels on a
    32x32 x 24^3 Maxwellian whose density jumps by 2x across q1 = 1/2 and
    q2 = 1/2, two RK4 steps.  At the jumps the WENO5 substencils disagree at
    O(1), so the face values depend on the nonlinear weights at full weight:
    an inexact reciprocal in the weights would show here (on smooth data it
    is hidden by the small third differences).  Agreement to 1e-13 normwise
    holds the Newton-refined reciprocal to FP64 rounding."""
    spec = C.make(N_q1=32, N_q2=32, N_p1=24, N_p2=24, N_p3=24, recon_q=recon, recon_p=recon,
                  p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
                  p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=1e-3, steps=2, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.05, k1=1, k2=1, u=[0.1, -0.2, 0.05]))
    g = spec['N_ghost']
    out = {}
    for prec in ('fp64', 'fp64-fast'):
        nls = make_solver(spec, prec)
        f = nls.f.clone()                                    # (Np, Ns, Nq1g, Nq2g)
        f[:, :, g:g + 16, :] *= 2.0
        f[:, :, :, g:g + 16] *= 1.5
        nls.f = f
        for _ in range(spec['steps']):
            nls.strang_timestep(spec['dt'])
        torch.cuda.synchronize()
        if prec == 'fp64-fast':
            assert nls.paired_launch_count() == 4 * spec['steps']
        out[prec] = (to_layout(nls.f, spec),
                     {k: moments_layout(nls.compute_moments(k)) for k in MOMENTS})
        nls.synchronize()
        del nls
    e = rel(interior(out['fp64-fast'][0], g), interior(out['fp64'][0], g))
    assert e < 1e-13, e
    errs = moment_errors({k: interior(v, g) for k, v in out['fp64-fast'][1].items()},
                         {k: interior(v, g) for k, v in out['fp64'][1].items()})
    assert max(errs.values()) < 1e-13, errs


@pytest.mark.parametrize('name', ['c1_1d1v_weno5_rk2', 'c3_2d3v_weno5_rk4_small',
                                  'mirror_dirichlet_2d3v_rk4', 'dirichlet_1d1v_weno5',
                                  'pc_2d3v_fields', 'fields_user_E_B_2d3v',
                                  'minmod_2d2v_fields_bgk'])
def test_fp32_dfdt_arithmetic_error(name):
    """The FP32 df/dt against the FP64 df/dt of the same FP32-rounded state,
    so that only the FP32 arithmetic differs: 1e-5 normwise, plus the
    rounding of the BGK Maxwellian to FP32 amplified by 1/tau.  On a near-
    equilibrium f the term (f0 - f)/tau cancels to a small df/dt, and each
    rounded f0 carries up to 2^-24 |f0| of error, so the bound adds
    2 * 2^-24 ||f|| / (tau ||df/dt||) (3.9e-4 on the 1D1V case with
    tau = 0.01, where 1.5e-4 is seen; at most 2.2e-5 on the others).  The
    fixture comparison's 1e-3 bound also absorbs the rounding of the input
    itself, which the flux differences amplify on the noisy cases."""
    spec = C.CASES[name]
    G = load_golden(name)
    g = spec['N_ghost']
    f32 = G['f0_refreshed'].astype(np.float32).astype(np.float64)
    out = {}
    for prec in ('fp64', 'fp32'):
        nls = make_solver(spec, prec)
        nls.f = af_from_layout(f32).to('cuda')
        if spec['fields_enabled']:
            nls.fields_solver.cell_centered_EM_fields = fields_af(G['fields_cell0'])
            nls.fields_solver.yee_grid_EM_fields = fields_af(G['fields_yee0'])
        nls.dt = spec['dt']
        out[prec] = interior(to_layout(nls.df_dt(), spec), g)
        nls.synchronize()
    e = rel(out['fp32'], out['fp64'])
    tol = 1e-5 + 2 * 2.0 ** -24 * np.linalg.norm(interior(f32, g)) / (
        spec['tau'] * np.linalg.norm(out['fp64']))
    assert e < tol, (e, tol)
