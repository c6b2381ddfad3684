"""Failure detection on the GPU without a GPU fault.

* Divergence (timestep.py:28-38): a NaN written into f from the host makes the
  next step's kernels flag a non-finite value; strang_timestep raises
  SystemExit('Solver Diverging!') at the first step boundary after those
  kernels finished (the flag is read from pinned host memory without
  synchronising).  Through the C ABI the same flag is bolt_divergence_flag.
* Timeouts: with the test hook bolt_test_stall_waits the stage kernels issue
  no tile copies, so every CTA's first bounded wait runs out after a short
  budget with nothing in flight; the CTAs record BOLT_ERR_TIMEOUT and return.
  check_divergence then raises a BoltError with that code, bolt_status_sync
  returns it, and the context stays usable once the hook is off.
No test here traps, hangs or faults the GPU: every wait is bounded and the
only thing injected is data (a NaN) or a copy that is never issued."""

import ctypes

import numpy as np
import pytest
import torch

import cases as C
import bolt_b200._native as N
from _modules import make_solver, to_layout
from _util import rel, interior

pytestmark = pytest.mark.gpu

SPEC = C.make(N_q1=16, N_q2=16, N_p1=8, N_p2=8, N_p3=4,
              p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
              p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
              tau=0.05, dt=1e-3, steps=2, integrator='RK4',
              riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
              init=dict(amp=0.1, k1=1, k2=1, u=[0.2, -0.1, 0.05]))


def _poison(nls):
    """A NaN in one interior cell of f, written from the host."""
    f = nls.f.clone()
    g = nls.N_ghost
    f[5, 0, g + 3, g + 4] = float('nan')
    nls.f = f


@pytest.mark.parametrize('precision', ['fp64', 'fp32', 'fp64-fast'])
def test_nan_in_f_raises_solver_diverging(precision):
    nls = make_solver(SPEC, precision)
    nls.strang_timestep(SPEC['dt'])
    torch.cuda.synchronize()
    nls.check_divergence()                          # a clean step leaves no flag
    _poison(nls)
    pair0 = nls.paired_launch_count()
    with pytest.raises(SystemExit, match='Solver Diverging!'):
        for _ in range(3):
            nls.strang_timestep(SPEC['dt'])
            torch.cuda.synchronize()
    if precision != 'fp64':
        assert nls.paired_launch_count() > pair0    # the paired kernel raised the flag
    nls.synchronize()                               # no timeout or CUDA error besides


def test_nan_through_c_abi_sets_divergence_flag():
    """bolt_step on a ctypes-created context, then bolt_divergence_flag: 0 on
    clean data, 1 after a NaN, 0 again after bolt_clear_divergence_flag."""
    from test_zz_no_alloc import grid_params
    lib = N.load()
    torch.cuda.set_device(0)
    spec = C.CASES['c3_2d3v_weno5_rk4_small']
    g, p = grid_params(spec, N.F64)
    f = torch.from_numpy(np.ascontiguousarray(C.initial_f(spec))).to('cuda', torch.float64)
    stream = torch.cuda.current_stream().cuda_stream
    ctx = ctypes.c_void_p()
    assert lib.bolt_ctx_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(ctx)) == N.BOLT_OK
    try:
        assert lib.bolt_step(ctx, f.data_ptr(), 1e-3, stream) == N.BOLT_OK
        assert lib.bolt_status_sync(ctx, stream) == N.BOLT_OK
        assert lib.bolt_divergence_flag(ctx) == 0
        Ng = spec['N_ghost']
        f[Ng + 2, Ng + 5, 0, 3, 4, 1] = float('nan')
        assert lib.bolt_invalidate(ctx) == N.BOLT_OK
        assert lib.bolt_step(ctx, f.data_ptr(), 1e-3, stream) == N.BOLT_OK
        assert lib.bolt_status_sync(ctx, stream) == N.BOLT_OK
        assert lib.bolt_divergence_flag(ctx) == 1
        assert lib.bolt_clear_divergence_flag(ctx) == N.BOLT_OK
        assert lib.bolt_divergence_flag(ctx) == 0
    finally:
        lib.bolt_ctx_destroy(ctx)


@pytest.mark.parametrize('precision', ['fp64', 'fp32', 'fp64-fast'])
def test_stalled_tile_wait_times_out_and_raises(precision):
    """Budget 1e5 cycles (~50 us) with the stall hook on: the step returns,
    its kernels record BOLT_ERR_TIMEOUT, check_divergence raises it as a
    BoltError, bolt_status_sync reports it; with the hook off and the error
    cleared, the same context steps correctly again."""
    nls = make_solver(SPEC, precision)
    lib, ctx = nls._lib, nls._ctx
    f0 = nls.f.clone()
    nls.set_wait_budget(100000)
    assert lib.bolt_test_stall_waits(ctx, 1) == N.BOLT_OK
    try:
        with pytest.raises(N.BoltError) as exc:
            for _ in range(3):
                nls.strang_timestep(SPEC['dt'])
                torch.cuda.synchronize()
        assert exc.value.code == N.BOLT_ERR_TIMEOUT
        assert lib.bolt_status_sync(ctx, nls._stream()) == N.BOLT_ERR_TIMEOUT
        assert lib.bolt_error_flag(ctx) == N.BOLT_ERR_TIMEOUT
    finally:
        lib.bolt_test_stall_waits(ctx, 0)
        nls.set_wait_budget(None)
    assert lib.bolt_clear_error(ctx) == N.BOLT_OK
    assert lib.bolt_error_flag(ctx) == N.BOLT_OK
    # the context is usable: from the saved state, one step equals a fresh solver's
    nls.f = f0
    nls.strang_timestep(SPEC['dt'])
    ref = make_solver(SPEC, precision)
    ref.f = f0
    ref.strang_timestep(SPEC['dt'])
    torch.cuda.synchronize()
    g = SPEC['N_ghost']
    assert rel(interior(to_layout(nls.f, SPEC), g), interior(to_layout(ref.f, SPEC), g)) == 0.0
    nls.synchronize()
