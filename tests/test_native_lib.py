"""The C-ABI library loads and exports every function include/bolt_b200.h
declares (no GPU work)."""

import ctypes
import os
import re

import bolt_b200._native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, 'include', 'bolt_b200.h')).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(bolt_[a-z_0-9]+)\s*\(', src)))


def test_library_exports_all_declared_symbols():
    lib = N.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, name


def test_struct_layouts_match_header():
    # BoltGrid: 7 ints, 4 doubles, 6 x 8 doubles (with alignment padding)
    assert ctypes.sizeof(N.BoltGrid) == 7 * 4 + 4 + 4 * 8 + 6 * 8 * 8
    assert ctypes.sizeof(N.BoltParams) == 12 * 4 + 2 * 8 * 8 + 4 * 8


def test_strerror_and_null_args():
    lib = N.load()
    assert N.strerror(0) == 'ok'
    assert N.strerror(3) == 'Solver Diverging!'
    # argument validation happens before any CUDA call
    assert lib.bolt_ctx_create(None, None, None) == N.BOLT_ERR_ARG
    assert lib.bolt_step(None, None, 0.0, None) == N.BOLT_ERR_ARG
    assert lib.bolt_launch_count(None) == 0
    # the semi-Lagrangian operators, in place and between buffers
    assert lib.bolt_asl_advect_q(None, None, 0.0, None) == N.BOLT_ERR_ARG
    assert lib.bolt_asl_source(None, None, 0.0, 0, None) == N.BOLT_ERR_ARG
    assert lib.bolt_asl_advect_q_to(None, None, None, 0.0, None) == N.BOLT_ERR_ARG
    assert lib.bolt_asl_source_to(None, None, None, None, 0.0, 0, None) == N.BOLT_ERR_ARG
    ptr = ctypes.c_void_p()
    assert lib.bolt_work_buffer(None, 0, ctypes.byref(ptr)) == N.BOLT_ERR_ARG
    # the p-space grid setter: a context is required
    assert lib.bolt_set_p_space_grid(None, N.PGRID['polar2D'], 1.0) == N.BOLT_ERR_ARG


def test_ctx_create_rejects_bad_grids_without_gpu():
    lib = N.load()
    g = N.BoltGrid()
    p = N.BoltParams()
    g.N_q1 = 0          # invalid
    ctx = ctypes.c_void_p()
    assert lib.bolt_ctx_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(ctx)) == N.BOLT_ERR_ARG


def test_ctx_create_checks_boundary_conditions_without_gpu():
    """Boundary codes are validated before any device work: an unknown code is
    an argument error; a mirror whose ghost zone is deeper than the grid, or a
    non-periodic axis without ghost cells, is unsupported."""
    lib = N.load()

    def create(bc_q1, bc_q2, N_q1=8, N_ghost=3):
        g = N.BoltGrid()
        g.N_q1, g.N_q2, g.N_ghost, g.N_p1, g.N_p2, g.N_p3, g.N_s = N_q1, 8, N_ghost, 8, 8, 1, 1
        p = N.BoltParams()
        p.dtype, p.recon_q, p.recon_p = N.F64, N.RECON['weno5'], N.RECON['weno5']
        p.integrator, p.p_dim = N.RK['RK2'], 2
        p.bc_q1, p.bc_q2 = N.BC[bc_q1] if bc_q1 in N.BC else bc_q1, N.BC[bc_q2]
        ctx = ctypes.c_void_p()
        return lib.bolt_ctx_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(ctx))
    assert create(7, 'periodic') == N.BOLT_ERR_ARG
    assert create(-1, 'periodic') == N.BOLT_ERR_ARG
    assert create('mirror', 'periodic', N_q1=2) == N.BOLT_ERR_UNSUPPORTED
    assert create('periodic', 'mirror+dirichlet', N_ghost=0) == N.BOLT_ERR_UNSUPPORTED


def test_batch_run_layout_and_validation_without_gpu():
    lib = N.load()
    # BoltBatchRun: 2 ints, 12 doubles
    assert ctypes.sizeof(N.BoltBatchRun) == 2 * 4 + 12 * 8
    runs = (N.BoltBatchRun * 1)()
    R = runs[0]
    R.N_q1, R.N_p1 = 32, 64
    R.q1_start, R.q1_end, R.p1_start, R.p1_end = 0.0, 1.0, -10.0, 10.0
    R.dp2 = R.dp3 = 1.0
    R.mass = R.boltzmann_constant = 1.0
    R.tau, R.dt = 0.01, 1e-3
    b = ctypes.c_void_p()
    # shapes outside the batch kernel and invalid constants are refused before any CUDA call
    R.N_q1 = 30
    assert lib.bolt_batch_create(runs, 1, 1, ctypes.byref(b)) == N.BOLT_ERR_UNSUPPORTED
    R.N_q1, R.N_p1 = 32, 48
    assert lib.bolt_batch_create(runs, 1, 1, ctypes.byref(b)) == N.BOLT_ERR_UNSUPPORTED
    R.N_p1, R.dt = 64, 0.0
    assert lib.bolt_batch_create(runs, 1, 1, ctypes.byref(b)) == N.BOLT_ERR_ARG
    R.dt, R.tau = 1e-3, 0.0
    assert lib.bolt_batch_create(runs, 1, 1, ctypes.byref(b)) == N.BOLT_ERR_ARG
    assert lib.bolt_batch_create(runs, 0, 1, ctypes.byref(b)) == N.BOLT_ERR_ARG
    assert lib.bolt_batch_run(None, 1, None) == N.BOLT_ERR_ARG
    assert lib.bolt_batch_f_offset(None, 0) == -1
