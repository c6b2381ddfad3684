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
    assert ctypes.sizeof(N.BoltParams) == 11 * 4 + 4 + 2 * 8 * 8 + 4 * 8


def test_strerror_and_null_args():
    lib = N.load()
    assert N.strerror(0) == 'ok'
    assert N.strerror(3) == 'Solver Diverging!'
    # argument validation happens before any CUDA call
    assert lib.bolt_ctx_create(None, None, None) == N.BOLT_ERR_ARG
    assert lib.bolt_step(None, None, 0.0, None) == N.BOLT_ERR_ARG
    assert lib.bolt_launch_count(None) == 0


def test_ctx_create_rejects_bad_grids_without_gpu():
    lib = N.load()
    g = N.BoltGrid()
    p = N.BoltParams()
    g.N_q1 = 0          # invalid
    ctx = ctypes.c_void_p()
    assert lib.bolt_ctx_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(ctx)) == N.BOLT_ERR_ARG


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
