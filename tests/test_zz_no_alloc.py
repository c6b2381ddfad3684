"""bolt_dfdt_noalloc: the allocation-free df/dt entry point.

Callers that cannot allocate device memory when they need an evaluation (a
fixed-budget memory pool, code that must not trigger the implicit device
synchronisation of cudaMalloc/cudaFree, an embedder that owns all device
memory) call bolt_dfdt_noalloc, whose only scratch is a fixed array inside the
library.  These tests call it through the C ABI and compare it with the
context-based bolt_dfdt on the same f, twice in a row (the shared scratch keeps
the previous call's contents, which must not leak into the next result), and
with the reference's df/dt of that f.  Tolerances: 1e-12 normwise (FP64) and
1e-6 (FP32) against bolt_dfdt (the same kernels, so agreement is expected to
be exact); against the reference fixture 1e-12 (FP64) and 1e-3 (FP32: flux
differences cancel, as in the other parity tests).  bolt_noalloc_status reads
the call's error word and non-finite flag."""

import ctypes

import numpy as np
import pytest
import torch

import cases as C
import bolt_b200._native as N
from _util import load_golden

SPEC = C.CASES['c3_2d3v_weno5_rk4_small']


def grid_params(spec, dtype):
    g = N.BoltGrid()
    g.N_q1, g.N_q2, g.N_ghost = spec['N_q1'], spec['N_q2'], spec['N_ghost']
    g.N_p1, g.N_p2, g.N_p3, g.N_s = spec['N_p1'], spec['N_p2'], spec['N_p3'], len(spec['mass'])
    g.q1_start, g.q2_start = spec['q1_start'], spec['q2_start']
    g.dq1 = (spec['q1_end'] - spec['q1_start']) / spec['N_q1']
    g.dq2 = (spec['q2_end'] - spec['q2_start']) / spec['N_q2']
    p = N.BoltParams()
    p.dtype = dtype
    p.recon_q = p.recon_p = N.RECON[spec['recon_q']]
    p.bc_q1 = p.bc_q2 = N.BC['periodic']
    p.integrator = N.RK[spec['integrator']]
    p.source_enabled = 1
    p.p_dim = spec['p_dim']
    p.boltzmann_constant = spec['boltzmann_constant']
    p.tau = spec['tau']
    p.eps = p.mu = 1.0
    for s in range(g.N_s):
        for d in (1, 2, 3):
            a, b, n = spec['p%d_start' % d][s], spec['p%d_end' % d][s], spec['N_p%d' % d]
            getattr(g, 'p%d_start' % d)[s] = a
            getattr(g, 'dp%d' % d)[s] = (b - a) / n
        p.mass[s] = spec['mass'][s]
        p.charge[s] = spec['charge'][s]
    return g, p


def _status(lib, stream):
    st = ctypes.c_int(-1)
    assert lib.bolt_noalloc_status(stream, ctypes.byref(st)) == N.BOLT_OK
    return st.value


@pytest.mark.gpu
@pytest.mark.parametrize('dtype,tol,tol_ref', [(N.F64, 1e-12, 1e-12), (N.F32, 1e-6, 1e-3)])
def test_noalloc_matches_context_dfdt_twice(dtype, tol, tol_ref):
    lib = N.load()
    torch.cuda.set_device(0)
    tdt = torch.float64 if dtype == N.F64 else torch.float32
    g, p = grid_params(SPEC, dtype)
    G = load_golden('c3_2d3v_weno5_rk4_small')
    # the reference's halo-refreshed initial state, whose df/dt the fixture holds
    f = torch.from_numpy(np.ascontiguousarray(G['f0_refreshed'])).to('cuda', tdt)
    stream = torch.cuda.current_stream().cuda_stream
    ctx = ctypes.c_void_p()
    assert lib.bolt_ctx_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(ctx)) == N.BOLT_OK
    try:
        ref = torch.zeros_like(f)
        assert lib.bolt_dfdt(ctx, f.data_ptr(), ref.data_ptr(), 0, 0.0, stream) == N.BOLT_OK
        assert lib.bolt_status_sync(ctx, stream) == N.BOLT_OK
    finally:
        lib.bolt_ctx_destroy(ctx)
    Ng = SPEC['N_ghost']
    inner = lambda t: t[Ng:-Ng, Ng:-Ng].double().cpu().numpy()
    r = inner(ref)
    outs = [torch.zeros_like(f), torch.full_like(f, float('nan'))]
    torch.cuda.synchronize()
    for call in range(2):
        free0 = torch.cuda.mem_get_info()[0]
        rc = lib.bolt_dfdt_noalloc(ctypes.byref(g), ctypes.byref(p), f.data_ptr(),
                                   outs[call].data_ptr(), stream)
        assert rc == N.BOLT_OK, N.strerror(rc)
        assert _status(lib, stream) == N.BOLT_OK
        if call:
            # no device memory was taken by the call (the first call on the
            # device may load the library's module; the second allocates nothing)
            assert torch.cuda.mem_get_info()[0] == free0
        got = inner(outs[call])
        err = np.linalg.norm(got - r) / np.linalg.norm(r)
        assert err < tol, (call, err)
        e_ref = np.linalg.norm(got - G['dfdt0']) / np.linalg.norm(G['dfdt0'])
        assert e_ref < tol_ref, (call, e_ref)


@pytest.mark.gpu
def test_noalloc_status_reports_nonfinite_and_clears():
    lib = N.load()
    torch.cuda.set_device(0)
    g, p = grid_params(SPEC, N.F64)
    G = load_golden('c3_2d3v_weno5_rk4_small')
    f = torch.from_numpy(np.ascontiguousarray(G['f0_refreshed'])).to('cuda', torch.float64)
    Ng = SPEC['N_ghost']
    f[Ng + 1, Ng + 2, 0, 1, 2, 3] = float('nan')
    out = torch.zeros_like(f)
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.bolt_dfdt_noalloc(ctypes.byref(g), ctypes.byref(p), f.data_ptr(), out.data_ptr(),
                                 stream) == N.BOLT_OK
    assert _status(lib, stream) == N.BOLT_ERR_NONFINITE
    assert _status(lib, stream) == N.BOLT_OK          # read once, then cleared


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Checked before any device work, so it needs no GPU."""
    lib = N.load()
    spec = dict(SPEC)
    spec['N_q1'], spec['N_q2'] = 512, 256          # 131072 q-cells > 65536
    g, p = grid_params(spec, N.F64)
    rc = lib.bolt_dfdt_noalloc(ctypes.byref(g), ctypes.byref(p), ctypes.c_void_p(16),
                               ctypes.c_void_p(16), None)
    assert rc == N.BOLT_ERR_UNSUPPORTED
    p.fields_enabled = 1
    g2, _ = grid_params(SPEC, N.F64)
    assert lib.bolt_dfdt_noalloc(ctypes.byref(g2), ctypes.byref(p), ctypes.c_void_p(16),
                                 ctypes.c_void_p(16), None) == N.BOLT_ERR_UNSUPPORTED


def test_noalloc_validates_like_the_context():
    """Grids and parameters bolt_ctx_create refuses are refused alike, before
    any device work: unknown boundary codes, a mirror deeper than the grid, a
    non-periodic axis without ghost cells, BGK without a positive tau."""
    lib = N.load()

    def call(**kw):
        g, p = grid_params(SPEC, N.F64)
        for k, v in kw.items():
            setattr(g if hasattr(g, k) and k.startswith('N_') else p, k, v)
        return lib.bolt_dfdt_noalloc(ctypes.byref(g), ctypes.byref(p), ctypes.c_void_p(16),
                                     ctypes.c_void_p(16), None)
    assert call(bc_q1=9) == N.BOLT_ERR_ARG
    assert call(bc_q2=-1) == N.BOLT_ERR_ARG
    assert call(bc_q1=N.BC['mirror'], N_ghost=9) == N.BOLT_ERR_UNSUPPORTED
    assert call(bc_q2=N.BC['dirichlet'], N_ghost=0) == N.BOLT_ERR_UNSUPPORTED
    assert call(tau=0.0) == N.BOLT_ERR_ARG
    assert lib.bolt_noalloc_status(None, None) == N.BOLT_ERR_ARG
