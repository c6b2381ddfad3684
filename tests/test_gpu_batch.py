"""Ragged batch of 1D1V runs (bolt_b200.batch.BatchSolver) against the same
runs advanced one at a time by nonlinear_solver (FP32, same scheme) and
against the oracle (FP64); mass conservation of a collisionless batch.

Tolerances (normwise relative): batch vs single runs 1e-5 in f and 1e-6 in
the moments (both FP32 f with FP64 moments, the batch evaluating the
Maxwellian's exponential at FP32 accuracy); batch vs oracle 2e-6 in f and
moments, as for the other FP32 parity tests."""

import os
import sys

import numpy as np
import pytest
import torch

import cases as C
from _util import interior, rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

pytestmark = pytest.mark.gpu

RUNS = [dict(N_q1=32, N_p1=64, tau=0.01, amp=0.05, k=1),
        dict(N_q1=48, N_p1=96, tau=0.002, amp=0.1, k=2),
        dict(N_q1=8, N_p1=32, tau=0.05, amp=0.02, k=1),
        dict(N_q1=44, N_p1=128, tau=0.001, amp=0.003, k=3),
        dict(N_q1=36, N_p1=32, tau=0.03, amp=0.08, k=4)]
for _r in RUNS:
    _r['dt'] = 0.5 * (1.0 / _r['N_q1']) / 10.0
STEPS = 12


def _case(run, source=True):
    """The same run as a case spec of tests/golden/cases.py (for the oracle)."""
    return C.make(N_q1=run['N_q1'], N_q2=1, N_p1=run['N_p1'], N_p2=1, N_p3=1,
                  p1_start=[-10.0], p1_end=[10.0], p2_start=[-0.5], p2_end=[0.5],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[0.0], p_dim=1,
                  tau=run['tau'], dt=run['dt'], integrator='RK4', source_enabled=source,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=run['amp'], k1=run['k'], k2=0))


def _q1p(af):
    """AF-ordered 1D1V f (N_p1, 1, N_q1g, N_q2g) -> numpy (N_q1g, N_p1) of the
    interior q2 row."""
    a = af.detach().to(torch.float64).cpu()
    return a[:, 0, :, a.shape[3] // 2].T.numpy()


def _oracle_f(spec, q1p):
    """(N_q1g, N_p1) -> the oracle's (q2g, q1g, s, p3, p2, p1) with the periodic
    q2 ghost rows (all equal for N_q2 = 1)."""
    q2g = spec['N_q2'] + 2 * spec['N_ghost']
    return np.ascontiguousarray(np.broadcast_to(q1p[None, :, None, None, None, :],
                                                (q2g,) + q1p.shape[:1] + (1, 1, 1) + q1p.shape[1:]))


def test_batch_matches_single_runs():
    from bolt_b200.batch import BatchSolver
    from bolt_b200.nonlinear_solver import nonlinear_solver
    bs = BatchSolver([bench.ragged_system(r) for r in RUNS], [r['dt'] for r in RUNS])
    bs.run(STEPS)
    bs.synchronize()
    for i, r in enumerate(RUNS):
        nls = nonlinear_solver(bench.ragged_system(r))
        for _ in range(STEPS):
            nls.strang_timestep(r['dt'])
        e = rel(_q1p(bs.f(i))[3:-3], _q1p(nls.f)[3:-3])
        assert e < 1e-5, (i, e)
        for name in ('density', 'energy'):
            a = bs.compute_moments(name, i)[0, 0, :, 0].cpu().numpy()
            b = nls.compute_moments(name)[0, 0, 3:-3, 3].cpu().numpy()
            assert rel(a, b) < 1e-6, (i, name, rel(a, b))
        assert abs(bs.time_elapsed[i] - nls.time_elapsed) < 1e-12


@pytest.mark.parametrize('i', [0, 1, 3])
def test_batch_matches_oracle(i):
    from bolt_b200.batch import BatchSolver
    from oracle.bolt_oracle import Oracle
    r = RUNS[i]
    spec = _case(r)
    bs = BatchSolver([bench.ragged_system(x) for x in RUNS], [x['dt'] for x in RUNS])
    o = Oracle(spec, _oracle_f(spec, _q1p(bs.f(i))))
    bs.run(STEPS)
    bs.synchronize()
    for _ in range(STEPS):
        o.step(r['dt'])
    e = rel(_q1p(bs.f(i))[3:-3], o.f[3, 3:-3, 0, 0, 0, :])
    assert e < 2e-6, e
    for name in ('density', 'mom_v1_bulk', 'energy'):
        a = bs.compute_moments(name, i)[0, 0, :, 0].cpu().numpy()
        b = interior(o.moments(name), 3)[0, :, 0]
        scale = max(np.linalg.norm(b), np.linalg.norm(interior(o.moments('density'), 3)))
        assert np.linalg.norm(a - b) / scale < 2e-6, (name,)


def test_collisionless_batch_conserves_mass():
    from bolt_b200.batch import BatchSolver
    runs = RUNS[:3]
    bs = BatchSolver([bench.ragged_system(r, source=False) for r in runs],
                     [r['dt'] for r in runs])
    m0 = [float(bs.compute_moments('density', i).sum()) for i in range(len(runs))]
    bs.run(40)
    bs.synchronize()
    for i in range(len(runs)):
        m1 = float(bs.compute_moments('density', i).sum())
        assert abs(m1 - m0[i]) < 2e-6 * abs(m0[i]), (i, m0[i], m1)


def test_every_schedule_gives_identical_results_and_autotune_keeps_the_state():
    """The autotuner's candidate schedules (tile height 16/32/64 q-cells,
    CTAs per SM, queue order) compute every cell the same way: f and the
    moments after the steps are bit-identical.  autotune() times them from
    the current f and leaves f unchanged."""
    from bolt_b200.batch import BatchSolver
    systems = [bench.ragged_system(r) for r in RUNS]
    dts = [r['dt'] for r in RUNS]
    ref = None
    for sched in [(32, 2, 1), (16, 4, 0), (64, 1, 1), (16, 1, 1), (8, 8, 1)]:
        bs = BatchSolver(systems, dts, autotune=False)
        bs.set_schedule(*sched)
        assert bs.schedule()[0] == sched[0]
        bs.run(STEPS)
        bs.synchronize()
        out = (bs._flat.clone(), [bs.compute_moments('energy', r) for r in range(len(RUNS))])
        if ref is None:
            ref = out
        else:
            assert torch.equal(out[0], ref[0]), sched
            assert all(torch.equal(a, b) for a, b in zip(out[1], ref[1])), sched
    bs = BatchSolver(systems, dts, autotune=False)
    before = bs._flat.clone()
    res = bs.autotune(steps=2, repeats=1)
    assert torch.equal(bs._flat, before)
    assert len(res) >= 6 and bs.tuning['chosen']['ms_per_step'] > 0
    bs.run(STEPS)
    bs.synchronize()
    assert torch.equal(bs._flat, ref[0])
