"""Hand-written adjoint of the 1D1V update (bolt_b200.adjoint) against autograd
of the FP64 PyTorch transcription of the reference scheme (oracle/bolt_torch.py)
and against central finite differences (relative step 1e-4).

Small problem: N_q1 = 32, N_p1 = 64, p1 in [-10, 10], tau = 0.02, dt = 4e-4,
60 RK4 steps, f0 = (1 + a cos 2 pi q1) times two Maxwellians at p1 = +-1.5 (a single
Maxwellian for the forward comparison with nonlinear_solver), a = 0.01.
Tolerances: forward J and f_N vs the transcription 1e-12 (FP64); gradients vs
autograd 1e-9 (the same derivatives, different operation order); vs central
differences 1e-4 (O(h^2) truncation plus FP64 round-off amplified by 1/h); the
checkpointed gradient equals the store-every-step one to 1e-14; FP32 gradient
within 1e-3 of FP64 (dJ/dtau 2e-2)."""

import math

import pytest
import torch

pytestmark = pytest.mark.gpu

NQ, NP, P0, P1, TAU, DT, STEPS, AMP = 32, 64, -10.0, 10.0, 0.02, 4e-4, 60, 0.01


def f_init(a, device, dtype=torch.float64, two_stream=True):
    """(1 + a cos 2 pi q1) times a symmetric pair of Maxwellians at p1 = +-1.5
    (far from the local Maxwellian, so BGK and tau matter from the start), or
    times a single Maxwellian."""
    dq = 1.0 / NQ
    x = (0.5 + torch.arange(NQ, dtype=torch.float64, device=device)) * dq
    dp = (P1 - P0) / NP
    v = P0 + (0.5 + torch.arange(NP, dtype=torch.float64, device=device)) * dp
    mx = lambda u: torch.exp(-(v - u) ** 2 / 2) / math.sqrt(2 * math.pi)
    shape = 0.5 * (mx(1.5) + mx(-1.5)) if two_stream else mx(0.0)
    return ((1 + a * torch.cos(2 * math.pi * x))[:, None] * shape[None, :]).to(dtype)


def roll(precision='fp64', snapshots=4, steps=STEPS):
    from bolt_b200.adjoint import Rollout1D1V
    return Rollout1D1V(NQ, NP, P0, P1, DT, TAU, steps, snapshots=snapshots, precision=precision)


def transcription(device='cuda'):
    from oracle.bolt_torch import Problem1D1V
    return Problem1D1V(NQ, NP, P0, P1, DT, TAU, device=device)


def test_forward_matches_transcription_and_solver():
    """The adjoint module's forward is the solver's scheme: J and f_N against the
    transcription, f_N against nonlinear_solver (FP64, the same 1D1V run)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from bolt_b200.nonlinear_solver import nonlinear_solver
    r = roll()
    f0 = f_init(AMP, 'cuda', two_stream=False)
    J, fN = r.forward(f0)
    pr = transcription()
    Jt, ft = pr.objective(f0, torch.tensor(TAU, dtype=torch.float64, device='cuda'), STEPS)
    assert abs(float(J) - float(Jt)) < 1e-12 * abs(float(Jt))
    assert float((fN - ft).norm() / ft.norm()) < 1e-12
    nls = nonlinear_solver(bench.ragged_system(dict(N_q1=NQ, N_p1=NP, tau=TAU, amp=AMP, k=1),
                                               precision='fp64'))
    for _ in range(STEPS):
        nls.strang_timestep(DT)
    fs = nls.f[:, 0, 3:-3, 3].T          # (N_q1, N_p1), interior q2 row
    assert float((fN - fs).norm() / fs.norm()) < 1e-12


def test_gradients_match_autograd_of_transcription():
    r = roll()
    a = torch.tensor(AMP, dtype=torch.float64, device='cuda', requires_grad=True)
    tau = torch.tensor(TAU, dtype=torch.float64, device='cuda', requires_grad=True)
    from bolt_b200.adjoint import rollout
    J = rollout(f_init(a, 'cuda'), tau, r)
    J.backward()
    g_a, g_tau = float(a.grad), float(tau.grad)
    f0 = f_init(AMP, 'cuda').requires_grad_(True)
    gf, _ = r.gradient(f0.detach())

    a2 = torch.tensor(AMP, dtype=torch.float64, device='cuda', requires_grad=True)
    tau2 = torch.tensor(TAU, dtype=torch.float64, device='cuda', requires_grad=True)
    f02 = f_init(a2, 'cuda')
    f02.retain_grad()
    Jt, _ = transcription().objective(f02, tau2, STEPS)
    Jt.backward()
    assert abs(float(J.detach()) - float(Jt.detach())) < 1e-12 * abs(float(Jt.detach()))
    assert abs(g_a - float(a2.grad)) < 1e-9 * abs(float(a2.grad))
    assert abs(g_tau - float(tau2.grad)) < 1e-9 * abs(float(tau2.grad))
    assert float((gf - f02.grad).norm() / f02.grad.norm()) < 1e-9


def test_gradients_match_central_differences():
    r = roll()
    tau0 = TAU
    J = lambda a, tau: float(r.forward(f_init(a, 'cuda'), tau)[0])
    a = torch.tensor(AMP, dtype=torch.float64, device='cuda', requires_grad=True)
    tau = torch.tensor(TAU, dtype=torch.float64, device='cuda', requires_grad=True)
    from bolt_b200.adjoint import rollout
    rollout(f_init(a, 'cuda'), tau, r).backward()
    h = 1e-4
    fd_a = (J(AMP * (1 + h), tau0) - J(AMP * (1 - h), tau0)) / (2 * AMP * h)
    fd_tau = (J(AMP, tau0 * (1 + h)) - J(AMP, tau0 * (1 - h))) / (2 * tau0 * h)
    assert abs(float(a.grad) - fd_a) < 1e-4 * abs(fd_a)
    assert abs(float(tau.grad) - fd_tau) < 1e-4 * abs(fd_tau)
    # dJ/df0 along a smooth random direction (white noise of relative size h is
    # not in the linear range of the WENO5 weights)
    g = torch.Generator().manual_seed(0)
    c = torch.rand(4, generator=g, dtype=torch.float64).tolist()
    f0 = f_init(AMP, 'cuda')
    x = ((0.5 + torch.arange(NQ, dtype=torch.float64)) / NQ).cuda()[:, None]
    v = (P0 + (0.5 + torch.arange(NP, dtype=torch.float64)) * (P1 - P0) / NP).cuda()[None, :]
    d = f0 * (c[0] * torch.sin(2 * math.pi * x) + c[1] * torch.cos(4 * math.pi * x)) \
        * (1 + c[2] * v + c[3] * v * v / 4)
    gf, _ = r.gradient(f0, tau0)
    eps = 1e-4 * float(f0.norm() / d.norm())
    fd = (float(r.forward(f0 + eps * d, tau0)[0]) - float(r.forward(f0 - eps * d, tau0)[0])) / (2 * eps)
    ad = float((gf * d).sum())
    assert abs(ad - fd) < 1e-4 * abs(fd)


def test_checkpointing_matches_store_all():
    f0 = f_init(AMP, 'cuda')
    g_all, t_all = roll(snapshots=STEPS).gradient(f0)
    r3 = roll(snapshots=3)
    g3, t3 = r3.gradient(f0)
    assert float((g3 - g_all).norm() / g_all.norm()) < 1e-14
    assert abs(float(t3) - float(t_all)) < 1e-14 * abs(float(t_all))
    assert r3.forward_steps > STEPS          # recomputation happened


def test_fp32_gradient_close_to_fp64():
    """FP32 f (FP64 moments) against FP64: dJ/df0 within 1e-3; dJ/dtau within
    2e-2, because it is the inner product of the adjoint with f0 - f, whose
    density, momentum and energy moments vanish, so FP32 rounding of f is
    measured against a strongly cancelled sum."""
    f0 = f_init(AMP, 'cuda')
    g64, t64 = roll('fp64').gradient(f0)
    g32, t32 = roll('fp32').gradient(f0)
    assert float((g32.double() - g64).norm() / g64.norm()) < 1e-3
    assert abs(float(t32) - float(t64)) < 2e-2 * abs(float(t64))


def test_minmod_adjoint_subgradient():
    """reconstruction='minmod': the forward equals the transcription's (1e-12),
    the hand-written subgradient equals autograd of the transcription, whose
    minmod routes the derivative through the same passed argument (1e-9 for
    dJ/da, dJ/dtau and dJ/df0), and the derivatives in a and tau match
    central differences to 1e-3 (J is only piecewise smooth: a kink of the
    limiter inside the +-h interval costs O(h))."""
    from bolt_b200.adjoint import Rollout1D1V, rollout
    from oracle.bolt_torch import Problem1D1V
    r = Rollout1D1V(NQ, NP, P0, P1, DT, TAU, STEPS, snapshots=4, precision='fp64',
                    reconstruction='minmod')
    pr = Problem1D1V(NQ, NP, P0, P1, DT, TAU, device='cuda', reconstruction='minmod')
    f0 = f_init(AMP, 'cuda')
    J, fN = r.forward(f0)
    Jt, ft = pr.objective(f0, torch.tensor(TAU, dtype=torch.float64, device='cuda'), STEPS)
    assert abs(float(J) - float(Jt)) < 1e-12 * abs(float(Jt))
    assert float((fN - ft).norm() / ft.norm()) < 1e-12

    a = torch.tensor(AMP, dtype=torch.float64, device='cuda', requires_grad=True)
    tau = torch.tensor(TAU, dtype=torch.float64, device='cuda', requires_grad=True)
    rollout(f_init(a, 'cuda'), tau, r).backward()
    gf, _ = r.gradient(f0)
    a2 = torch.tensor(AMP, dtype=torch.float64, device='cuda', requires_grad=True)
    tau2 = torch.tensor(TAU, dtype=torch.float64, device='cuda', requires_grad=True)
    f02 = f_init(a2, 'cuda')
    f02.retain_grad()
    pr.objective(f02, tau2, STEPS)[0].backward()
    assert abs(float(a.grad) - float(a2.grad)) < 1e-9 * abs(float(a2.grad))
    assert abs(float(tau.grad) - float(tau2.grad)) < 1e-9 * abs(float(tau2.grad))
    assert float((gf - f02.grad).norm() / f02.grad.norm()) < 1e-9

    h = 1e-4
    Jf = lambda amp, t: float(r.forward(f_init(amp, 'cuda'), t)[0])
    fd_a = (Jf(AMP * (1 + h), TAU) - Jf(AMP * (1 - h), TAU)) / (2 * AMP * h)
    fd_tau = (Jf(AMP, TAU * (1 + h)) - Jf(AMP, TAU * (1 - h))) / (2 * TAU * h)
    assert abs(float(a.grad) - fd_a) < 1e-3 * abs(fd_a)
    assert abs(float(tau.grad) - fd_tau) < 1e-3 * abs(fd_tau)


@pytest.mark.parametrize('precision,tol,tol_tau', [('fp64', 1e-10, 1e-9), ('fp32', 1e-5, 2e-2)])
def test_cooperative_steps_match_separate_launches(monkeypatch, precision, tol, tol_tau):
    """Whole RK4 steps and step adjoints as single cooperative launches
    (the default) against the same passes as separate launches
    (BOLT_ADJ_SEPARATE): J, f_N and the gradients agree to rounding (the
    fused epilogues may contract the elementwise combines into FMAs where the
    separate axpby launches do not; 60 adjoint steps through the WENO weight
    derivatives amplify that to ~1e-11 in FP64; dJ/dtau in FP32 is a strongly
    cancelled sum, see test_fp32_gradient_close_to_fp64)."""
    f0 = f_init(AMP, 'cuda')
    coop = roll(precision)
    Jc, fc = coop.forward(f0)
    gc, tc = coop.gradient(f0)
    monkeypatch.setenv('BOLT_ADJ_SEPARATE', '1')
    sep = roll(precision)
    Js, fs = sep.forward(f0)
    gs, ts = sep.gradient(f0)
    assert abs(float(Jc) - float(Js)) <= tol * abs(float(Js))
    assert float((fc - fs).norm() / fs.norm()) <= tol
    assert float((gc - gs).norm() / gs.norm()) <= tol
    assert abs(float(tc) - float(ts)) <= tol_tau * abs(float(ts))
