"""FP64 PyTorch transcription of Bolt's 1D1V FVM update, differentiable by
autograd.  TEST INFRASTRUCTURE: the checker of the hand-written adjoint
(bolt_b200.adjoint); only tests/ and bench.py's checks import it.

It restates, on torch tensors f[i, p] (N_q1 periodic q-cells x N_p1 p-cells,
p_dim = 1, one species, fields off):
  * reconstruct_weno5 (bolt/lib/nonlinear/finite_volume/reconstruction/
    weno5.py:17-96): circular shifts along q, smoothness indicators with
    eps * (1 + |a| + |b| + |c|), weights c/(16 beta^2) style, normalised sums;
    or reconstruct_minmod (minmod.py:4-71);
  * riemann_solver (riemann.py:46-49): left state where the velocity is
    positive, right state otherwise (the LLF flux with alpha = |v| equals it);
  * the q-flux divergence of df_dt_fvm.py:56-89, -(F_i+1/2 - F_i-1/2)/dq1;
  * BGK and f0 (src/nonrelativistic_boltzmann/collision_operator.py:49-128)
    with the moments of moments.py (density, mom_v1_bulk, energy; p2 and p3
    centred at 0);
  * RK4 (integrators.py:15-28);
  * the objective J = sum_{n >= 1} dt |nhat_1(f_n)|^2 with
    nhat_1 = (1/N_q1) sum_i n_i exp(-2 pi i x_i / L), x_i the cell centres.
"""

import math

import torch


def weno5_faces(f):
    """(left_value, right_value) of every cell along dim 0 (weno5.py:58-96)."""
    eps = 1e-17
    y0 = torch.roll(f, 2, 0)
    y1 = torch.roll(f, 1, 0)
    y2 = f
    y3 = torch.roll(f, -1, 0)
    y4 = torch.roll(f, -2, 0)
    beta1 = ((4 / 3) * y0 * y0 - (19 / 3) * y0 * y1 + (25 / 3) * y1 * y1
             + (11 / 3) * y0 * y2 - (31 / 3) * y1 * y2 + (10 / 3) * y2 * y2) \
        + eps * (1.0 + y0.abs() + y1.abs() + y2.abs())
    beta2 = ((4 / 3) * y1 * y1 - (19 / 3) * y1 * y2 + (25 / 3) * y2 * y2
             + (11 / 3) * y1 * y3 - (31 / 3) * y2 * y3 + (10 / 3) * y3 * y3) \
        + eps * (1.0 + y1.abs() + y2.abs() + y3.abs())
    beta3 = ((4 / 3) * y2 * y2 - (19 / 3) * y2 * y3 + (25 / 3) * y3 * y3
             + (11 / 3) * y2 * y4 - (31 / 3) * y3 * y4 + (10 / 3) * y4 * y4) \
        + eps * (1.0 + y2.abs() + y3.abs() + y4.abs())
    w1r, w2r, w3r = 1 / (16 * beta1 * beta1), 5 / (8 * beta2 * beta2), 5 / (16 * beta3 * beta3)
    w1l, w2l, w3l = 5 / (16 * beta1 * beta1), 5 / (8 * beta2 * beta2), 1 / (16 * beta3 * beta3)
    u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2
    u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3
    u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4
    u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2
    u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3
    u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4
    left = (w1l * u1l + w2l * u2l + w3l * u3l) / (w1l + w2l + w3l)
    right = (w1r * u1r + w2r * u2r + w3r * u3r) / (w1r + w2r + w3r)
    return left, right


def minmod_faces(f):
    """(left_value, right_value) of every cell along dim 0 with the minmod
    limited slope of minmod.py:4-71 (theta = 2, sign(0) = +1).  The slope is
    written as the passed argument itself (the first of equal magnitudes)
    where the three arguments share a sign, else 0 -- the same values as the
    reference's 0.25 |sx + sy| (sx + sz) min|.|, and the subgradient autograd
    takes through it is the hand-written adjoint's."""
    bwd = f - torch.roll(f, 1, 0)
    fwd = torch.roll(f, -1, 0) - f
    cen = bwd + fwd
    x0, x1, x2 = 2 * bwd, 0.5 * cen, 2 * fwd
    a0, a1, a2 = x0.abs().detach(), x1.abs().detach(), x2.abs().detach()
    m = torch.minimum(torch.minimum(a0, a1), a2)
    sel = torch.where(a0 == m, x0, torch.where(a1 == m, x1, x2))
    neg0, neg1, neg2 = x0.detach() < 0, x1.detach() < 0, x2.detach() < 0
    agree = (neg0 == neg1) & (neg0 == neg2)
    slope = torch.where(agree, sel, torch.zeros_like(sel))
    return f - 0.5 * slope, f + 0.5 * slope


class Problem1D1V(object):
    """Grid and constants of one 1D1V run (p1 centres v, dp2 = dp3 given)."""

    def __init__(self, N_q1, N_p1, p1_start, p1_end, dt, tau, mass=1.0, kB=1.0,
                 q1_start=0.0, q1_end=1.0, dp2=1.0, dp3=1.0, device='cpu',
                 reconstruction='weno5'):
        self.faces = minmod_faces if reconstruction == 'minmod' else weno5_faces
        self.N_q1, self.N_p1 = N_q1, N_p1
        self.dq1 = (q1_end - q1_start) / N_q1
        self.dp1 = (p1_end - p1_start) / N_p1
        self.v = (p1_start + (0.5 + torch.arange(N_p1, dtype=torch.float64)) * self.dp1).to(device)
        self.x = (q1_start + (0.5 + torch.arange(N_q1, dtype=torch.float64)) * self.dq1).to(device)
        self.dt, self.tau, self.mass, self.kB = dt, tau, mass, kB
        self.measure = dp3 * dp2 * self.dp1
        th = 2 * math.pi * (torch.arange(N_q1, dtype=torch.float64) + 0.5) / N_q1
        self.cos, self.sin = torch.cos(th).to(device), torch.sin(th).to(device)

    def dfdt(self, f, tau):
        v = self.v[None, :]
        left, right = self.faces(f)
        # state at face i+1/2: right value of cell i (v > 0) or left value of cell i+1
        face = torch.where(v > 0, right, torch.roll(left, -1, 0))
        F = v * face
        out = -(F - torch.roll(F, 1, 0)) / self.dq1
        if tau is not None:
            m, k, eps = self.mass, self.kB, 1e-30
            n = f.sum(1, keepdim=True) * self.measure
            m1 = (f * v).sum(1, keepdim=True) * self.measure
            E = (0.5 * f * v * v).sum(1, keepdim=True) * self.measure
            u = m1 / (n + eps)
            T = (2 * E * m - n * m * u ** 2) / (n + eps) + eps      # p_dim = 1, v2 = v3 = 0
            f0 = n * torch.sqrt(m / (2 * math.pi * k * T)) * torch.exp(-m * (v - u) ** 2 / (2 * k * T))
            out = out - (f - f0) / tau
        return out

    def step(self, f, tau):
        dt = self.dt
        k1 = self.dfdt(f, tau)
        k2 = self.dfdt(f + 0.5 * dt * k1, tau)
        k3 = self.dfdt(f + 0.5 * dt * k2, tau)
        k4 = self.dfdt(f + dt * k3, tau)
        return f + (dt / 6) * (k1 + 2 * k2 + 2 * k3 + k4)

    def mode_power(self, f):
        n = f.sum(1) * self.measure
        re = (n * self.cos).sum() / self.N_q1
        im = -(n * self.sin).sum() / self.N_q1
        return re * re + im * im

    def objective(self, f0, tau, nsteps, checkpoint_every=0):
        """J and f_N; checkpoint_every > 0 recomputes blocks of steps in the
        backward pass (torch.utils.checkpoint) to bound memory."""
        f = f0
        J = torch.zeros((), dtype=torch.float64, device=f0.device)

        def block(f, tau, k):
            J = torch.zeros((), dtype=torch.float64, device=f.device)
            for _ in range(k):
                f = self.step(f, tau)
                J = J + self.dt * self.mode_power(f)
            return f, J
        n = 0
        while n < nsteps:
            k = min(checkpoint_every or nsteps, nsteps - n)
            if checkpoint_every:
                from torch.utils.checkpoint import checkpoint
                f, dJ = checkpoint(block, f, tau, k, use_reentrant=False)
            else:
                f, dJ = block(f, tau, k)
            J = J + dJ
            n += k
        return J, f
