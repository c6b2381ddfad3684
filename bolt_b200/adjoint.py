"""Gradients of a velocity-moment functional of the 1D1V kinetic update.

``Rollout1D1V`` advances f[N_q1, N_p1] (q1 periodic, p_dim = 1, one species,
fields off; WENO5 + upwind/LLF, BGK, RK4: the scheme of bolt_step for a 1D1V
system) with the adjoint kernels of libbolt_b200.so (include/bolt_b200.h,
"Adjoint"), and evaluates

    J = sum_{n = 1..N} dt |nhat_1(f_n)|^2,
    nhat_1 = (1/N_q1) sum_i n_i exp(-2 pi i x_i / L),

the time-integrated squared k = 1 Fourier amplitude of the density.  Its
gradient with respect to the initial f (every cell) and to the BGK collision
time tau comes from the hand-written adjoint of the RK4 step (exact
derivatives of the WENO5 nonlinear weights -- or, with
``reconstruction='minmod'``, a subgradient of the minmod limiter -- and of
the Maxwellian through the moments), run backwards over the trajectory with binomial checkpointing: at
most ``snapshots`` copies of f are held, and the forward steps are recomputed
in the recursive schedule of Griewank's treeverse (the left segment of n
steps with c snapshots and t sweeps holds at most C(c + t - 1, c) steps).

``rollout(f0, tau)`` is a torch.autograd.Function: J as a 0-d FP64 tensor whose
backward returns dJ/df0 and dJ/dtau, so gradients with respect to anything f0
is built from (for example the amplitude of the initial density
perturbation) follow from torch's chain rule.
"""

import math

import torch

from . import _native as N


def _beta(c, t):
    return math.comb(c + t, c)


class Rollout1D1V(object):

    def __init__(self, N_q1, N_p1, p1_start, p1_end, dt, tau, nsteps, snapshots=20,
                 precision='fp64', q1_start=0.0, q1_end=1.0, dp2=1.0, dp3=1.0, mass=1.0,
                 boltzmann_constant=1.0, reconstruction='weno5'):
        if not torch.cuda.is_available():
            raise RuntimeError('bolt_b200 runs on a CUDA device (sm_100a); no CUDA device '
                               'is available and there is no CPU fallback')
        self._lib = N.load()
        self.device = torch.device('cuda', torch.cuda.current_device())
        self.dtype = torch.float32 if precision in ('fp32', 'float32', 'single') else torch.float64
        self.shape = (int(N_q1), int(N_p1))
        self.nsteps = int(nsteps)
        self.snapshots = max(0, int(snapshots))
        s = N.BoltAdj1DSpec()
        s.N_q1, s.N_p1 = self.shape
        s.q1_start, s.q1_end, s.p1_start, s.p1_end = q1_start, q1_end, p1_start, p1_end
        s.dp2, s.dp3, s.mass, s.boltzmann_constant = dp2, dp3, mass, boltzmann_constant
        s.tau, s.dt = float(tau), float(dt)
        if reconstruction not in ('weno5', 'minmod'):
            raise NotImplementedError('adjoint reconstruction: weno5 or minmod')
        s.recon = N.RECON[reconstruction]
        self.reconstruction = reconstruction
        self.spec = s
        self.dt = float(dt)
        c = N.ctypes.c_void_p()
        N.check(self._lib.bolt_adj1d_create(N.ctypes.byref(s),
                                            N.F32 if self.dtype == torch.float32 else N.F64,
                                            N.ctypes.byref(c)), 'bolt_adj1d_create')
        self._c = c
        self.forward_steps = 0          # steps advanced by the last gradient (recomputation)

    def __del__(self):
        try:
            if getattr(self, '_c', None) is not None:
                self._lib.bolt_adj1d_destroy(self._c)
                self._c = None
        except Exception:
            pass

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _prep(self, f0):
        f = torch.as_tensor(f0, device=self.device).to(self.dtype).reshape(self.shape)
        return f.contiguous().clone()

    def set_tau(self, tau):
        N.check(self._lib.bolt_adj1d_set_tau(self._c, float(tau)), 'bolt_adj1d_set_tau')

    def _advance(self, f, k, J=None):
        for _ in range(k):
            N.check(self._lib.bolt_adj1d_step(self._c, f.data_ptr(),
                                              0 if J is None else J.data_ptr(), self._stream()),
                    'bolt_adj1d_step')
        self.forward_steps += k
        return f

    def forward(self, f0, tau=None):
        """J and f_N from f0 (the same scheme and precision as the gradient)."""
        if tau is not None:
            self.set_tau(tau)
        f = self._prep(f0)
        J = torch.zeros((), dtype=torch.float64, device=self.device)
        self._advance(f, self.nsteps, J)
        return J, f

    def gradient(self, f0, tau=None):
        """dJ/df0 (shape (N_q1, N_p1)) and dJ/dtau (0-d FP64 tensor)."""
        if tau is not None:
            self.set_tau(tau)
        self.forward_steps = 0
        f = self._prep(f0)
        self._J = torch.zeros((), dtype=torch.float64, device=self.device)
        self._dtau = torch.zeros((), dtype=torch.float64, device=self.device)
        self._lam = None
        self._reverse(0, self.nsteps, f, self.snapshots)
        lam = self._lam if self._lam is not None else torch.zeros_like(f)
        return lam, self._dtau

    # ---- binomial checkpointing -----------------------------------------------------
    def _adjoint_step(self, state, n):
        """Adjoint of step n -> n+1 from the state f_n (a copy is not needed:
        the adjoint only reads it)."""
        if self._lam is None:
            # first visit (the schedule reverses the last step first): lam = dJ/df_N
            fN = self._advance(state.clone(), 1)
            self._lam = torch.zeros_like(state)
            N.check(self._lib.bolt_adj1d_objective(self._c, fN.data_ptr(), self._J.data_ptr(),
                                                   self._lam.data_ptr(), self._stream()),
                    'bolt_adj1d_objective')
        N.check(self._lib.bolt_adj1d_step_adjoint(self._c, state.data_ptr(), self._lam.data_ptr(),
                                                  1 if n >= 1 else 0, self._dtau.data_ptr(),
                                                  self._stream()), 'bolt_adj1d_step_adjoint')

    def _reverse(self, s, e, state_s, c):
        """Adjoint of steps s..e-1 given the state f_s; at most c further
        snapshots may be held."""
        n = e - s
        if n <= 0:
            return
        if n == 1:
            self._adjoint_step(state_s, s)
            return
        if c == 0:
            for k in range(e - 1, s - 1, -1):
                self._adjoint_step(self._advance(state_s.clone(), k - s), k)
            return
        t = 1
        while _beta(c, t) < n:
            t += 1
        m = s + max(1, n - _beta(c - 1, t))
        state_m = self._advance(state_s.clone(), m - s)
        self._reverse(m, e, state_m, c - 1)
        del state_m
        self._reverse(s, m, state_s, c)


class _RolloutFn(torch.autograd.Function):

    @staticmethod
    def forward(ctx, f0, tau, roll):
        ctx.roll = roll
        ctx.save_for_backward(f0, tau)
        J, _ = roll.forward(f0, float(tau))
        return J

    @staticmethod
    def backward(ctx, gJ):
        f0, tau = ctx.saved_tensors
        gf, gtau = ctx.roll.gradient(f0, float(tau))
        gf = gf.to(f0.dtype).reshape(f0.shape) * gJ
        return gf, (gtau * gJ).to(tau.dtype), None


def rollout(f0, tau, roll):
    """J(f0, tau) of the Rollout1D1V problem ``roll`` as a differentiable torch
    scalar (f0: (N_q1, N_p1) tensor, tau: 0-d tensor)."""
    return _RolloutFn.apply(f0, tau, roll)
