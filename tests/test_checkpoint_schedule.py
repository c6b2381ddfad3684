"""Binomial checkpointing of bolt_b200.adjoint.Rollout1D1V on the CPU: the
recursive schedule is driven with a scalar linear recurrence standing in for
the RK4 step (f_{n+1} = a f_n, objective sum_{n>=1} f_n^2), whose gradient
is known in closed form.  Checks the gradient for several step and snapshot
counts, the bound on live snapshots, and the recomputation count against the
binomial bound t N."""

import math

import pytest

from bolt_b200.adjoint import Rollout1D1V, _beta

A = 0.97


class _Toy(Rollout1D1V):
    """Rollout1D1V's schedule with a scalar state: f is a one-element list."""

    def __init__(self, nsteps, snapshots):
        self.nsteps, self.snapshots = nsteps, snapshots
        self.forward_steps = 0

    def _advance(self, f, k, J=None):
        f[0] *= A ** k
        self.forward_steps += k
        return f

    def _adjoint_step(self, state, n):
        if self._lam is None:
            fN = state[0] * A
            self.forward_steps += 1
            self._lam = 2 * fN
        self._lam = A * self._lam + (2 * state[0] if n >= 1 else 0.0)

    def grad(self, f0):
        self._lam = None
        _Copyable.live = _Copyable.max_live = 0
        self._reverse(0, self.nsteps, _Copyable([f0]), self.snapshots)
        return self._lam


class _Copyable(list):
    """A state whose live copies are counted (freed by reference counting)."""
    live = 0
    max_live = 0

    def __init__(self, *a):
        super().__init__(*a)
        _Copyable.live += 1
        _Copyable.max_live = max(_Copyable.max_live, _Copyable.live)

    def __del__(self):
        _Copyable.live -= 1

    def clone(self):
        return _Copyable(self)


def exact_grad(f0, n):
    # J = sum_{k=1..n} (A^k f0)^2 -> dJ/df0 = 2 f0 sum A^{2k}
    return 2 * f0 * sum(A ** (2 * k) for k in range(1, n + 1))


@pytest.mark.parametrize('n,c', [(1, 0), (2, 0), (7, 0), (10, 1), (40, 3), (100, 5),
                                 (2000, 20), (37, 37)])
def test_schedule_gradient_and_costs(n, c):
    toy = _Toy(n, c)
    g = toy.grad(1.3)
    assert g == pytest.approx(exact_grad(1.3, n), rel=1e-12)
    # live states: f0 plus at most c snapshots plus the step being recomputed
    assert _Copyable.max_live <= c + 2
    if c > 0:
        t = 1
        while _beta(c, t) < n:
            t += 1
        assert toy.forward_steps <= t * n + 1


def test_binomial_capacity():
    assert _beta(20, 3) == math.comb(23, 3) == 1771
    assert _beta(20, 4) == 10626
