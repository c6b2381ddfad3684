"""CPU oracle for Bolt's nonlinear finite-volume kinetic update (FP64, numpy).

TEST INFRASTRUCTURE ONLY.  This module is the checker: tests/, the smoke test
and bench.py's CPU-baseline leg may import it; the product path
(bolt_b200.*) never does.

It restates, in its own code, the algorithm of Bolt's FVM path:

  df/dt = -d(C_q1 f)/dq1 - d(C_q2 f)/dq2 + BGK[f] - sum_i d(C_pi f)/dpi

Arrays use the layout of the GPU path (and of Bolt's q-expanded arrays, which
are column-major (Np, Ns, Nq1g, Nq2g)): C-order (Nq2g, Nq1g, Ns, Np3, Np2, Np1)
with ghost zones included along q1 and q2.

Reference files followed (paths within the Bolt project):
  bolt/lib/nonlinear/finite_volume/df_dt_fvm.py:33-339      df_dt
  bolt/lib/nonlinear/finite_volume/reconstruction/weno5.py:4-98
  bolt/lib/nonlinear/finite_volume/reconstruction/minmod.py:4-71
  bolt/lib/nonlinear/finite_volume/reconstruction/ppm.py:4-100
  bolt/lib/nonlinear/finite_volume/riemann.py:8-58          upwind select
  bolt/lib/nonlinear/finite_volume/fvm_operator.py:6-35     RK2 midpoint
  bolt/lib/nonlinear/temporal_evolution/integrators.py:15-28 RK4 stages
  bolt/lib/nonlinear/communicate.py:8-38 + boundaries.py:147-225,415-577 ghosts
  bolt/lib/nonlinear/compute_moments.py:7-59, src/utils/integral_over_v.py:6-7
  bolt/src/nonrelativistic_boltzmann/collision_operator.py:16-128 (f0, BGK)
  bolt/src/nonrelativistic_boltzmann/advection_terms.py:64-97,147-188 (C_q, C_p)
  bolt/src/nonrelativistic_boltzmann/moments.py:6-58
  bolt/lib/nonlinear/fields/fields.py:421-690, electrodynamic/fdtd_explicit.py:9-177,
  electrostatic/fft.py:9-78  (Yee-grid FDTD, cell<->Yee maps, FFT Poisson init)

Pinned against golden fixtures produced by running the unmodified Bolt source
over numpy stand-ins of ArrayFire/PETSc/MPI (tests/golden/make_golden.py) and
against the analytic known-answer tests of Bolt's own unit tests.
"""

import numpy as np

# axis numbers in the (q2, q1, s, p3, p2, p1) layout
AX_Q2, AX_Q1, AX_S, AX_P3, AX_P2, AX_P1 = 0, 1, 2, 3, 4, 5
WENO_EPS = 1e-17          # weno5.py:18
BGK_EPS = 1e-30           # collision_operator.py:106


# ---------------------------------------------------------------------------
# reconstruction: each returns (left_face_value, right_face_value) of every
# cell along `axis`, with circular neighbours like ArrayFire's af.shift.
# ---------------------------------------------------------------------------
def _nb(a, s, axis):
    """a shifted so that out[i] = a[i - s] (af.shift semantics)."""
    return np.roll(a, s, axis=axis)


def recon_weno5(a, axis):
    """Point-value WENO5 of weno5.py:4-98 (y0..y4 = a[i-2..i+2])."""
    y0, y1, y2, y3, y4 = (_nb(a, 2, axis), _nb(a, 1, axis), a,
                          _nb(a, -1, axis), _nb(a, -2, axis))
    eps = WENO_EPS
    b1 = ((4 / 3) * y0 * y0 - (19 / 3) * y0 * y1 + (25 / 3) * y1 * y1
          + (11 / 3) * y0 * y2 - (31 / 3) * y1 * y2 + (10 / 3) * y2 * y2) \
        + eps * (1.0 + np.abs(y0) + np.abs(y1) + np.abs(y2))
    b2 = ((4 / 3) * y1 * y1 - (19 / 3) * y1 * y2 + (25 / 3) * y2 * y2
          + (11 / 3) * y1 * y3 - (31 / 3) * y2 * y3 + (10 / 3) * y3 * y3) \
        + eps * (1.0 + np.abs(y1) + np.abs(y2) + np.abs(y3))
    b3 = ((4 / 3) * y2 * y2 - (19 / 3) * y2 * y3 + (25 / 3) * y3 * y3
          + (11 / 3) * y2 * y4 - (31 / 3) * y3 * y4 + (10 / 3) * y4 * y4) \
        + eps * (1.0 + np.abs(y2) + np.abs(y3) + np.abs(y4))
    w1r = 1 / (16 * b1 * b1); w2r = 5 / (8 * b2 * b2); w3r = 5 / (16 * b3 * b3)
    w1l = 5 / (16 * b1 * b1); w2l = 5 / (8 * b2 * b2); w3l = 1 / (16 * b3 * b3)
    denl = w1l + w2l + w3l
    denr = w1r + w2r + w3r
    u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2
    u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3
    u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4
    u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2
    u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3
    u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4
    left = (w1l * u1l + w2l * u2l + w3l * u3l) / denl
    right = (w1r * u1r + w2r * u2r + w3r * u3r) / denr
    return left, right


def _minmod3(x, y, z):
    """minmod.py:4-16; the sign convention there gives sign(0) = +1."""
    m = np.minimum(np.minimum(np.abs(x), np.abs(y)), np.abs(z))
    sx = 1 - 2 * (x < 0)
    sy = 1 - 2 * (y < 0)
    sz = 1 - 2 * (z < 0)
    return 0.25 * np.abs(sx + sy) * (sx + sz) * m


def recon_minmod(a, axis):
    """MC-limited linear reconstruction, theta = 2 (minmod.py:18-71)."""
    fwd = _nb(a, -1, axis) - a
    bwd = a - _nb(a, 1, axis)
    cen = bwd + fwd
    slope = _minmod3(2 * bwd, 0.5 * cen, 2 * fwd)
    return a - 0.5 * slope, a + 0.5 * slope


def recon_ppm(a, axis):
    """PPM with monotonised slopes and extremum corrections (ppm.py:4-100)."""
    y0, y1, y2, y3, y4 = (_nb(a, 2, axis), _nb(a, 1, axis), a,
                          _nb(a, -1, axis), _nb(a, -2, axis))
    d0 = 2 * (y1 - y0); d1 = 2 * (y2 - y1); d2 = 2 * (y3 - y2); d3 = 2 * (y4 - y3)
    D1 = 0.5 * (y2 - y0); D2 = 0.5 * (y3 - y1); D3 = 0.5 * (y4 - y2)

    def dq(D, da, db):
        zero = (db * da <= 0)
        sgn = (D > 0) * 2 - 1
        return (1 - zero) * sgn * np.minimum(np.abs(D), np.minimum(np.abs(da), np.abs(db)))

    DQ1 = dq(D1, d0, d1); DQ2 = dq(D2, d1, d2); DQ3 = dq(D3, d2, d3)
    left = 0.5 * (y2 + y1) - (DQ2 - DQ1) / 6
    right = 0.5 * (y3 + y2) - (DQ3 - DQ2) / 6
    c1 = ((right - y2) * (y2 - left) <= 0)
    qd = right - left
    qe = 6 * (y2 - 0.5 * (right + left))
    c2 = (qd * (qd - qe) < 0)
    c3 = (qd * (qd + qe) < 0)
    left = left * (1 - c1) + c1 * y2
    right = right * (1 - c1) + c1 * y2
    left = left * (1 - c2) + c2 * (3 * y2 - 2 * right)
    right = right * c2 + (1 - c2) * right * (1 - c3) + (1 - c2) * c3 * (3 * y2 - 2 * left)
    return left, right


def reconstruct(a, axis, method):
    """Dispatch of reconstruct.py:7-51 (WENO5 without the disabling guard)."""
    if method == 'piecewise-constant':
        return a, a
    if method == 'minmod':
        return recon_minmod(a, axis)
    if method == 'ppm':
        return recon_ppm(a, axis)
    if method == 'weno5':
        return recon_weno5(a, axis)
    raise NotImplementedError(method)


def riemann(left_state, right_state, vel, method='upwind-flux'):
    """Face value times velocity -> flux.

    'upwind-flux' follows riemann.py:46-49 (select(vel > 0, left, right)).
    'lax-friedrichs' is the local Lax-Friedrichs flux
    F = 0.5*(C*(fL + fR) - alpha*(fR - fL)), alpha = |C| at the face, which is
    the maximum wavespeed of the two neighbouring cells because C_q1/C_q2 do not
    vary along their own axis and C_pi does not depend on p_i
    (advection_terms.py:94-97,184-188).
    """
    if method in ('upwind-flux', 'upwind'):
        return vel * np.where(vel > 0, left_state, right_state)
    if method in ('lax-friedrichs', 'llf', 'local-lax-friedrichs'):
        alpha = np.abs(vel)
        return 0.5 * (vel * (left_state + right_state) - alpha * (right_state - left_state))
    raise NotImplementedError(method)


# ---------------------------------------------------------------------------
# grids (calculate_q.py:7-41, calculate_p.py:8-57, physical_system.py:176-187)
# ---------------------------------------------------------------------------
class Grid(object):
    def __init__(self, spec):
        s = spec
        self.spec = s
        self.Ng = s['N_ghost']
        self.Nq1, self.Nq2 = s['N_q1'], s['N_q2']
        self.Np1, self.Np2, self.Np3 = s['N_p1'], s['N_p2'], s['N_p3']
        self.Ns = len(s['mass'])
        self.dq1 = (s['q1_end'] - s['q1_start']) / self.Nq1
        self.dq2 = (s['q2_end'] - s['q2_start']) / self.Nq2
        self.Nq1g = self.Nq1 + 2 * self.Ng
        self.Nq2g = self.Nq2 + 2 * self.Ng
        i1 = np.arange(-self.Ng, self.Nq1 + self.Ng)
        i2 = np.arange(-self.Ng, self.Nq2 + self.Ng)
        q1_lb = s['q1_start'] + i1 * self.dq1
        q2_lb = s['q2_start'] + i2 * self.dq2
        # (Nq2g, Nq1g) arrays, broadcastable against the 6-D layout
        self.q1_left = np.broadcast_to(q1_lb[None, :], (self.Nq2g, self.Nq1g))
        self.q2_bot = np.broadcast_to(q2_lb[:, None], (self.Nq2g, self.Nq1g))
        self.q1_center = self.q1_left + 0.5 * self.dq1
        self.q2_center = self.q2_bot + 0.5 * self.dq2
        self.dp1 = np.array([(s['p1_end'][k] - s['p1_start'][k]) / self.Np1 for k in range(self.Ns)])
        self.dp2 = np.array([(s['p2_end'][k] - s['p2_start'][k]) / self.Np2 for k in range(self.Ns)])
        self.dp3 = np.array([(s['p3_end'][k] - s['p3_start'][k]) / self.Np3 for k in range(self.Ns)])
        shp = (self.Ns, self.Np3, self.Np2, self.Np1)
        self.p1c = np.empty(shp); self.p2c = np.empty(shp); self.p3c = np.empty(shp)
        self.p1l = np.empty(shp); self.p2b = np.empty(shp); self.p3b = np.empty(shp)
        for k in range(self.Ns):
            p1 = s['p1_start'][k] + (0.5 + np.arange(self.Np1)) * self.dp1[k]
            p2 = s['p2_start'][k] + (0.5 + np.arange(self.Np2)) * self.dp2[k]
            p3 = s['p3_start'][k] + (0.5 + np.arange(self.Np3)) * self.dp3[k]
            self.p1c[k] = p1[None, None, :]
            self.p2c[k] = p2[None, :, None]
            self.p3c[k] = p3[:, None, None]
            self.p1l[k] = (s['p1_start'][k] + np.arange(self.Np1) * self.dp1[k])[None, None, :]
            self.p2b[k] = (s['p2_start'][k] + np.arange(self.Np2) * self.dp2[k])[None, :, None]
            self.p3b[k] = (s['p3_start'][k] + np.arange(self.Np3) * self.dp3[k])[:, None, None]
        self.mass = np.array(s['mass'], dtype=np.float64)
        self.charge = np.array(s['charge'], dtype=np.float64)
        # 6-D broadcast helpers
        self.q1c6 = self.q1_center[:, :, None, None, None, None]
        self.q2c6 = self.q2_center[:, :, None, None, None, None]
        self.measure = (self.dp3 * self.dp2 * self.dp1)[None, None, :]  # (1,1,Ns)
        # p-space grid (compute_moments.py:42-56): on 'polar2D' every moment is
        # scaled by params.initial_mu
        self.polar2d = s.get('p_space_grid', 'cartesian') == 'polar2D'
        self.initial_mu = float(s.get('initial_mu', 1.0))

    @property
    def fshape(self):
        return (self.Nq2g, self.Nq1g, self.Ns, self.Np3, self.Np2, self.Np1)

    def interior(self, a):
        g = self.Ng
        return a[g:a.shape[0] - g if g else None, g:a.shape[1] - g if g else None]


# ---------------------------------------------------------------------------
# moments (compute_moments.py:7-59; moments.py:6-58) -> (Nq2g, Nq1g, Ns)
# ---------------------------------------------------------------------------
def moment(grid, f, name):
    g = grid
    v1, v2, v3 = g.p1c[None, None], g.p2c[None, None], g.p3c[None, None]
    if name == 'density':
        integrand = f
    elif name == 'mom_v1_bulk':
        integrand = f * v1
    elif name == 'mom_v2_bulk':
        integrand = f * v2
    elif name == 'mom_v3_bulk':
        integrand = f * v3
    elif name == 'energy':
        integrand = 0.5 * f * (v1 ** 2 + v2 ** 2 + v3 ** 2)
    elif name == 'energy_q1':
        integrand = 0.5 * f * v1 ** 2
    elif name == 'energy_q2':
        integrand = 0.5 * f * v2 ** 2
    elif name == 'energy_q3':
        integrand = 0.5 * f * v3 ** 2
    elif name in ('q_q1', 'q_q2', 'q_q3'):
        vv = {'q_q1': v1, 'q_q2': v2, 'q_q3': v3}[name]
        integrand = f * vv * (v1 ** 2 + v2 ** 2 + v3 ** 2)
    else:
        raise KeyError(name)
    s = integrand.reshape(integrand.shape[:3] + (-1,)).sum(axis=3)
    if g.polar2d:
        return g.initial_mu * (s * g.measure)
    return s * g.measure


# ---------------------------------------------------------------------------
# BGK source (collision_operator.py:16-128)
# ---------------------------------------------------------------------------
def maxwell_params(grid, f):
    """n, bulk velocities and temperature per (q2, q1, s)."""
    g = grid
    m = g.mass[None, None, :]
    n = moment(g, f, 'density')
    eps = BGK_EPS
    u1 = moment(g, f, 'mom_v1_bulk') / (n + eps)
    u2 = moment(g, f, 'mom_v2_bulk') / (n + eps)
    u3 = moment(g, f, 'mom_v3_bulk') / (n + eps)
    E = moment(g, f, 'energy')
    T = (1 / g.spec['p_dim']) * (2 * (E * m) - (n * m) * u1 ** 2 - (n * m) * u2 ** 2
                                 - (n * m) * u3 ** 2) / (n + eps) + eps
    return n, u1, u2, u3, T


def f_maxwellian(grid, n, u1, u2, u3, T):
    g = grid
    k = g.spec['boltzmann_constant']
    m = g.mass[None, None, :, None, None, None]
    ex = lambda a: a[:, :, :, None, None, None]
    n6, u16, u26, u36, T6 = ex(n), ex(u1), ex(u2), ex(u3), ex(T)
    v1, v2, v3 = g.p1c[None, None], g.p2c[None, None], g.p3c[None, None]
    pd = g.spec['p_dim']
    e1 = np.exp(-m * (v1 - u16) ** 2 / (2 * k * T6))
    if pd == 3:
        e2 = np.exp(-m * (v2 - u26) ** 2 / (2 * k * T6))
        e3 = np.exp(-m * (v3 - u36) ** 2 / (2 * k * T6))
        return n6 * (m / (2 * np.pi * k * T6)) ** (3 / 2) * e1 * e2 * e3
    if pd == 2:
        e2 = np.exp(-m * (v2 - u26) ** 2 / (2 * k * T6))
        return n6 * (m / (2 * np.pi * k * T6)) * e1 * e2
    return n6 * np.sqrt(m / (2 * np.pi * k * T6)) * e1


def bgk(grid, f, tau):
    n, u1, u2, u3, T = maxwell_params(grid, f)
    fMB = f_maxwellian(grid, n, u1, u2, u3, T)
    return -(f - fMB) / tau


# ---------------------------------------------------------------------------
# fields (fields.py, fdtd_explicit.py, fft.py). Field arrays: (6, Nq2g, Nq1g)
# ---------------------------------------------------------------------------
def _sh(a, s1, s2):
    """af.shift(a, 0, 0, s1, s2) on (..., Nq2g, Nq1g) arrays."""
    out = a
    if s1:
        out = np.roll(out, s1, axis=-1)
    if s2:
        out = np.roll(out, s2, axis=-2)
    return out


def _periodic_fill(grid, a):
    """Ghost refresh of a (..., Nq2g, Nq1g) field array (communicate_fields)."""
    g = grid
    Ng = g.Ng
    out = a.copy()
    if Ng == 0:
        return out
    per1 = g.spec['bc_q1'] == 'periodic'
    per2 = g.spec['bc_q2'] == 'periodic'
    N1, N2 = g.Nq1, g.Nq2
    idx1 = np.arange(-Ng, N1 + Ng)
    idx2 = np.arange(-Ng, N2 + Ng)
    for jj, j in enumerate(idx2):
        for ii, i in enumerate(idx1):
            inside1 = 0 <= i < N1
            inside2 = 0 <= j < N2
            if inside1 and inside2:
                continue
            if (not inside1 and not per1) or (not inside2 and not per2):
                continue
            out[..., jj, ii] = a[..., Ng + (j % N2), Ng + (i % N1)]
    return out


class FieldState(object):
    """Electrodynamic fields as the reference holds them after fields_solver
    construction: a Yee-grid array and ONE cell-centred array.  In the
    reference the names cell_centered_EM_fields, ..._at_n and
    ..._at_n_plus_half are bound to the same af.Array object
    (fields.py:493-494) and are only ever updated in place afterwards, so all
    three always hold the same values; get_fields therefore returns that array
    whichever time level its toggle selects (fields.py:649-690)."""

    def __init__(self, grid, rho_total, user=None):
        """``user``: the initialize module's field functions by name
        (initialize_E / initialize_A_phi, initialize_B / initialize_A /
        initialize_A3_B3) as numpy callables of (q1, q2, params)."""
        self.g = grid
        sp = grid.spec
        self.eps = sp.get('eps', 1.0)
        self.mu = sp.get('mu', 1.0)
        Nq2g, Nq1g = grid.Nq2g, grid.Nq1g
        self.cell = np.zeros((6, Nq2g, Nq1g))
        self.yee = np.zeros((6, Nq2g, Nq1g))
        # a q-block: fills the Yee ghosts of its external axes from the
        # neighbouring blocks after every periodic halo refresh of the update
        self.exchange = None
        init = sp.get('fields_initialize', 'fft')
        user = user or {}
        if init == 'user-defined':
            # fields.py:472-475: Yee E and B from the user's functions, then
            # every cell-centred field from the (not yet refreshed) Yee grid
            self.yee[0:3] = self._user_E(user)
            self.yee[3:6] = self._user_B(user)
            self.cell = self._yee_to_cell()
            self.yee = _periodic_fill(grid, self.yee)
            self.J = None
            return
        if init not in ('fft', 'fft + user-defined magnetic fields'):
            raise NotImplementedError(init)
        self._fft_poisson(rho_total)
        self.cell = _periodic_fill(grid, self.cell)
        self._cell_to_yee_E()
        if init != 'fft':
            # fields.py:477-482: user B on the Yee grid, then its cell values
            self.yee[3:6] = self._user_B(user)
            self.cell[3:6] = self._yee_to_cell()[3:6]
        # the constructor's constraint check calls compute_divE, which
        # refreshes the Yee-grid halos (fields.py:37, 278)
        self.yee = _periodic_fill(grid, self.yee)
        self.J = None

    def _user_E(self, user):
        """fields.py:280-337: E1 on the 'left-centre' grid, E2 at (centre,
        bottom), E3 at the centre; or from A and phi by one-sided differences.
        The reference's left-centre grid is (q1 left, q2 BOTTOM):
        calculate_q.py:35-38 pairs q1_left_center with q2_center_bot."""
        g, dq1, dq2 = self.g, self.g.dq1, self.g.dq2
        q1l, q2b, q1c, q2c = g.q1_left, g.q2_bot, g.q1_center, g.q2_center
        if 'initialize_E' in user:
            E = user['initialize_E']
            return np.stack([E(q1l, q2b, None)[0], E(q1c, q2b, None)[1], E(q1c, q2c, None)[2]])
        if 'initialize_A_phi' in user:
            F = user['initialize_A_phi']
            A1, A2 = F(q1c, q2b, None)[0], F(q1l, q2b, None)[1]
            A3, phi = F(q1l, q2b, None)[2], F(q1c, q2c, None)[3]
            dA3_dq2 = (_sh(A3, 0, -1) - A3) / dq2
            dA3_dq1 = (_sh(A3, -1, 0) - A3) / dq1
            dA2_dq1 = (_sh(A2, -1, 0) - A2) / dq1
            dA1_dq2 = (_sh(A1, 0, -1) - A1) / dq2
            dphi_dq1 = -(_sh(phi, 1, 0) - phi) / dq1
            dphi_dq2 = -(_sh(phi, 0, 1) - phi) / dq2
            return np.stack([dA3_dq2 - dphi_dq1, -dA3_dq1 - dphi_dq2, dA2_dq1 - dA1_dq2])
        raise NotImplementedError('initial electric fields')

    def _user_B(self, user):
        """fields.py:339-410: B1 at (centre, bottom), B2 on the 'left-centre'
        grid (q1 left, q2 bottom, as above), B3 at (left, bottom); or from A,
        or from A3 and B3."""
        g, dq1, dq2 = self.g, self.g.dq1, self.g.dq2
        q1l, q2b, q1c, q2c = g.q1_left, g.q2_bot, g.q1_center, g.q2_center
        if 'initialize_B' in user and 'initialize_A3_B3' in user:
            raise ValueError('initialize_B and initialize_A3_B3 together')
        if 'initialize_B' in user:
            B = user['initialize_B']
            return np.stack([B(q1c, q2b, None)[0], B(q1l, q2b, None)[1], B(q1l, q2b, None)[2]])
        if 'initialize_A' in user:
            F = user['initialize_A']
            A1, A2, A3 = F(q1l, q2b, None)[0], F(q1c, q2b, None)[1], F(q1c, q2c, None)[2]
            B1 = (_sh(A3, 0, -1) - A3) / dq2
            B2 = -(_sh(A3, -1, 0) - A3) / dq1
            B3 = (_sh(A2, -1, 0) - A2) / dq1 - (_sh(A1, 0, -1) - A1) / dq2
            return np.stack([B1, B2, B3])
        if 'initialize_A3_B3' in user:
            F = user['initialize_A3_B3']
            A3 = F(q1c, q2c, None)[0]
            # backward differences (np.roll by +1 along q2 and q1)
            B1 = (A3 - _sh(A3, 0, 1)) / dq2
            B2 = -(A3 - _sh(A3, 1, 0)) / dq1
            return np.stack([B1, B2, F(q1l, q2b, None)[1]])
        raise NotImplementedError('initial magnetic fields')

    def _fft_poisson(self, rho):
        """fft.py:9-78 (serial). rho: (Nq2g, Nq1g) total charge density."""
        g = self.g
        Ng = g.Ng
        r = g.interior(rho).T  # (Nq1, Nq2), as af.reorder(rho, 2,3,0,1)
        k1 = np.fft.fftfreq(r.shape[0], g.dq1)
        k2 = np.fft.fftfreq(r.shape[1], g.dq2)
        k2, k1 = np.meshgrid(k2, k1)
        r = r - r.mean()
        rh = np.fft.fft2(r)
        with np.errstate(divide='ignore', invalid='ignore'):
            ph = rh / (4 * np.pi ** 2 * (k1 ** 2 + k2 ** 2))
        ph[0, 0] = 0
        E1h = -1j * 2 * np.pi * k1 * ph
        E2h = -1j * 2 * np.pi * k2 * ph
        N = E1h.shape[0] * E1h.shape[1]
        E1 = np.real(np.fft.ifft2(E1h) * N / N)
        E2 = np.real(np.fft.ifft2(E2h) * N / N)
        sl = (slice(Ng, g.Nq2g - Ng), slice(Ng, g.Nq1g - Ng))
        self.cell[0][sl] = E1.T / self.eps
        self.cell[1][sl] = E2.T / self.eps

    def _cell_to_yee_E(self):
        """fields.py:511-514."""
        c = self.cell
        self.yee[0] = 0.5 * (c[0] + _sh(c[0], 1, 0))
        self.yee[1] = 0.5 * (c[1] + _sh(c[1], 0, 1))
        self.yee[2] = c[2]

    def _yee_to_cell(self):
        """fields.py:527-557 (both E and B)."""
        y = self.yee
        out = np.empty_like(self.cell)
        out[0] = 0.5 * (y[0] + _sh(y[0], -1, 0))
        out[1] = 0.5 * (y[1] + _sh(y[1], 0, -1))
        out[2] = y[2]
        out[3] = 0.5 * (y[3] + _sh(y[3], 0, -1))
        out[4] = 0.5 * (y[4] + _sh(y[4], -1, 0))
        out[5] = 0.25 * (y[5] + _sh(y[5], 0, -1) + _sh(y[5], -1, 0) + _sh(y[5], -1, -1))
        return out

    def _halo(self, y):
        """communicate_fields (communicate.py:40-77): the periodic refresh,
        then, for a block, its external ghosts from the neighbours."""
        y = _periodic_fill(self.g, y)
        return self.exchange(y) if self.exchange is not None else y

    def evolve(self, J1, J2, J3, dt):
        """evolve_electrodynamic_fields (fields.py:568-647) with the aliasing of
        the three cell-centred names taken into account: the result is
        cell[:3] = 0.5*(E_before + E_after), cell[3:] = B_after."""
        E_before = self.cell[:3].copy()
        # fdtd (fdtd_explicit.py:141-177)
        y = self._halo(self.yee)
        eps, mu = self.eps, self.mu
        dq1, dq2 = self.g.dq1, self.g.dq2
        B1, B2, B3 = y[3], y[4], y[5]
        curlB_1 = (_sh(B3, 0, -1) - B3) / dq2
        curlB_2 = -(_sh(B3, -1, 0) - B3) / dq1
        curlB_3 = (_sh(B2, -1, 0) - B2) / dq1 - (_sh(B1, 0, -1) - B1) / dq2
        y[0] = y[0] + ((dt / (mu * eps)) * curlB_1 - J1 * dt / eps)
        y[1] = y[1] + ((dt / (mu * eps)) * curlB_2 - J2 * dt / eps)
        y[2] = y[2] + ((dt / (mu * eps)) * curlB_3 - J3 * dt / eps)
        y = self._halo(y)
        E1, E2, E3 = y[0], y[1], y[2]
        curlE_1 = (E3 - _sh(E3, 0, 1)) / dq2
        curlE_2 = -(E3 - _sh(E3, 1, 0)) / dq1
        curlE_3 = (E2 - _sh(E2, 1, 0)) / dq1 - (E1 - _sh(E1, 0, 1)) / dq2
        y[3] = y[3] + -dt * curlE_1
        y[4] = y[4] + -dt * curlE_2
        y[5] = y[5] + -dt * curlE_3
        self.yee = y
        cell = self._yee_to_cell()
        cell[:3] = 0.5 * (E_before + cell[:3])
        self.cell = cell


def initial_rho(grid, f):
    """charge * density summed over species (nonlinear_solver.py:494-496,
    fields.py:276)."""
    return (moment(grid, f, 'density') * grid.charge[None, None, :]).sum(axis=2)


# ---------------------------------------------------------------------------
# df/dt (df_dt_fvm.py:33-339)
# ---------------------------------------------------------------------------
class Oracle(object):
    """Holds grid, tau, optional fields, and evaluates df/dt and RK steps the
    way Bolt's nonlinear_solver does for the FVM path."""

    def __init__(self, spec, f0, tau=None, field_functions=None):
        self.spec = spec
        self.g = Grid(spec)
        self.f = np.array(f0, dtype=np.float64).reshape(self.g.fshape)
        self.tau = spec.get('tau', 1.0) if tau is None else tau
        # an 'external' axis: called on every stage input before its halo
        # refresh, to fill the ghost rows / columns from the neighbouring blocks
        self.exchange = None
        self.time_elapsed = 0.0
        self.fields = None
        self.dirichlet = {}
        if spec.get('fields_enabled', False):
            rho = initial_rho(self.g, self.f)
            self.fields = FieldState(self.g, rho, field_functions)
            self.at_n = True

    # ghost refresh: communicate_f + apply_bcs_f -----------------------------
    def refresh(self, f):
        g = self.g
        sp = self.spec
        Ng = g.Ng
        if Ng == 0:
            return f
        out = np.zeros_like(f)
        sl = (slice(Ng, g.Nq2g - Ng), slice(Ng, g.Nq1g - Ng))
        out[sl] = f[sl]
        # periodic wrap for periodic axes (DMDA globalToLocal); ghosts on
        # 'ghosted' axes hold the local buffer's contents, which stay zero
        # (a shearing-box axis is periodic in the DMDA, nonlinear_solver.py:186-194)
        per1 = sp['bc_q1'] in ('periodic', 'shearing-box')
        per2 = sp['bc_q2'] in ('periodic', 'shearing-box')
        i1 = np.arange(-Ng, g.Nq1 + Ng)
        i2 = np.arange(-Ng, g.Nq2 + Ng)
        src1 = np.where((i1 >= 0) & (i1 < g.Nq1), i1, i1 % g.Nq1)
        src2 = np.where((i2 >= 0) & (i2 < g.Nq2), i2, i2 % g.Nq2)
        ok1 = per1 | ((i1 >= 0) & (i1 < g.Nq1))
        ok2 = per2 | ((i2 >= 0) & (i2 < g.Nq2))
        inner = f[sl]
        filled = inner[src2][:, src1]
        mask = ok2[:, None] & ok1[None, :]
        out[mask] = filled[mask]
        if sp['bc_q2'] == 'external':
            # a q2 slab: its ghost rows were supplied by the neighbouring slabs
            out[:Ng] = f[:Ng]
            out[g.Nq2g - Ng:] = f[g.Nq2g - Ng:]
        if sp['bc_q1'] == 'external':
            # a q1 block: its ghost columns were supplied by the neighbours
            out[:, :Ng] = f[:, :Ng]
            out[:, g.Nq1g - Ng:] = f[:, g.Nq1g - Ng:]
        # apply_bcs_f (boundaries.py:415-577): side by side in the order left,
        # right, bottom, top, the mirror image (boundaries.py:226-301) and/or
        # the Dirichlet inflow values (boundaries.py:147-225)
        for side in ('left', 'right', 'bottom', 'top'):
            axis_bc = sp['bc_q1'] if side in ('left', 'right') else sp['bc_q2']
            if axis_bc == 'shearing-box':
                self._shear_strip(out, side)
                continue
            if axis_bc in ('mirror', 'mirror+dirichlet'):
                # ghost cells take the interior cells mirrored across the edge,
                # with the p-index normal to the edge reversed (p1 for q1 edges,
                # p2 for q2 edges; axes -1 / -2 of (q2, q1, s, p3, p2, p1));
                # on the polar2D grid the q2 edges are the same (theta -> -theta)
                if side in ('left', 'right') and g.polar2d:
                    # polar2D (boundaries.py:313-413), p2 the angle: a q1 edge
                    # maps theta -> pi - theta, each half of the p2 range
                    # reversed on its own (N_p2 // 2 cells in the first half)
                    H = g.Np2 // 2
                    k = np.arange(g.Np2)
                    perm = np.where(k < H, H - 1 - k, g.Np2 - 1 + H - k)
                    if side == 'left':
                        out[:, :Ng] = out[:, Ng:2 * Ng][:, ::-1][..., perm, :]
                    else:
                        out[:, -Ng:] = out[:, -2 * Ng:-Ng][:, ::-1][..., perm, :]
                elif side == 'left':
                    out[:, :Ng] = out[:, Ng:2 * Ng][:, ::-1][..., ::-1]
                elif side == 'right':
                    out[:, -Ng:] = out[:, -2 * Ng:-Ng][:, ::-1][..., ::-1]
                elif side == 'bottom':
                    out[:Ng] = out[Ng:2 * Ng][::-1][..., ::-1, :]
                else:
                    out[-Ng:] = out[-2 * Ng:-Ng][::-1][..., ::-1, :]
            if axis_bc not in ('dirichlet', 'mirror+dirichlet'):
                continue
            # Dirichlet inflow: ghost = user value where the q-velocity points
            # into the domain, else keep
            val = self.dirichlet[side]          # full f-shaped array
            v = g.p1c if side in ('left', 'right') else g.p2c
            v = np.broadcast_to(v[None, None], out.shape)
            if side == 'left':
                sel = np.where(v > 0, val, out)
                out[:, :Ng] = sel[:, :Ng]
            elif side == 'right':
                sel = np.where(v < 0, val, out)
                out[:, -Ng:] = sel[:, -Ng:]
            elif side == 'bottom':
                sel = np.where(v > 0, val, out)
                out[:Ng] = sel[:Ng]
            else:
                sel = np.where(v < 0, val, out)
                out[-Ng:] = sel[-Ng:]
        return out

    def _shear_strip(self, out, side):
        """Shearing-box ghost strip (boundaries.py:6-145): the strip of N_g
        ghost columns (left/right) or rows (bottom/top), already filled
        periodically, resampled along the other q axis at the positions
        sheared by -/+ q omega L t (L the length of the strip's own axis,
        t = time_elapsed), wrapped into the domain.  The reference resamples
        with ArrayFire's approx2(BICUBIC_SPLINE); at the strip's own grid
        positions that is the one-dimensional Catmull-Rom cubic (Catmull and
        Rom 1974: the cubic Hermite segment whose end tangents are the
        centred differences (p_{k+1} - p_{k-1})/2) along the sheared axis,
        which is what this evaluates.  The shift is first reduced modulo the
        period with the exact fmod, so the wrap below takes at most two steps
        (the reference subtracts the period repeatedly; the two agree to
        rounding)."""
        g, sp, Ng = self.g, self.spec, self.g.Ng
        shear = sp['shear_q'] * sp['shear_omega'] * self.time_elapsed
        if side in ('left', 'right'):
            lo, hi, N, d = sp['q2_start'], sp['q2_end'], g.Nq2, g.dq2
            shift = shear * (sp['q1_end'] - sp['q1_start'])
            centres = g.q2_center[:, 0]                     # ghosted q2 centres
            strip = (slice(None), slice(0, Ng)) if side == 'left' \
                else (slice(None), slice(g.Nq1g - Ng, g.Nq1g))
            axis = 0
        else:
            lo, hi, N, d = sp['q1_start'], sp['q1_end'], g.Nq1, g.dq1
            shift = shear * (sp['q2_end'] - sp['q2_start'])
            centres = g.q1_center[0, :]
            strip = (slice(0, Ng), slice(None)) if side == 'bottom' \
                else (slice(g.Nq2g - Ng, g.Nq2g), slice(None))
            axis = 1
        L = hi - lo
        shift = np.fmod(shift, L)
        pos = centres - shift if side in ('left', 'bottom') else centres + shift
        while np.any(pos > hi):
            pos = np.where(pos > hi, pos - L, pos)
        while np.any(pos < lo):
            pos = np.where(pos < lo, pos + L, pos)
        x = (pos - centres[0]) / d                          # index in the ghosted strip
        j = np.floor(x).astype(int)
        t = x - j
        assert j.min() - 1 >= 0 and j.max() + 2 <= N + 2 * Ng - 1
        data = out[strip].copy()
        take = lambda k: np.take(data, j + k, axis=axis)
        p0, p1, p2, p3 = take(-1), take(0), take(1), take(2)
        shp = [1] * data.ndim
        shp[axis] = -1
        t = t.reshape(shp)
        val = p1 + 0.5 * t * ((p2 - p0) + t * ((2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3)
                                             + t * (3.0 * (p1 - p2) + p3 - p0)))
        out[strip] = val

    # -----------------------------------------------------------------------
    def dfdt(self, f, evolve_fields=None, term='all'):
        g = self.g
        sp = self.spec
        rq, rp = sp['recon_q'], sp['recon_p']
        fq, fp = sp.get('riemann_q', 'upwind-flux'), sp.get('riemann_p', 'upwind-flux')
        v1 = np.broadcast_to(g.p1c[None, None], f.shape)
        v2 = np.broadcast_to(g.p2c[None, None], f.shape)
        df = 0.0
        # q-space (df_dt_fvm.py:56-97), with the source: only for the FVM in q
        # (the semi-Lagrangian q-step advects and collides by itself)
        if sp.get('solver_q', 'FVM') == 'FVM':
            lp, rm = reconstruct(f, AX_Q1, rq)
            bp, tm = reconstruct(f, AX_Q2, rq)
            lm = _nb(rm, 1, AX_Q1)
            bm = _nb(tm, 1, AX_Q2)
            left_flux = riemann(lm, lp, v1, fq)
            bot_flux = riemann(bm, bp, v2, fq)
            right_flux = _nb(left_flux, -1, AX_Q1)
            top_flux = _nb(bot_flux, -1, AX_Q2)
            df = df - (right_flux - left_flux) / g.dq1 - (top_flux - bot_flux) / g.dq2
            if sp.get('source_enabled', False):
                df = df + bgk(g, f, self.tau)
        # p-space (df_dt_fvm.py:99-323)
        if sp.get('fields_enabled', False):
            fs = self.fields
            if evolve_fields is None:
                evolve_fields = not self.at_n
            if sp.get('fields_type', 'electrodynamic') == 'electrostatic':
                # df_dt_fvm.py:234-242 + fields.py:559-566: the fields of this
                # df/dt argument from its charge density, by the FFT solve,
                # then the periodic halo refresh
                evolve_fields = False
                fs._fft_poisson(initial_rho(g, f))
                fs.cell = _periodic_fill(g, fs.cell)
            if evolve_fields:
                f_left = np.where(v1 > 0, lm, lp)
                f_bot = np.where(v2 > 0, bm, bp)
                q = g.charge[None, None, :]
                J1 = (q * moment(g, f_left, 'mom_v1_bulk')).sum(axis=2)
                J2 = (q * moment(g, f_bot, 'mom_v2_bulk')).sum(axis=2)
                J3 = (q * moment(g, f, 'mom_v3_bulk')).sum(axis=2)
                fs.evolve(J1, J2, J3, self.dt)
            # three get_fields calls toggle at_n (fields.py:685-688)
            self.at_n = not self.at_n
            E1, E2, E3, B1, B2, B3 = [c[:, :, None, None, None, None] for c in fs.cell]
            em = (g.charge / g.mass)[None, None, :, None, None, None]
            # C_p at p-faces: p1_left with p2,p3 centred, etc.
            P1l, P2c, P3c = g.p1l[None, None], g.p2c[None, None], g.p3c[None, None]
            P1c, P2b, P3b = g.p1c[None, None], g.p2b[None, None], g.p3b[None, None]
            C1 = em * (E1 + P2c * B3 - P3c * B2)
            C2 = em * (E2 + P3c * B1 - P1c * B3)
            C3 = em * (E3 + P1c * B2 - P2c * B1)
            C1 = np.broadcast_to(C1, f.shape)
            C2 = np.broadcast_to(C2, f.shape)
            C3 = np.broadcast_to(C3, f.shape)
            l1, r1 = reconstruct(f, AX_P1, rp)
            l2, r2 = reconstruct(f, AX_P2, rp)
            l3, r3 = reconstruct(f, AX_P3, rp)
            m1 = _nb(r1, 1, AX_P1)
            m2 = _nb(r2, 1, AX_P2)
            m3 = _nb(r3, 1, AX_P3)
            F1 = riemann(m1, l1, C1, fp)
            F2 = riemann(m2, l2, C2, fp)
            F3 = riemann(m3, l3, C3, fp)
            dp1 = g.dp1[None, None, :, None, None, None]
            dp2 = g.dp2[None, None, :, None, None, None]
            dp3 = g.dp3[None, None, :, None, None, None]
            d1 = (_nb(F1, -1, AX_P1) - F1) * (1 / dp1)
            d2 = (_nb(F2, -1, AX_P2) - F2) * (1 / dp2)
            d3 = (_nb(F3, -1, AX_P3) - F3) * (1 / dp3)
            if term == 'd_flux_p1_dp1':
                return d1
            if term == 'd_flux_p2_dp2':
                return d2
            if term == 'd_flux_p3_dp3':
                return d3
            df = df - (d1 + d2 + d3)
        return np.broadcast_to(df, f.shape).copy() if np.ndim(df) else np.zeros_like(f)

    # time stepping ---------------------------------------------------------
    def step(self, dt):
        """One strang_timestep with the FVM in q and p (timestep.py:101-160)."""
        self.fvm_step(dt)
        if np.any(np.isinf(self.f)) or np.any(np.isnan(self.f)):
            raise SystemExit('Solver Diverging!')
        self.time_elapsed += dt

    def fvm_step(self, dt):
        """op_fvm (fvm_operator.py:37-50): the RK step of df_dt_fvm."""
        self.dt = dt
        integ = self.spec.get('integrator', 'RK2')

        def refresh(x):
            return self.refresh(self.exchange(x) if self.exchange else x)
        if integ == 'RK2':
            # fvm_operator.py:6-35
            self.f = refresh(self.f)
            f_initial = self.f
            self.f = self.f + self.dfdt(self.f) * (dt / 2)
            self.f = refresh(self.f)
            self.f = f_initial + self.dfdt(self.f) * dt
        elif integ == 'RK4':
            # integrators.py:15-28 with the refresh of fvm_operator.py before
            # every stage; electrodynamic fields advance once per step, in the
            # stage whose input is the first midpoint state (stage 2), with
            # the currents of that state.
            fe = self.fields is not None
            self.f = refresh(self.f)
            f_initial = self.f
            k1 = self.dfdt(self.f, evolve_fields=False if fe else None)
            x = refresh(f_initial + 0.5 * k1 * dt)
            k2 = self.dfdt(x, evolve_fields=True if fe else None)
            x = refresh(f_initial + 0.5 * k2 * dt)
            k3 = self.dfdt(x, evolve_fields=False if fe else None)
            x = refresh(f_initial + k3 * dt)
            k4 = self.dfdt(x, evolve_fields=False if fe else None)
            self.f = f_initial + ((k1 + 2 * k2 + 2 * k3 + k4) / 6) * dt
        else:
            raise NotImplementedError(integ)

    def moments(self, name, f=None):
        return moment(self.g, self.f if f is None else f, name)

    # advective semi-Lagrangian in q (asl_operators.py:20-83) --------------------
    def asl_advect_q(self, dt):
        """op_advect_q: ghost refresh, then every cell's value taken at the foot
        of its characteristic, q - A_q dt with A_q = (p1, p2)
        (advection_terms.py:29-61), by bicubic interpolation over the ghosted
        q-plane (interpolation_routines.py:9-56)."""
        g = self.g
        f = self.refresh(self.exchange(self.f) if self.exchange else self.f)
        q1c = g.q1_center[0]                     # (Nq1g,)
        q2c = g.q2_center[:, 0]                  # (Nq2g,)
        v1 = g.p1c[None, None]                   # (1, 1, Ns, Np3, Np2, Np1)
        v2 = g.p2c[None, None]
        x = ((q1c[None, :, None, None, None, None] - v1 * dt) - q1c[0]) / (q1c[1] - q1c[0])
        if g.Nq2g > 1:
            y = ((q2c[:, None, None, None, None, None] - v2 * dt) - q2c[0]) / (q2c[1] - q2c[0])
        else:
            y = np.zeros((1, 1) + v2.shape[2:]) + 0.0 * v2
        self.f = interp2_catmull_rom(f, x, y)

    def asl_source(self, dt):
        """op_solve_src (asl_operators.py:40-83): f <- f_MB where collisions are
        instantaneous, else one RK2 step (integrators.py:6-13) of the BGK
        source when the source is enabled."""
        g = self.g
        if self.spec.get('instantaneous', False):
            n, u1, u2, u3, T = maxwell_params(g, self.f)
            self.f = f_maxwellian(g, n, u1, u2, u3, T)
        elif self.spec.get('source_enabled', True):
            x = self.f + bgk(g, self.f, self.tau) * (dt / 2)
            self.f = self.f + bgk(g, x, self.tau) * dt

    def split_step(self, dt, scheme=None):
        """One timestep of ASL in q: the splitting of op_advect_q and
        op_solve_src named by ``scheme`` (timestep.py:39-240,
        operator_splitting_methods.py); with (electrostatic) fields that pair,
        split by the same scheme, is itself split with op_fvm, the FVM in p
        (Strang and Lie only here)."""
        scheme = scheme or self.spec.get('splitting', 'strang')
        op1, op2 = self.asl_advect_q, self.asl_source
        if self.fields is not None:
            if scheme not in ('strang', 'lie'):
                raise NotImplementedError('ASL with fields: Strang or Lie splitting')

            adv, src = op1, op2

            def pair(d):
                if scheme == 'strang':
                    adv(0.5 * d)
                    src(d)
                    adv(0.5 * d)
                else:
                    adv(d)
                    src(d)
            op1, op2 = pair, self.fvm_step

        def strang(a, b):
            a(0.5 * dt)
            b(dt)
            a(0.5 * dt)

        def swss(a, b):
            f_start = self.f
            a(dt)
            b(dt)
            f_mid = self.f
            self.f = f_start
            b(dt)
            a(dt)
            self.f = 0.5 * (self.f + f_mid)

        if scheme == 'strang':
            strang(op1, op2)
        elif scheme == 'lie':
            op1(dt)
            op2(dt)
        elif scheme == 'swss':
            swss(op1, op2)
        elif scheme == 'jia':
            f_start = self.f
            strang(op1, op2)
            f1 = self.f
            self.f = f_start
            strang(op2, op1)
            f2 = self.f
            self.f = f_start
            swss(op1, op2)
            self.f = (2 / 3) * (f1 + f2) - (1 / 3) * self.f
        else:
            raise NotImplementedError(scheme)
        if np.any(np.isinf(self.f)) or np.any(np.isnan(self.f)):
            raise SystemExit('Solver Diverging!')
        self.time_elapsed += dt


def catmull_rom(t):
    """Weights of the Catmull-Rom cubic through samples at -1, 0, 1, 2 for a
    point t in [0, 1) past sample 0 (Catmull and Rom 1974)."""
    t2, t3 = t * t, t * t * t
    return (0.5 * (-t + 2 * t2 - t3), 0.5 * (2 - 5 * t2 + 3 * t3),
            0.5 * (t + 4 * t2 - 3 * t3), 0.5 * (t3 - t2))


def interp2_catmull_rom(a, x, y):
    """a (Nq2g, Nq1g, ...) at q1 index positions x and q2 index positions y
    (broadcast against a): the tensor product of Catmull-Rom cubics, the
    neighbouring samples clamped to the array, 0 where a position lies
    outside [0, n - 1] -- the restatement of ArrayFire's approx2 with
    BICUBIC_SPLINE that the semi-Lagrangian step calls (ArrayFire itself,
    a third-party library, is absent: parity of this interpolation is
    unpinned beyond its own restatement)."""
    n2, n1 = a.shape[0], a.shape[1]
    shape = np.broadcast_shapes(a.shape, np.shape(x), np.shape(y))
    x = np.broadcast_to(x, shape)
    y = np.broadcast_to(y, shape)
    off = (x < 0) | (x > n1 - 1) | (y < 0) | (y > n2 - 1)
    xs, ys = np.clip(x, 0, n1 - 1), np.clip(y, 0, n2 - 1)
    i0 = np.floor(xs).astype(np.int64)
    j0 = np.floor(ys).astype(np.int64)
    wx, wy = catmull_rom(xs - i0), catmull_rom(ys - j0)
    idx = np.indices(shape[2:])
    out = np.zeros(shape)
    for b in range(4):
        jj = np.clip(j0 - 1 + b, 0, n2 - 1)
        row = np.zeros(shape)
        for c in range(4):
            ii = np.clip(i0 - 1 + c, 0, n1 - 1)
            row = row + wx[c] * a[(jj, ii) + tuple(np.broadcast_to(k, shape) for k in idx)]
        out = out + wy[b] * row
    out[off] = 0.0
    return out
