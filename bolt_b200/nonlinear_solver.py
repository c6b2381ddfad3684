"""nonlinear_solver: finite-volume kinetic update on one B200 (drop-in for
bolt/lib/nonlinear/nonlinear_solver.py:55-521 on its FVM path).

The distribution function lives on the GPU in Bolt's q-expanded memory
layout -- column-major (Np1*Np2*Np3, Ns, Nq1+2Ng, Nq2+2Ng), i.e. p1 fastest --
and ``solver.f`` is a torch view with exactly that shape and indexing, so
``solver.f[:, :, Ng:-Ng, Ng:-Ng]`` means what it means in Bolt.

Every df/dt evaluation, stage update, halo refresh, moment and field update
runs in the CUDA kernels of libbolt_b200.so (include/bolt_b200.h); there is no
CPU or PyTorch fallback.  The Python layer evaluates the user's configuration
callbacks (initialize_f, tau, Dirichlet boundary functions, initial fields) on
torch tensors and hands device pointers to the C ABI.

Supported plug-ins: bolt_b200.src.nonrelativistic_boltzmann (or Bolt's module
of the same name) C_q / C_p / BGK / moments.  Other plug-ins raise
NotImplementedError.
"""

import ctypes
import math
import os

import numpy as np
import torch

from . import _native as N

_PLUGIN_SUFFIX = 'nonrelativistic_boltzmann'
# conditions whose ghost values take the user's f_left / f_right / f_bottom / f_top
_DIRICHLET_BCS = ('dirichlet', 'mirror+dirichlet')


def _plugin_ok(fn, module_tail, name):
    mod = getattr(fn, '__module__', '') or ''
    return mod.endswith(_PLUGIN_SUFFIX + '.' + module_tail) and fn.__name__ == name


class _FieldsSolver(object):
    """View of the fields held by the native context (fields.py:19-690 API)."""

    def __init__(self, nls):
        self._nls = nls
        self.time_elapsed = 0.0          # advanced by evolve_electrodynamic_fields

    # the grid attributes the reference's fields_solver carries (fields.py:200-240)
    N_g = property(lambda self: self._nls.N_ghost)
    dq1 = property(lambda self: self._nls.dq1)
    dq2 = property(lambda self: self._nls.dq2)
    q1_center = property(lambda self: self._nls.q1_center)
    q2_center = property(lambda self: self._nls.q2_center)

    def _fetch(self):
        nls = self._nls
        shape = (6, nls.N_q2_local_with_Ng, nls.N_q1_local_with_Ng)
        cell = torch.empty(shape, dtype=torch.float64, device=nls.device)
        yee = torch.empty(shape, dtype=torch.float64, device=nls.device)
        N.check(nls._lib.bolt_fields_get(nls._ctx, cell.data_ptr(), yee.data_ptr(),
                                         nls._stream()), 'bolt_fields_get')
        return cell, yee

    @staticmethod
    def _af(a):
        # (6, Nq2g, Nq1g) -> (6, 1, Nq1g, Nq2g)
        return a.permute(0, 2, 1).unsqueeze(1)

    def _store(self, cell=None, yee=None):
        nls = self._nls
        conv = lambda a: None if a is None else \
            torch.as_tensor(a, dtype=torch.float64, device=nls.device)[:, 0].permute(0, 2, 1).contiguous()
        c, y = conv(cell), conv(yee)
        self._keep = (c, y)
        N.check(nls._lib.bolt_fields_set(nls._ctx, 0 if c is None else c.data_ptr(),
                                         0 if y is None else y.data_ptr(), nls._stream()),
                'bolt_fields_set')

    @property
    def cell_centered_EM_fields(self):
        return self._af(self._fetch()[0])

    @cell_centered_EM_fields.setter
    def cell_centered_EM_fields(self, value):
        self._store(cell=value)

    @property
    def yee_grid_EM_fields(self):
        return self._af(self._fetch()[1])

    @yee_grid_EM_fields.setter
    def yee_grid_EM_fields(self, value):
        self._store(yee=value)

    @property
    def at_n(self):
        return bool(self._nls._lib.bolt_get_at_n(self._nls._ctx))

    @at_n.setter
    def at_n(self, v):
        self._nls._lib.bolt_set_at_n(self._nls._ctx, 1 if v else 0)

    def get_fields(self):
        """Cell-centred (E1, E2, E3, B1, B2, B3), each (1, 1, Nq1g, Nq2g)."""
        c = self.cell_centered_EM_fields
        out = tuple(c[i:i + 1] for i in range(6))
        self.at_n = not self.at_n
        return out

    def evolve_electrodynamic_fields(self, J1, J2, J3, dt):
        """fields.py:568-647: one FDTD update with the caller's currents, each
        (1, N_s, Nq1g, Nq2g) (summed over species, as af.sum(J, 1)),
        (1, 1, Nq1g, Nq2g) or a scalar, on the E components' Yee positions."""
        nls = self._nls
        Nq1g, Nq2g = nls.N_q1_local_with_Ng, nls.N_q2_local_with_Ng

        def yee_layout(J):
            J = torch.as_tensor(J, dtype=torch.float64, device=nls.device)
            if J.dim() == 4:
                J = J.sum(dim=1, keepdim=True)
            return J.expand(1, 1, Nq1g, Nq2g).reshape(Nq1g, Nq2g).T
        J = torch.stack([yee_layout(J1), yee_layout(J2), yee_layout(J3)]).contiguous()
        self._keep_j = J                     # alive until the stream has used it
        N.check(nls._lib.bolt_fields_evolve(nls._ctx, J.data_ptr(), float(dt), nls._stream()),
                'bolt_fields_evolve')
        self.time_elapsed += dt

    def compute_divB(self):
        """fields.py:22-32: (B1 - B1 one cell back in q1) / dq1 + (B2 - B2 one
        cell back in q2) / dq2 at the cell's left-bottom corner, (1, 1, Nq1g, Nq2g)."""
        y = self._fetch()[1]
        d = (y[3] - _shift(y[3], 1, 0)) / self.dq1 + (y[4] - _shift(y[4], 0, 1)) / self.dq2
        return self._af(d.unsqueeze(0))

    def compute_divE(self):
        """fields.py:35-46: the divergence of E at the cell centre, after the
        periodic refresh of the Yee-grid halos, (1, 1, Nq1g, Nq2g)."""
        nls = self._nls
        y = _periodic_fill_fields(self._fetch()[1], nls.N_ghost, nls.N_q1, nls.N_q2)
        d = (_shift(y[0], -1, 0) - y[0]) / self.dq1 + (_shift(y[1], 0, -1) - y[1]) / self.dq2
        return self._af(d.unsqueeze(0))

    def check_maxwells_contraint_equations(self, rho):
        """fields.py:48-75: prints max |div B| and max |div E - rho + mean(rho)|
        over the interior cells."""
        g = self.N_g
        inner = lambda a: a[..., g:a.shape[-2] - g, g:a.shape[-1] - g]
        rho = torch.as_tensor(rho, dtype=torch.float64, device=self._nls.device)
        print("Initial Maxwell's Constraints:")
        print('MAX(|divB|) =', float(inner(self.compute_divB()).abs().max()))
        print('MAX(|divE-rho|) =',
              float(inner(self.compute_divE() - rho + rho.mean()).abs().max()))


class nonlinear_solver(object):

    def __init__(self, physical_system, performance_test_flag=False):
        if not torch.cuda.is_available():
            raise RuntimeError('bolt_b200 runs on a CUDA device (sm_100a); no CUDA device '
                               'is available and there is no CPU fallback')
        self._lib = N.load()
        self.physical_system = ps = physical_system
        params = ps.params
        self.performance_test_flag = performance_test_flag
        self.device = torch.device('cuda', torch.cuda.current_device())

        # ---- path checks ----------------------------------------------------
        # FVM in q and p, or the advective semi-Lagrangian method (ASL) in q
        # with fields off (timestep.py: then the method in p is not used) or
        # electrostatic fields and the FVM in p; ASL in p, and ASL in q with
        # electrodynamic fields, are not implemented
        self._asl = params.solver_method_in_q == 'ASL'
        fields_on = bool(getattr(params, 'fields_enabled', False))
        es = getattr(params, 'fields_type', 'electrodynamic') == 'electrostatic'
        if not ((params.solver_method_in_q == 'FVM' and params.solver_method_in_p == 'FVM') or
                (self._asl and (not fields_on or
                                (es and params.solver_method_in_p == 'FVM')))):
            raise NotImplementedError('solver methods: FVM in q and p, or ASL in q without '
                                      'fields or with electrostatic fields and the FVM in p')
        self._instantaneous = bool(getattr(params, 'instantaneous_collisions', False))
        if not (_plugin_ok(ps.C_q, 'advection_terms', 'C_q') and
                _plugin_ok(ps.C_p, 'advection_terms', 'C_p')):
            raise NotImplementedError('advection terms must be the nonrelativistic_boltzmann '
                                      'C_q / C_p')
        if not _plugin_ok(ps.source, 'collision_operator', 'BGK'):
            raise NotImplementedError('source must be nonrelativistic_boltzmann BGK')
        if getattr(params, 'hybrid_model_enabled', False):
            raise NotImplementedError('hybrid model')
        # p-space grid (compute_moments.py:42-56, boundaries.py:432-553): cartesian,
        # or polar2D (p1 the radius, p2 the angle)
        self._p_space_grid = getattr(params, 'p_space_grid', 'cartesian')
        if self._p_space_grid not in ('cartesian', 'polar2D'):
            raise NotImplementedError('Unsupported coordinate system in p_space')
        self.fields_enabled = bool(getattr(params, 'fields_enabled', False))
        self.fields_type = getattr(params, 'fields_type', 'electrodynamic')
        if self.fields_enabled:
            ok = (self.fields_type == 'electrodynamic' and
                  getattr(params, 'fields_solver', 'fdtd') == 'fdtd') or \
                (self.fields_type == 'electrostatic' and
                 getattr(params, 'fields_solver', 'fft') == 'fft')
            if not ok:
                raise NotImplementedError('fields: electrodynamic FDTD or electrostatic FFT only')

        # ---- domain ---------------------------------------------------------------
        self.q1_start, self.q1_end = ps.q1_start, ps.q1_end
        self.q2_start, self.q2_end = ps.q2_start, ps.q2_end
        self.p1_start, self.p1_end = ps.p1_start, ps.p1_end
        self.p2_start, self.p2_end = ps.p2_start, ps.p2_end
        self.p3_start, self.p3_end = ps.p3_start, ps.p3_end
        self.N_q1, self.dq1 = ps.N_q1, ps.dq1
        self.N_q2, self.dq2 = ps.N_q2, ps.dq2
        self.N_p1, self.N_p2, self.N_p3 = ps.N_p1, ps.N_p2, ps.N_p3
        N_g = self.N_ghost = ps.N_ghost
        self.N_g1 = self.N_g2 = N_g
        self.boundary_conditions = bc = ps.boundary_conditions
        self._comm = ps.mpi_communicator
        Ns = self.N_species = ps.N_species
        if Ns > N.MAX_SPECIES:
            raise NotImplementedError('at most %d species' % N.MAX_SPECIES)

        def axis_bc(lo, hi):
            a, b = getattr(bc, lo), getattr(bc, hi)
            if a != b:
                raise Exception('%s and %s boundary conditions must match' % (lo, hi))
            if a not in N.BC:
                raise NotImplementedError('boundary condition %r' % a)
            return a
        self._bc_q1 = axis_bc('in_q1_left', 'in_q1_right')
        self._bc_q2 = axis_bc('in_q2_bottom', 'in_q2_top')

        self.N_q1_local, self.N_q2_local = self.N_q1, self.N_q2
        self.N_q1_local_with_Ng = self.N_q1 + 2 * N_g
        self.N_q2_local_with_Ng = self.N_q2 + 2 * N_g
        self.i_q1_start, self.i_q1_end = N_g, -N_g if N_g else None
        self.i_q2_start, self.i_q2_end = N_g, -N_g if N_g else None
        self._mass = [float(m) for m in _as_list(params.mass, Ns)]
        self._charge = [float(c) for c in _as_list(params.charge, Ns)]
        prec = getattr(params, 'precision', 'fp64')
        self.dtype = torch.float32 if prec in ('fp32', 'float32', 'single') else torch.float64
        # 'fp64-fast': FP64 f whose fused q-stage runs the paired kernel with
        # FMA and Newton-refined reciprocals (the reference's operation order
        # is kept by 'fp64')
        self._fast64 = prec == 'fp64-fast'
        self.time_integrator = getattr(params, 'time_integrator', 'RK2')
        if self.time_integrator not in N.RK:
            raise NotImplementedError('time_integrator %r' % self.time_integrator)

        self._build_grids(params)
        self._dp1_list, self._dp2_list, self._dp3_list = list(ps.dp1), list(ps.dp2), list(ps.dp3)
        # the reference turns these into (1, Ns) arrays (nonlinear_solver.py:133-145,378-389)
        t = lambda v: torch.tensor(v, dtype=torch.float64, device=self.device).reshape(1, Ns, 1, 1)
        params.mass = t(self._mass)
        params.charge = t(self._charge)
        self.dp1, self.dp2, self.dp3 = t(ps.dp1), t(ps.dp2), t(ps.dp3)

        # ---- native context ----------------------------------------------------------
        self._fstore = None
        self._ctx = None
        self._create_context(params)

        # ---- initial state (nonlinear_solver.py:464-500) -----------------------------
        self._initialize(params)
        self.time_elapsed = 0
        self._A_q, self._C_q, self._A_p, self._C_p = ps.A_q, ps.C_q, ps.A_p, ps.C_p
        self._source = ps.source
        self._perf = {'time_ts': 0.0, 'steps': 0}
        self._perf_parts = np.zeros(len(N.TIMING_NAMES))
        if performance_test_flag:
            # per-component device time of every launch group (CUDA events)
            N.check(self._lib.bolt_set_timing(self._ctx, 1), 'bolt_set_timing')

    # -----------------------------------------------------------------------------
    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _build_grids(self, params):
        """q (with ghosts) and p grids as AF-shaped float64 tensors
        (calculate_q.py:7-41, calculate_p.py:8-57)."""
        dev, Ng = self.device, self.N_ghost
        i1 = torch.arange(-Ng, self.N_q1 + Ng, dtype=torch.float64, device=dev)
        i2 = torch.arange(-Ng, self.N_q2 + Ng, dtype=torch.float64, device=dev)
        q1_lb = (self.q1_start + i1 * self.dq1).reshape(1, 1, -1, 1)
        q2_lb = (self.q2_start + i2 * self.dq2).reshape(1, 1, 1, -1)
        shape = (1, 1, i1.numel(), i2.numel())
        self.q1_left_bot = q1_lb.expand(shape).contiguous()
        self.q2_left_bot = q2_lb.expand(shape).contiguous()
        self.q1_center_bot = self.q1_left_bot + 0.5 * self.dq1
        self.q2_center_bot = self.q2_left_bot
        # calculate_q.py:35-38 returns (q1_left_center, q2_center_bot) as the
        # left-centre grid: its q2 is the cell's bottom face, as here
        self.q1_left_center = self.q1_left_bot
        self.q2_left_center = self.q2_center_bot
        self.q1_center = self.q1_left_bot + 0.5 * self.dq1
        self.q2_center = self.q2_left_bot + 0.5 * self.dq2
        ps = self.physical_system
        Np = self.N_p1 * self.N_p2 * self.N_p3
        Ns = self.N_species
        pc = [torch.empty(Np, Ns, dtype=torch.float64) for _ in range(3)]
        pl = [torch.empty(Np, Ns, dtype=torch.float64) for _ in range(3)]
        for s in range(Ns):
            for d, (st, dp, n) in enumerate(((ps.p1_start[s], ps.dp1[s], self.N_p1),
                                            (ps.p2_start[s], ps.dp2[s], self.N_p2),
                                            (ps.p3_start[s], ps.dp3[s], self.N_p3))):
                c = st + (0.5 + np.arange(n)) * dp
                l = st + np.arange(n) * dp
                shp = [1, 1, 1]
                shp[2 - d] = n           # (p3, p2, p1) flattened, p1 fastest
                pc[d][:, s] = torch.from_numpy(np.broadcast_to(c.reshape(shp), (self.N_p3, self.N_p2, self.N_p1)).reshape(-1).copy())
                pl[d][:, s] = torch.from_numpy(np.broadcast_to(l.reshape(shp), (self.N_p3, self.N_p2, self.N_p1)).reshape(-1).copy())
        to4 = lambda a: a.reshape(Np, Ns, 1, 1).to(dev)
        self.p1_center, self.p2_center, self.p3_center = (to4(a) for a in pc)
        self.p1_left, self.p2_bottom, self.p3_back = (to4(a) for a in pl)
        self.p2_left = self.p2_center
        self.p3_left = self.p3_center
        self.p1_bottom = self.p1_center
        self.p3_bottom = self.p3_center
        self.p1_back = self.p1_center
        self.p2_back = self.p2_center

    def _create_context(self, params):
        ps = self.physical_system
        g = N.BoltGrid()
        g.N_q1, g.N_q2, g.N_ghost = self.N_q1, self.N_q2, self.N_ghost
        g.N_p1, g.N_p2, g.N_p3, g.N_s = self.N_p1, self.N_p2, self.N_p3, self.N_species
        g.q1_start, g.q2_start, g.dq1, g.dq2 = self.q1_start, self.q2_start, self.dq1, self.dq2
        for s in range(self.N_species):
            g.p1_start[s], g.p2_start[s], g.p3_start[s] = ps.p1_start[s], ps.p2_start[s], ps.p3_start[s]
            g.dp1[s], g.dp2[s], g.dp3[s] = ps.dp1[s], ps.dp2[s], ps.dp3[s]
        p = N.BoltParams()
        p.dtype = N.F32 if self.dtype == torch.float32 else (N.F64_FAST if self._fast64 else N.F64)
        try:
            p.recon_q = N.RECON[params.reconstruction_method_in_q]
            p.recon_p = N.RECON[params.reconstruction_method_in_p]
        except KeyError:
            raise NotImplementedError('Reconstruction method invalid/not-implemented')
        p.flux_q = N.FLUX.get(getattr(params, 'riemann_solver_in_q', 'upwind-flux'), 0)
        p.flux_p = N.FLUX.get(getattr(params, 'riemann_solver_in_p', 'upwind-flux'), 0)
        p.bc_q1, p.bc_q2 = N.BC[self._bc_q1], N.BC[self._bc_q2]
        p.integrator = N.RK[self.time_integrator]
        p.source_enabled = 1 if getattr(params, 'source_enabled', False) else 0
        p.fields_enabled = 1 if self.fields_enabled else 0
        p.fields_type = N.FIELDS[self.fields_type] if self.fields_enabled else 0
        p.p_dim = int(params.p_dim)
        for s in range(self.N_species):
            p.mass[s], p.charge[s] = self._mass[s], self._charge[s]
        p.boltzmann_constant = float(params.boltzmann_constant)
        p.tau = 1.0
        p.eps = float(getattr(params, 'eps', 1.0))
        p.mu = float(getattr(params, 'mu', 1.0))
        self._tau_arr = None
        if p.source_enabled:
            tau = params.tau(self.q1_center, self.q2_center,
                             self.p1_center, self.p2_center, self.p3_center)
            tau = torch.as_tensor(tau, dtype=torch.float64, device=self.device)
            flat = tau.reshape(-1)
            if bool(torch.all(flat == flat[0])):
                p.tau = float(flat[0])
            else:
                full = torch.broadcast_to(tau, self._af_shape())
                self._tau_arr = self._to_store(full)
        ctx = N.ctypes.c_void_p()
        N.check(self._lib.bolt_ctx_create(N.ctypes.byref(g), N.ctypes.byref(p),
                                          N.ctypes.byref(ctx)), 'bolt_ctx_create')
        self._ctx = ctx
        if self._tau_arr is not None:
            N.check(self._lib.bolt_set_tau_array(ctx, self._tau_arr.data_ptr()), 'bolt_set_tau_array')
        if self._p_space_grid == 'polar2D':
            N.check(self._lib.bolt_set_p_space_grid(ctx, N.PGRID['polar2D'],
                                                    float(params.initial_mu)),
                    'bolt_set_p_space_grid')
        self._shearing = 'shearing-box' in (self._bc_q1, self._bc_q2)
        if self._asl and (self._has_dirichlet() or self._shearing or
                          self._tau_arr is not None):
            raise NotImplementedError('the semi-Lagrangian q-step takes periodic or mirror '
                                      'q boundaries and a constant tau')
        if self._shearing:
            # boundaries.py:17-18: the shear rate q omega of the params module
            N.check(self._lib.bolt_set_shear(ctx, float(params.q), float(params.omega)),
                    'bolt_set_shear')

    def __del__(self):
        try:
            if self._ctx is not None:
                self._lib.bolt_ctx_destroy(self._ctx)
                self._ctx = None
        except Exception:
            pass

    # ---- layout helpers ---------------------------------------------------------------
    def _af_shape(self):
        return (self.N_p1 * self.N_p2 * self.N_p3, self.N_species,
                self.N_q1_local_with_Ng, self.N_q2_local_with_Ng)

    def _store_shape(self):
        return (self.N_q2_local_with_Ng, self.N_q1_local_with_Ng, self.N_species,
                self.N_p1 * self.N_p2 * self.N_p3)

    def _to_store(self, af_array):
        """AF-ordered (Np, Ns, Nq1g, Nq2g) tensor -> contiguous storage tensor."""
        out = torch.empty(self._store_shape(), dtype=self.dtype, device=self.device)
        out.permute(3, 2, 1, 0).copy_(torch.broadcast_to(af_array, self._af_shape()))
        return out

    @property
    def f(self):
        return self._fstore.permute(3, 2, 1, 0)

    @f.setter
    def f(self, value):
        # a host tensor with the same (permuted) strides is copied with one
        # asynchronous memcpy; anything else goes through torch's copy
        self.f.copy_(torch.as_tensor(value), non_blocking=True)
        self._invalidate()

    def _invalidate(self):
        if self._ctx is not None:
            self._lib.bolt_invalidate(self._ctx)

    def _sync_external_edits(self):
        v = self._fstore._version
        if v != self._seen_version:
            self._invalidate()
            self._refresh_boundaries()
            self._seen_version = v

    def _has_dirichlet(self):
        return any(b in _DIRICHLET_BCS for b in (self._bc_q1, self._bc_q2))

    def _refresh_boundaries(self):
        """Evaluate the Dirichlet boundary functions (boundaries.py:147-225)."""
        if not self._has_dirichlet():
            return
        bc = self.boundary_conditions
        args = (self.f, self.time_elapsed, self.q1_center, self.q2_center,
                self.p1_center, self.p2_center, self.p3_center, self.physical_system.params)
        self._dirichlet = {}
        sides = ['left', 'right'] if self._bc_q1 in _DIRICHLET_BCS else []
        sides += ['bottom', 'top'] if self._bc_q2 in _DIRICHLET_BCS else []
        for k, side in enumerate(('left', 'right', 'bottom', 'top')):
            if side not in sides:
                continue
            val = getattr(bc, 'f_' + side)(*args)
            arr = self._to_store(torch.as_tensor(val, device=self.device))
            self._dirichlet[side] = arr
            N.check(self._lib.bolt_set_dirichlet(self._ctx, k, arr.data_ptr()), 'bolt_set_dirichlet')

    def _initialize(self, params):
        ic = self.physical_system.initial_conditions
        f0 = ic.initialize_f(self.q1_center, self.q2_center, self.p1_center,
                             self.p2_center, self.p3_center, params)
        self._fstore = self._to_store(torch.as_tensor(f0, device=self.device))
        self.time_elapsed = 0
        self._refresh_boundaries()
        N.check(self._lib.bolt_fill_ghosts(self._ctx, self._fstore.data_ptr(), self._stream()),
                'bolt_fill_ghosts')
        self._seen_version = self._fstore._version
        self.f_initial = self.f.clone()
        if self.fields_enabled:
            self._init_fields(params)

    # ---- fields initialisation (fields.py:421-495, fft.py:9-78) -------------------------
    def _user_field(self, fn, k, q1, q2, params):
        """Component k of a user field function on one of the staggered q-grids,
        as a (N_q2 + 2N_g, N_q1 + 2N_g) FP64 tensor."""
        Nq1g, Nq2g = self.N_q1_local_with_Ng, self.N_q2_local_with_Ng
        a = torch.as_tensor(fn(q1, q2, params)[k], dtype=torch.float64, device=self.device)
        return a.expand(1, 1, Nq1g, Nq2g).reshape(Nq1g, Nq2g).T

    def _user_E(self, params):
        """fields.py:280-337: E1 on the left-centre grid (q2 at the bottom face,
        see _build_grids), E2 at (centre, bottom), E3 at the centre, from
        initialize_E; or from initialize_A_phi by the reference's one-sided
        differences of A and phi."""
        ini = self.physical_system.initial_conditions
        u = lambda fn, k, at: self._user_field(fn, k, *at, params)
        lc = (self.q1_left_center, self.q2_left_center)
        cb = (self.q1_center_bot, self.q2_center_bot)
        cc = (self.q1_center, self.q2_center)
        lb = (self.q1_left_bot, self.q2_left_bot)
        if hasattr(ini, 'initialize_E'):
            E = ini.initialize_E
            return torch.stack([u(E, 0, lc), u(E, 1, cb), u(E, 2, cc)])
        if hasattr(ini, 'initialize_A_phi'):
            F = ini.initialize_A_phi
            A1, A2, A3, phi = u(F, 0, cb), u(F, 1, lc), u(F, 2, lb), u(F, 3, cc)
            dA3_dq2 = (_shift(A3, 0, -1) - A3) / self.dq2
            dA3_dq1 = (_shift(A3, -1, 0) - A3) / self.dq1
            dA2_dq1 = (_shift(A2, -1, 0) - A2) / self.dq1
            dA1_dq2 = (_shift(A1, 0, -1) - A1) / self.dq2
            dphi_dq1 = -(_shift(phi, 1, 0) - phi) / self.dq1
            dphi_dq2 = -(_shift(phi, 0, 1) - phi) / self.dq2
            return torch.stack([dA3_dq2 - dphi_dq1, -dA3_dq1 - dphi_dq2, dA2_dq1 - dA1_dq2])
        raise NotImplementedError('Initialization method for electric fields not valid/found')

    def _user_B(self, params):
        """fields.py:339-410: B1 at (centre, bottom), B2 on the left-centre
        grid, B3 at (left, bottom), from initialize_B; or from initialize_A, or
        from initialize_A3_B3 (B1, B2 as backward differences of A3)."""
        ini = self.physical_system.initial_conditions
        u = lambda fn, k, at: self._user_field(fn, k, *at, params)
        lc = (self.q1_left_center, self.q2_left_center)
        cb = (self.q1_center_bot, self.q2_center_bot)
        cc = (self.q1_center, self.q2_center)
        lb = (self.q1_left_bot, self.q2_left_bot)
        if hasattr(ini, 'initialize_B') and hasattr(ini, 'initialize_A3_B3'):
            raise Exception('Can\'t use both initialize_B and initialize_A3_B3!')
        if hasattr(ini, 'initialize_B'):
            B = ini.initialize_B
            return torch.stack([u(B, 0, cb), u(B, 1, lc), u(B, 2, lb)])
        if hasattr(ini, 'initialize_A'):
            F = ini.initialize_A
            A1, A2, A3 = u(F, 0, lc), u(F, 1, cb), u(F, 2, cc)
            B1 = (_shift(A3, 0, -1) - A3) / self.dq2
            B2 = -(_shift(A3, -1, 0) - A3) / self.dq1
            B3 = (_shift(A2, -1, 0) - A2) / self.dq1 - (_shift(A1, 0, -1) - A1) / self.dq2
            return torch.stack([B1, B2, B3])
        if hasattr(ini, 'initialize_A3_B3'):
            F = ini.initialize_A3_B3
            A3 = u(F, 0, cc)
            B1 = (A3 - _shift(A3, 0, 1)) / self.dq2
            B2 = -(A3 - _shift(A3, 1, 0)) / self.dq1
            return torch.stack([B1, B2, u(F, 1, lb)])
        raise NotImplementedError('Initialization method for magnetic fields not valid/found')

    def _init_fields(self, params):
        dev, Ng = self.device, self.N_ghost
        Nq1g, Nq2g = self.N_q1_local_with_Ng, self.N_q2_local_with_Ng
        cell = torch.zeros((6, Nq2g, Nq1g), dtype=torch.float64, device=dev)
        yee = torch.zeros_like(cell)
        eps = float(getattr(params, 'eps', 1.0))
        init = params.fields_initialize
        if init in ('fft', 'fft + user-defined magnetic fields'):
            dens = self._moment_store('density')                       # (Nq2g, Nq1g, Ns)
            q = torch.tensor(self._charge, dtype=torch.float64, device=dev)
            rho = (dens * q).sum(dim=2)
            r = rho[Ng:Nq2g - Ng, Ng:Nq1g - Ng].T.contiguous()         # (Nq1, Nq2)
            k1 = torch.from_numpy(np.fft.fftfreq(r.shape[0], self.dq1)).to(dev)
            k2 = torch.from_numpy(np.fft.fftfreq(r.shape[1], self.dq2)).to(dev)
            k1, k2 = torch.meshgrid(k1, k2, indexing='ij')
            r = r - r.mean()
            rh = torch.fft.fft2(r)
            den = 4 * math.pi ** 2 * (k1 ** 2 + k2 ** 2)
            den[0, 0] = 1.0
            ph = rh / den
            ph[0, 0] = 0
            E1 = torch.fft.ifft2(-1j * 2 * math.pi * k1 * ph).real
            E2 = torch.fft.ifft2(-1j * 2 * math.pi * k2 * ph).real
            cell[0, Ng:Nq2g - Ng, Ng:Nq1g - Ng] = E1.T / eps
            cell[1, Ng:Nq2g - Ng, Ng:Nq1g - Ng] = E2.T / eps
            cell = _periodic_fill_fields(cell, Ng, self.N_q1, self.N_q2)
            yee[0] = 0.5 * (cell[0] + torch.roll(cell[0], 1, dims=1))
            yee[1] = 0.5 * (cell[1] + torch.roll(cell[1], 1, dims=0))
            yee[2] = cell[2]
            if init != 'fft':
                # fields.py:477-482: user B on the Yee grid, then its cell values
                yee[3:6] = self._user_B(params)
                cell[3:6] = _yee_to_cell(yee)[3:6]
            yee = _periodic_fill_fields(yee, Ng, self.N_q1, self.N_q2)
        elif init == 'user-defined':
            # fields.py:472-475: Yee E and B from the user's functions, then
            # every cell-centred field from the (not yet refreshed) Yee grid
            yee[0:3] = self._user_E(params)
            yee[3:6] = self._user_B(params)
            cell = _yee_to_cell(yee)
            yee = _periodic_fill_fields(yee, Ng, self.N_q1, self.N_q2)
        else:
            raise NotImplementedError('fields_initialize %r' % init)
        self._cell0, self._yee0 = cell.contiguous(), yee.contiguous()
        N.check(self._lib.bolt_fields_set(self._ctx, self._cell0.data_ptr(), self._yee0.data_ptr(),
                                          self._stream()), 'bolt_fields_set')
        self.fields_solver = _FieldsSolver(self)

    # ---- time stepping (timestep.py:40-285) ------------------------------------------------
    def _step(self, dt):
        self.dt = dt
        self._sync_external_edits()
        if self.performance_test_flag:
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record()
        if self._has_dirichlet():
            self._refresh_boundaries()
        if self._shearing:
            # the strips of every stage are sheared to the step's start time
            # (the reference's time_elapsed, advanced after the step)
            self._lib.bolt_set_time(self._ctx, float(self.time_elapsed))
        N.check(self._lib.bolt_step(self._ctx, self._fstore.data_ptr(), float(dt), self._stream()),
                'bolt_step')
        self._seen_version = self._fstore._version
        if self.performance_test_flag:
            t1.record()
            t1.synchronize()
            self._perf['time_ts'] += t0.elapsed_time(t1) * 1e-3
            self._perf['steps'] += 1
        self.check_divergence()
        self.time_elapsed += dt

    def _communicate_f(self):
        """communicate.py:8-38 with apply_bcs_f (boundaries.py:415-577): one
        pass of the ghost kernel fills every ghost cell of f -- periodic
        images, mirror images, Dirichlet inflow -- from the interior."""
        self._sync_external_edits()
        if self._has_dirichlet():
            self._refresh_boundaries()
        if self._shearing:
            self._lib.bolt_set_time(self._ctx, float(self.time_elapsed))
        N.check(self._lib.bolt_fill_ghosts(self._ctx, self._fstore.data_ptr(), self._stream()),
                'bolt_fill_ghosts')
        self._seen_version = self._fstore._version

    # the ghost pass applies the boundary conditions too; calling it again is
    # harmless (every ghost is a function of the interior)
    _apply_bcs_f = _communicate_f

    def check_divergence(self):
        """timestep.py:28-38 -- the device flags any non-finite f value written
        by a step; the flag is read from pinned host memory without
        synchronising, so it reports steps whose kernels have completed (the
        reference's check is synchronous; here a non-finite step raises at the
        first step boundary after its kernels finished).  A stage whose
        bounded tile wait ran out left part of f unwritten: its error word is
        read the same way and raised as a BoltError (BOLT_ERR_TIMEOUT)."""
        err = self._lib.bolt_error_flag(self._ctx)
        if err:
            raise N.BoltError(err, 'stage kernel')
        if self._lib.bolt_divergence_flag(self._ctx):
            raise SystemExit('Solver Diverging!')

    def set_wait_budget(self, cycles):
        """Budget of the stage kernels' bounded tile waits in SM clock cycles
        (None or <= 0: the default, about 2 s)."""
        N.check(self._lib.bolt_set_wait_budget(self._ctx, int(cycles or 0)),
                'bolt_set_wait_budget')

    # with the FVM in both q and p every splitting scheme is the same step
    # (timestep.py:13-15); ASL in q splits op_advect_q and op_solve_src
    def strang_timestep(self, dt):
        self._asl_step(dt, 'strang') if self._asl else self._step(dt)

    def lie_timestep(self, dt):
        self._asl_step(dt, 'lie') if self._asl else self._step(dt)

    def swss_timestep(self, dt):
        self._asl_step(dt, 'swss') if self._asl else self._step(dt)

    def jia_timestep(self, dt):
        self._asl_step(dt, 'jia') if self._asl else self._step(dt)

    # ---- advective semi-Lagrangian in q (asl_operators.py:20-83) ------------------
    def _work_buffer(self):
        # device address of the context's f-shaped work buffer 0
        if getattr(self, '_wbuf', None) is None:
            ptr = ctypes.c_void_p()
            N.check(self._lib.bolt_work_buffer(self._ctx, 0, ctypes.byref(ptr)),
                    'bolt_work_buffer')
            self._wbuf = ptr.value
        return self._wbuf

    def _op_advect_q(self, dt):
        N.check(self._lib.bolt_asl_advect_q(self._ctx, self._fstore.data_ptr(), float(dt),
                                            self._stream()), 'bolt_asl_advect_q')

    def _op_solve_src(self, dt):
        # f <- f_MB where collisions are instantaneous, else RK2 of the source
        # when it is enabled (asl_operators.py:40-83)
        if self._instantaneous or self.physical_system.params.source_enabled:
            N.check(self._lib.bolt_asl_source(self._ctx, self._fstore.data_ptr(), float(dt),
                                              int(self._instantaneous), self._stream()),
                    'bolt_asl_source')

    def _asl_step(self, dt, scheme):
        """One timestep of ASL in q without fields: op_advect_q and
        op_solve_src composed by the named splitting (timestep.py:39-240,
        operator_splitting_methods.py); SWSS and Jia keep copies of f."""
        self.dt = dt
        self._sync_external_edits()
        if self.performance_test_flag:
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record()
        op1, op2 = self._op_advect_q, self._op_solve_src
        f = self._fstore
        if self.fields_enabled:
            # (op_advect_q, op_solve_src) by the scheme, split again with op_fvm,
            # the FVM in p (timestep.py:134-148)
            if scheme not in ('strang', 'lie'):
                raise NotImplementedError('ASL in q with fields: Strang or Lie splitting')
            adv, src = op1, op2

            def pair(d):
                if scheme == 'strang':
                    adv(0.5 * d)
                    src(d)
                    adv(0.5 * d)
                else:
                    adv(d)
                    src(d)

            def op_fvm(d):
                N.check(self._lib.bolt_fvm_p_step(self._ctx, f.data_ptr(), float(d),
                                                  self._stream()), 'bolt_fvm_p_step')
            op1, op2 = pair, op_fvm

        def strang(a, b):
            a(0.5 * dt)
            b(dt)
            a(0.5 * dt)

        src_on = self._instantaneous or self.physical_system.params.source_enabled
        if not self.fields_enabled and src_on and scheme in ('strang', 'lie'):
            # f handed between the operators through the context's work
            # buffer w, no copy back: Strang f -> w -> w -> f, Lie f -> w -> f
            w = self._work_buffer()
            fp = f.data_ptr()

            def adv_to(src, dst, d):
                N.check(self._lib.bolt_asl_advect_q_to(self._ctx, src, dst, float(d),
                                                       self._stream()), 'bolt_asl_advect_q_to')

            def src_to(src, dst, d):
                N.check(self._lib.bolt_asl_source_to(self._ctx, src, dst, fp, float(d),
                                                     int(self._instantaneous), self._stream()),
                        'bolt_asl_source_to')

            if scheme == 'strang':
                adv_to(fp, w, 0.5 * dt)
                src_to(w, w, dt)
                adv_to(w, fp, 0.5 * dt)
            else:
                adv_to(fp, w, dt)
                src_to(w, fp, dt)
            scheme = None

        def swss(a, b):
            start = f.clone()
            a(dt)
            b(dt)
            mid = f.clone()
            f.copy_(start)
            b(dt)
            a(dt)
            f.add_(mid).mul_(0.5)

        if scheme is None:
            pass
        elif scheme == 'strang':
            strang(op1, op2)
        elif scheme == 'lie':
            op1(dt)
            op2(dt)
        elif scheme == 'swss':
            swss(op1, op2)
        else:                                            # jia
            start = f.clone()
            strang(op1, op2)
            f1 = f.clone()
            f.copy_(start)
            strang(op2, op1)
            f2 = f.clone()
            f.copy_(start)
            swss(op1, op2)
            f.copy_((2 / 3) * (f1 + f2) - (1 / 3) * f)
        if scheme in ('swss', 'jia'):
            # f was combined outside the context: its ghosts and moments are new
            self._lib.bolt_invalidate(self._ctx)
        self._seen_version = self._fstore._version
        if self.performance_test_flag:
            t1.record()
            t1.synchronize()
            self._perf['time_ts'] += t0.elapsed_time(t1) * 1e-3
            self._perf['steps'] += 1
        # timestep.py:28-38: the operators' kernels flag a non-finite value
        # they write (read from pinned memory without synchronising)
        self.check_divergence()
        self.time_elapsed += dt

    def run(self, dt, n_steps):
        """n_steps strang steps launched back to back (no per-step host work)."""
        self.dt = dt
        self._sync_external_edits()
        if self._has_dirichlet() or self._shearing:
            # per-step host work: boundary values / the strips' shear time
            for _ in range(n_steps):
                self._step(dt)
            return
        N.check(self._lib.bolt_run(self._ctx, self._fstore.data_ptr(), float(dt), int(n_steps),
                                   self._stream()), 'bolt_run')
        self._seen_version = self._fstore._version
        self.check_divergence()
        self.time_elapsed += dt * n_steps

    # ---- stage-level stepping (q2 slabs exchange halos between stages) ----------------
    def stage_count(self):
        return int(self._lib.bolt_stage_count(self._ctx))

    def stage_input(self, k):
        """The buffer RK stage k of the next step reads, as a tensor of the
        storage shape (N_q2 + 2N_g, N_q1 + 2N_g, N_s, N_p) (its ghost rows must
        be current before stage k runs)."""
        if k == 0:
            return self._fstore
        ptr = self._lib.bolt_stage_input(self._ctx, self._fstore.data_ptr(), int(k))
        if not ptr:
            raise ValueError('stage %d of %d' % (k, self.stage_count()))
        flat = torch.as_tensor(N.DeviceArray(ptr, self._fstore.numel(),
                                             '<f4' if self.dtype == torch.float32 else '<f8'),
                               device=self.device)
        return flat.view(self._store_shape())

    def stage(self, k, dt):
        """Run RK stage k of the step of f (stages 0 .. stage_count()-1 in
        order make one strang_timestep, without its time bookkeeping)."""
        self.dt = dt
        N.check(self._lib.bolt_stage(self._ctx, self._fstore.data_ptr(), float(dt), int(k),
                                     self._stream()), 'bolt_stage')
        self._seen_version = self._fstore._version

    def stage_region(self, k, region, dt):
        """Part of RK stage k of a block (bolt_stage_region): region 0 updates
        the q-tiles that read no ghost cell of an external axis, region 1 the
        others, region 2 finishes the stage after both.  Returns False, having
        done nothing, when the stage cannot be split; the caller then runs
        stage(k, dt)."""
        self.dt = dt
        rc = self._lib.bolt_stage_region(self._ctx, self._fstore.data_ptr(), float(dt), int(k),
                                         int(region), self._stream())
        if rc == N.BOLT_ERR_UNSUPPORTED:
            return False
        N.check(rc, 'bolt_stage_region')
        self._seen_version = self._fstore._version
        return True

    _TERMS = {'d_flux_p1_dp1': 1, 'd_flux_p2_dp2': 2, 'd_flux_p3_dp3': 3}

    def df_dt(self, f=None, evolve_fields=None, term_to_return=None):
        """df/dt of f (df_dt_fvm.py:33-339) as an AF-ordered tensor.  Ghost
        cells of f are refreshed first (as fvm_operator.py does before every
        evaluation); with fields, evolve_fields=None follows the reference's
        at_n alternation.  term_to_return = 'd_flux_p1_dp1', 'd_flux_p2_dp2'
        or 'd_flux_p3_dp3' returns that p-flux divergence alone
        (df_dt_fvm.py:325-339); like the reference it needs fields."""
        term = 0
        if term_to_return is not None and term_to_return in self._TERMS:
            if not self.fields_enabled:
                raise ValueError('term_to_return=%r needs fields_enabled (the p-fluxes are '
                                 'computed only with fields)' % term_to_return)
            term = self._TERMS[term_to_return]
        if f is None:
            self._sync_external_edits()
            src = self._fstore.clone()
        else:
            src = self._to_store(torch.as_tensor(f, device=self.device))
        if self._shearing:
            self._lib.bolt_set_time(self._ctx, float(self.time_elapsed))
        N.check(self._lib.bolt_fill_ghosts(self._ctx, src.data_ptr(), self._stream()),
                'bolt_fill_ghosts')
        self._invalidate()
        out = torch.zeros_like(src)
        ev = 0
        if self.fields_enabled:
            at_n = bool(self._lib.bolt_get_at_n(self._ctx))
            ev = int((not at_n) if evolve_fields is None else bool(evolve_fields))
            self._lib.bolt_set_at_n(self._ctx, 0 if at_n else 1)
        if term:
            N.check(self._lib.bolt_dfdt_term(self._ctx, src.data_ptr(), out.data_ptr(), term, ev,
                                             float(getattr(self, 'dt', 0.0)), self._stream()),
                    'bolt_dfdt_term')
        else:
            N.check(self._lib.bolt_dfdt(self._ctx, src.data_ptr(), out.data_ptr(), ev,
                                        float(getattr(self, 'dt', 0.0)), self._stream()),
                    'bolt_dfdt')
        return out.permute(3, 2, 1, 0)

    # ---- moments (compute_moments.py:7-59) -------------------------------------------------
    def _moment_store(self, moment_name, store=None):
        if moment_name not in N.MOMENT_IDS:
            raise NotImplementedError('moment %r is not one of the nonrelativistic moments'
                                      % moment_name)
        src = self._fstore if store is None else store
        out = torch.empty((self.N_q2_local_with_Ng, self.N_q1_local_with_Ng, self.N_species),
                          dtype=torch.float64, device=self.device)
        N.check(self._lib.bolt_moments(self._ctx, src.data_ptr(), N.MOMENT_IDS[moment_name],
                                       out.data_ptr(), self._stream()), 'bolt_moments')
        return out

    def compute_moments(self, moment_name, f=None):
        """Moment over the whole ghosted grid, shape (1, Ns, Nq1g, Nq2g), FP64."""
        store = None if f is None else self._to_store(torch.as_tensor(f, device=self.device))
        return self._moment_store(moment_name, store).permute(2, 1, 0).unsqueeze(0)

    # ---- file I/O (file_io/dump.py, load.py): PETSc binary Vec format ------------------------
    def _interior_store(self):
        g = self.N_ghost
        s = self._fstore
        return s[g:s.shape[0] - g, g:s.shape[1] - g]

    def dump_distribution_function(self, file_name):
        """Interior f as a PETSc binary Vec (dump.py:121-168): big-endian int32
        class id 1211214, int32 length, big-endian float64 values ordered
        (q2, q1, s, p) with p1 fastest (the DMDA natural ordering)."""
        data = self._interior_store().to(torch.float64).cpu().numpy()
        _write_petsc_vec(file_name + '.bin', data.reshape(-1),
                         block=self.N_species * self.N_p1 * self.N_p2 * self.N_p3)

    def load_distribution_function(self, file_name):
        """load.py:10-43: read the Vec, copy to the interior, refresh halos."""
        self._load_interior(_read_petsc_vec(file_name + '.bin'))

    def _load_interior(self, vals):
        """FP64 interior values in natural order (q2, q1, s, p) -> f, ghosts refilled."""
        inner = torch.from_numpy(np.ascontiguousarray(vals)).to(self.device, self.dtype)
        self._interior_store().copy_(inner.reshape(self._interior_store().shape))
        self._invalidate()
        N.check(self._lib.bolt_fill_ghosts(self._ctx, self._fstore.data_ptr(), self._stream()),
                'bolt_fill_ghosts')
        self._seen_version = self._fstore._version

    def dump_moments(self, file_name):
        """dump.py:41-119: all moments of the moments module, alphabetical,
        joined along the species axis, interior cells, PETSc binary Vec."""
        arr = self._moments_interior()
        _write_petsc_vec(file_name + '.bin', arr.reshape(-1), block=arr.shape[2])

    def _moments_interior(self):
        """(N_q2, N_q1, N_moments N_s) FP64 numpy array of dump_moments."""
        attrs = [a for a in dir(self.physical_system.moments) if not a.startswith('_')]
        if 'integral_over_v' in attrs:
            attrs.remove('integral_over_v')
        g = self.N_ghost
        parts = []
        for a in attrs:
            m = self._moment_store(a)
            parts.append(m[g:m.shape[0] - g, g:m.shape[1] - g])
        return torch.cat(parts, dim=2).cpu().numpy()

    def dump_EM_fields(self, file_name):
        """dump.py:170-207: interior Yee-grid fields (q2, q1, component)."""
        g = self.N_ghost
        yee = self.fields_solver._fetch()[1]
        inner = yee[:, g:yee.shape[1] - g, g:yee.shape[2] - g].permute(1, 2, 0)
        _write_petsc_vec(file_name + '.bin', inner.cpu().numpy().reshape(-1), block=6)

    def load_EM_fields(self, file_name):
        """load.py:45-79: Yee fields from file, halo refresh, cell centring."""
        g = self.N_ghost
        vals = torch.from_numpy(_read_petsc_vec(file_name + '.bin')).to(self.device)
        yee = torch.zeros((6, self.N_q2_local_with_Ng, self.N_q1_local_with_Ng),
                          dtype=torch.float64, device=self.device)
        yee[:, g:yee.shape[1] - g, g:yee.shape[2] - g] = \
            vals.reshape(self.N_q2, self.N_q1, 6).permute(2, 0, 1)
        yee = _periodic_fill_fields(yee, g, self.N_q1, self.N_q2)
        cell = _yee_to_cell(yee)
        self._cell0, self._yee0 = cell.contiguous(), yee.contiguous()
        N.check(self._lib.bolt_fields_set(self._ctx, self._cell0.data_ptr(), self._yee0.data_ptr(),
                                          self._stream()), 'bolt_fields_set')

    # ---- diagnostics (performance_timings.py:9-165) ----------------------------------------
    def performance_timings(self):
        """Device seconds spent in each component since the solver was made
        (performance_test_flag=True): the timestep total and the ghost pass,
        moments, q-stage, p-stage and field solve (CUDA events)."""
        import ctypes
        if self.performance_test_flag:
            buf = (ctypes.c_double * len(N.TIMING_NAMES))()
            N.check(self._lib.bolt_timings(self._ctx, buf), 'bolt_timings')
            self._perf_parts += np.array(list(buf)) * 1e-3
        out = {'timestep': self._perf['time_ts']}
        out.update({k: float(v) for k, v in zip(N.TIMING_NAMES, self._perf_parts)})
        return out

    def print_performance_timings(self, N_iters):
        """performance_timings.py:9-165: seconds per iteration of the step and
        of its parts, as a table, then Spatial Zone Cycles/s.  The reference's
        FVM_SOLVER row splits into RECONSTRUCTION, RIEMANN-SOLVER and
        DFDT_INTEGRATION; those are fused in one kernel here, so the rows are
        the kernels: the q-stage (q-fluxes, BGK, RK combine, moments of the
        result) and, with fields, the p-stage; FIELD-STEP is the FDTD update
        or the electrostatic solve; APPLY_BCS_F + COMMUNICATE_F is the one
        ghost pass that does both."""
        n = max(N_iters, 1)
        t = self.performance_timings()
        ts = t['timestep'] / n
        cells = self.N_q1 * self.N_q2 * self.N_species * self.N_p1 * self.N_p2 * self.N_p3
        rows = [('TIMESTEP', t['timestep']),
                ('FVM_SOLVER', t['q-stage'] + t['p-stage']),
                ('  Q-STAGE (fluxes + BGK + combine)', t['q-stage']),
                ('  P-STAGE (p-fluxes)', t['p-stage']),
                ('FIELD-STEP', t['fields']),
                ('MOMENTS (BGK input)', t['moments']),
                ('APPLY_BCS_F + COMMUNICATE_F', t['ghosts'])]
        w = max(len(r[0]) for r in rows)
        print('%-*s | %-18s | %s' % (w, 'Method', 'Time-Taken(s/iter)', 'Percentage(%)'))
        for name, v in rows:
            pct = 100.0 * v / t['timestep'] if t['timestep'] > 0 else 0.0
            print('%-*s | %-18.6e | %.2f' % (w, name, v / n, pct))
        if ts > 0:
            print('Spatial Zone Cycles/s =', self.N_q1 * self.N_q2 / ts)
            print('Phase-space cell updates/s =', cells / ts)

    def launch_count(self):
        return int(self._lib.bolt_launch_count(self._ctx))

    def paired_launch_count(self):
        """Launches of the paired FP32 stage kernel among launch_count()."""
        return int(self._lib.bolt_paired_launch_count(self._ctx))

    def split_info(self):
        """(nsplit, chunks_per_split) of the q-stage grid's p-split."""
        import ctypes
        n, c = ctypes.c_int(), ctypes.c_int()
        N.check(self._lib.bolt_split_info(self._ctx, ctypes.byref(n), ctypes.byref(c)),
                'bolt_split_info')
        return n.value, c.value

    def synchronize(self):
        rc = self._lib.bolt_status_sync(self._ctx, self._stream())
        N.check(rc, 'bolt_status_sync')


# ---------------------------------------------------------------------------------------------
def _as_list(v, n):
    if torch.is_tensor(v):
        return [float(x) for x in v.reshape(-1)[:n].tolist()]
    return list(v)


def _shift(a, s1, s2):
    """af.shift(a, 0, 0, s1, s2) of Bolt's (..., q1, q2) arrays on this
    module's (..., N_q2g, N_q1g) arrays: circular, out[i] = a[i - s]."""
    if s1:
        a = torch.roll(a, s1, dims=-1)
    if s2:
        a = torch.roll(a, s2, dims=-2)
    return a


def _periodic_fill_fields(a, Ng, N1, N2):
    """communicate_fields with periodic boundaries on (..., Nq2g, Nq1g) arrays."""
    if Ng == 0:
        return a
    out = a.clone()
    i1 = (torch.arange(-Ng, N1 + Ng, device=a.device) % N1) + Ng
    i2 = (torch.arange(-Ng, N2 + Ng, device=a.device) % N2) + Ng
    return out[..., i2, :][..., :, i1]


def _yee_to_cell(y):
    """fields.py:527-557."""
    sh = lambda a, s1, s2: torch.roll(torch.roll(a, s1, dims=-1), s2, dims=-2)
    c = torch.empty_like(y)
    c[0] = 0.5 * (y[0] + sh(y[0], -1, 0))
    c[1] = 0.5 * (y[1] + sh(y[1], 0, -1))
    c[2] = y[2]
    c[3] = 0.5 * (y[3] + sh(y[3], 0, -1))
    c[4] = 0.5 * (y[4] + sh(y[4], -1, 0))
    c[5] = 0.25 * (y[5] + sh(y[5], 0, -1) + sh(y[5], -1, 0) + sh(y[5], -1, -1))
    return c


def _write_petsc_vec(path, values, block=None):
    with open(path, 'wb') as fh:
        np.array([1211214, values.size], dtype='>i4').tofile(fh)
        np.asarray(values, dtype='>f8').tofile(fh)
    if block:
        with open(path + '.info', 'w') as fh:
            fh.write('-vecload_block_size %d\n' % block)


def _read_petsc_vec(path):
    with open(path, 'rb') as fh:
        hdr = np.fromfile(fh, dtype='>i4', count=2)
        if hdr.size != 2 or int(hdr[0]) != 1211214:
            raise IOError('%s is not a PETSc binary Vec' % path)
        return np.fromfile(fh, dtype='>f8', count=int(hdr[1])).astype(np.float64)
