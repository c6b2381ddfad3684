"""Ragged batch of independent 1D1V runs, advanced together on one GPU.

Bolt advances one system per ``nonlinear_solver`` (nonlinear_solver.py:67);
a parameter sweep is a Python loop over such runs.  ``BatchSolver`` takes a
list of Bolt ``physical_system`` objects -- each a 1D1V problem (q1 periodic,
N_q2 = N_p2 = N_p3 = 1, one species, p_dim = 1, fields off) with the
nonrelativistic_boltzmann plug-ins, WENO5 + upwind/LLF in q, RK4 and FP32
precision -- plus one dt per run, and advances all of them with the batch
kernels of libbolt_b200.so (include/bolt_b200.h, "Ragged batch"): FP32 f with
FP64 moments, one launch per RK stage over the packed runs, ``run(nsteps)``
replayed as one CUDA graph.  Grids, ranges, tau and dt may differ per run.

Per run, ``f(r)`` is a torch view of the run's f in Bolt's layout
(N_p1, 1, N_q1 + 2 N_g, 1) and ``compute_moments(name, r)`` returns the
moment over the interior q-cells, shape (1, 1, N_q1, 1), FP64.

The launch schedule is chosen by an autotuner (``autotune``).  It covers the
q-cells per work item (the pencil-to-block tile), the persistent CTAs per SM
and the queue order. Before the first ``run``, each candidate is timed on
the batch itself, a few steps from its current state with CUDA events, and
the state is restored afterwards. The fastest is kept, and it is remembered
for batches with the same run shapes in this process.  Every schedule gives
bit-identical results.
"""

import torch

from . import _native as N
from .nonlinear_solver import nonlinear_solver, _plugin_ok

BATCH_MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')

# schedules the autotuner times: (q-cells per work item, CTAs per SM, queue
# order 1 = longest items first / 0 = run by run)
TUNE_CANDIDATES = tuple((tq, c, o) for tq in (8, 16, 32, 64) for c in (1, 2, 4, 8, 16)
                        for o in (1, 0))
_TUNED = {}    # (collisional, run shapes) -> schedule chosen in this process


class _RunGrid(object):
    """The attributes nonlinear_solver._build_grids reads, for one run."""

    def __init__(self, ps, device):
        self.physical_system = ps
        self.device = device
        self.N_ghost = ps.N_ghost
        self.N_q1, self.N_q2 = ps.N_q1, ps.N_q2
        self.q1_start, self.q2_start = ps.q1_start, ps.q2_start
        self.dq1, self.dq2 = ps.dq1, ps.dq2
        self.N_p1, self.N_p2, self.N_p3 = ps.N_p1, ps.N_p2, ps.N_p3
        self.N_species = ps.N_species


def _check_system(ps, r):
    params = ps.params
    bc = ps.boundary_conditions

    def need(cond, what):
        if not cond:
            raise NotImplementedError('batch run %d: %s' % (r, what))
    need(ps.N_q2 == 1 and ps.N_p2 == 1 and ps.N_p3 == 1, '1D1V only (N_q2 = N_p2 = N_p3 = 1)')
    need(ps.N_species == 1, 'one species')
    need(int(params.p_dim) == 1, 'p_dim = 1')
    need(ps.N_ghost == 3, 'N_ghost = 3')
    need(bc.in_q1_left == 'periodic' and bc.in_q1_right == 'periodic', 'periodic q1')
    need(not getattr(params, 'fields_enabled', False), 'fields disabled')
    need(params.solver_method_in_q == 'FVM', 'FVM in q')
    need(params.reconstruction_method_in_q == 'weno5', 'WENO5 in q')
    need(getattr(params, 'riemann_solver_in_q', 'upwind-flux') in N.FLUX, 'upwind or LLF flux')
    need(getattr(params, 'time_integrator', 'RK2') == 'RK4', 'RK4')
    need(getattr(params, 'precision', 'fp64') in ('fp32', 'float32', 'single'),
         'FP32 f (FP64 moments)')
    need(_plugin_ok(ps.C_q, 'advection_terms', 'C_q'), 'nonrelativistic_boltzmann C_q')
    need(_plugin_ok(ps.source, 'collision_operator', 'BGK'), 'nonrelativistic_boltzmann BGK')


class BatchSolver(object):

    def __init__(self, systems, dts, autotune=True):
        if not torch.cuda.is_available():
            raise RuntimeError('bolt_b200 runs on a CUDA device (sm_100a); no CUDA device '
                               'is available and there is no CPU fallback')
        systems = list(systems)
        dts = [float(d) for d in dts]
        if len(systems) == 0 or len(dts) != len(systems):
            raise ValueError('one dt per system is required')
        self._lib = N.load()
        self.device = torch.device('cuda', torch.cuda.current_device())
        self.systems = systems
        self.nruns = len(systems)
        srcs = {bool(getattr(ps.params, 'source_enabled', False)) for ps in systems}
        if len(srcs) != 1:
            raise NotImplementedError('all runs of a batch either collide (BGK) or not')
        self.source_enabled = srcs.pop()

        grids, f0s = [], []
        runs = (N.BoltBatchRun * self.nruns)()
        for r, ps in enumerate(systems):
            _check_system(ps, r)
            params = ps.params
            g = _RunGrid(ps, self.device)
            nonlinear_solver._build_grids(g, params)
            R = runs[r]
            R.N_q1, R.N_p1 = ps.N_q1, ps.N_p1
            R.q1_start, R.q1_end = ps.q1_start, ps.q1_end
            R.p1_start, R.p1_end = ps.p1_start[0], ps.p1_end[0]
            R.p2_center = ps.p2_start[0] + 0.5 * ps.dp2[0]
            R.p3_center = ps.p3_start[0] + 0.5 * ps.dp3[0]
            R.dp2, R.dp3 = ps.dp2[0], ps.dp3[0]
            R.mass = float(params.mass if not isinstance(params.mass, (list, tuple))
                           else params.mass[0])
            R.boltzmann_constant = float(params.boltzmann_constant)
            R.dt = dts[r]
            R.tau = 1.0
            if self.source_enabled:
                tau = torch.as_tensor(params.tau(g.q1_center, g.q2_center, g.p1_center,
                                                 g.p2_center, g.p3_center),
                                      dtype=torch.float64).reshape(-1)
                if not bool(torch.all(tau == tau[0])):
                    raise NotImplementedError('batch run %d: constant tau only' % r)
                R.tau = float(tau[0])
            f0 = ps.initial_conditions.initialize_f(g.q1_center, g.q2_center, g.p1_center,
                                                    g.p2_center, g.p3_center, params)
            grids.append(g)
            f0s.append(f0)

        b = N.ctypes.c_void_p()
        N.check(self._lib.bolt_batch_create(runs, self.nruns, 1 if self.source_enabled else 0,
                                            N.ctypes.byref(b)), 'bolt_batch_create')
        self._b = b
        self._runs = runs
        count = self._lib.bolt_batch_f_count(b)
        self._flat = torch.as_tensor(N.DeviceArray(self._lib.bolt_batch_f(b), count, '<f4'),
                                     device=self.device)
        self._f_off = [int(self._lib.bolt_batch_f_offset(b, r)) for r in range(self.nruns)]
        self._q_off = [int(self._lib.bolt_batch_q_offset(b, r)) for r in range(self.nruns)]
        self._q_count = int(self._lib.bolt_batch_q_count(b))
        self.dt = dts
        self.time_elapsed = [0.0] * self.nruns
        self._measure = [(R.dp3 * R.dp2) * ((R.p1_end - R.p1_start) / R.N_p1) for R in runs]
        for r, f0 in enumerate(f0s):
            # Bolt's grids carry N_g ghost rows in q2 even for N_q2 = 1; the
            # batch stores the interior q2 row only
            Ng = systems[r].N_ghost
            f0 = torch.as_tensor(f0, device=self.device)
            if f0.dim() == 4 and f0.shape[3] == 1 + 2 * Ng:
                f0 = f0[:, :, :, Ng:Ng + 1]
            self.f(r).copy_(torch.broadcast_to(f0, self.f(r).shape))
        self._prepared = False
        self._seen = self._flat._version
        self._key = (self.source_enabled, tuple((R.N_q1, R.N_p1) for R in runs))
        self.tuning = None
        self._tune_pending = bool(autotune)
        if autotune and self._key in _TUNED:
            self.set_schedule(*_TUNED[self._key])
            self._tune_pending = False

    def __del__(self):
        try:
            if getattr(self, '_b', None) is not None:
                self._lib.bolt_batch_destroy(self._b)
                self._b = None
        except Exception:
            pass

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def f(self, r):
        """Run r's distribution function, a view with Bolt's layout
        (N_p1, 1, N_q1 + 2 N_g, 1) of the packed device buffer."""
        R = self._runs[r]
        n = (R.N_q1 + 6) * R.N_p1
        store = self._flat[self._f_off[r]:self._f_off[r] + n].view(R.N_q1 + 6, R.N_p1)
        return store.permute(1, 0).unsqueeze(1).unsqueeze(3)

    # ---- launch schedule ------------------------------------------------------------
    def set_schedule(self, tile_cells, ctas_per_sm, lpt_order):
        N.check(self._lib.bolt_batch_set_schedule(self._b, int(tile_cells), int(ctas_per_sm),
                                                  int(lpt_order)), 'bolt_batch_set_schedule')

    def schedule(self):
        """(q-cells per work item, CTAs launched, queue order)."""
        v = [N.ctypes.c_int() for _ in range(3)]
        N.check(self._lib.bolt_batch_get_schedule(self._b, *[N.ctypes.byref(x) for x in v]),
                'bolt_batch_get_schedule')
        return tuple(x.value for x in v)

    def autotune(self, steps=4, repeats=2, candidates=TUNE_CANDIDATES):
        """Time every candidate schedule over ``steps`` RK4 steps of this batch
        (best of ``repeats`` CUDA-event timings, after one untimed replay that
        also captures the graph) from the current f, then restore f and keep
        the fastest.  Returns [((tile_cells, ctas, order), ms per step), ...]."""
        saved = self._flat.clone()
        stream = self._stream()
        results, seen = [], set()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for tq, cps, order in candidates:
            self.set_schedule(tq, cps, order)
            eff = self.schedule()
            if eff in seen:
                continue
            seen.add(eff)
            self._flat.copy_(saved)
            N.check(self._lib.bolt_batch_prepare(self._b, stream), 'bolt_batch_prepare')
            N.check(self._lib.bolt_batch_run(self._b, steps, stream), 'bolt_batch_run')
            best = float('inf')
            for _ in range(repeats):
                e0.record()
                N.check(self._lib.bolt_batch_run(self._b, steps, stream), 'bolt_batch_run')
                e1.record()
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1) / steps)
            results.append(((tq, cps, order), eff, best))
        (tq, cps, order), eff, ms = min(results, key=lambda x: x[2])
        self.set_schedule(tq, cps, order)
        self._flat.copy_(saved)
        self._prepared = False
        self._seen = -1
        self._lib.bolt_batch_divergence_flag(self._b)       # tuning steps leave no flag
        _TUNED[self._key] = (tq, cps, order)
        self.tuning = {'chosen': {'tile_cells': eff[0], 'ctas': eff[1], 'lpt_order': eff[2],
                                  'ms_per_step': ms},
                       'candidates': [{'tile_cells': e[0], 'ctas': e[1], 'lpt_order': e[2],
                                       'ms_per_step': t} for _, e, t in results]}
        self._tune_pending = False
        return results

    def run(self, nsteps):
        """Advance every run by nsteps RK4 steps of its own dt."""
        if self._tune_pending:
            self.autotune()
        if not self._prepared or self._flat._version != self._seen:
            N.check(self._lib.bolt_batch_prepare(self._b, self._stream()), 'bolt_batch_prepare')
            self._prepared = True
            self._seen = self._flat._version
        N.check(self._lib.bolt_batch_run(self._b, int(nsteps), self._stream()), 'bolt_batch_run')
        for r in range(self.nruns):
            self.time_elapsed[r] += nsteps * self.dt[r]
        if self._lib.bolt_batch_divergence_flag(self._b):
            raise SystemExit('Solver Diverging!')

    def synchronize(self):
        torch.cuda.current_stream(self.device).synchronize()
        if self._lib.bolt_batch_divergence_flag(self._b):
            raise SystemExit('Solver Diverging!')

    def compute_moments(self, moment_name, r):
        """Moment of run r over its interior q-cells (compute_moments.py:7-59),
        shape (1, 1, N_q1, 1), FP64."""
        if moment_name not in BATCH_MOMENTS:
            raise NotImplementedError('batch moments: %s' % (BATCH_MOMENTS,))
        if not self._prepared or self._flat._version != self._seen:
            N.check(self._lib.bolt_batch_prepare(self._b, self._stream()), 'bolt_batch_prepare')
            self._prepared = True
            self._seen = self._flat._version
        out = torch.empty((self._q_count, 5), dtype=torch.float64, device=self.device)
        N.check(self._lib.bolt_batch_moments(self._b, out.data_ptr(), self._stream()),
                'bolt_batch_moments')
        R = self._runs[r]
        col = BATCH_MOMENTS.index(moment_name)
        vals = out[self._q_off[r]:self._q_off[r] + R.N_q1, col] * self._measure[r]
        return vals.reshape(1, 1, R.N_q1, 1)
