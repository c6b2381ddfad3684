"""q2-slab decomposition of one run over the ranks of a torch.distributed group.

Bolt distributes a run over MPI ranks with a PETSc DMDA whose halos are
exchanged by ``communicate_f`` before every df/dt evaluation
(nonlinear_solver.py:251-280, communicate.py:8-38).  Here the q2 axis is cut
into equal slabs, one per rank (one process per GPU); each rank's solver sees
q2 as ``BOLT_BC_EXTERNAL`` and, before every RK stage, the N_g ghost rows of
the stage input are exchanged with the neighbouring slabs (periodic over the
ranks) by point-to-point sends and receives -- NCCL over NVLink between GPUs,
gloo between CPU processes.  Rows are the slowest axis of the layout, so every
message is one contiguous block of N_g (N_q1 + 2 N_g) N_s N_p values sent from
and received into the stage buffer itself.  q1 stays whole and periodic on
every rank; fields are not distributed (the reference's FFT initial solve is
serial too, fft.py:26-27).
"""

import types

import torch.distributed as dist


def _group_info(group):
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def exchange_q2_halos(store, Ng, group=None):
    """Fill the N_g ghost rows at both ends of dim 0 of ``store`` (this rank's
    slab, (N_q2 + 2 N_g, ...)) with the boundary rows of the neighbouring
    ranks' slabs; with one rank the slab wraps onto itself (periodic q2)."""
    rank, world = _group_info(group)
    n2g = store.shape[0]
    bot_ghost, top_ghost = store[:Ng], store[n2g - Ng:]
    bot_inner, top_inner = store[Ng:2 * Ng], store[n2g - 2 * Ng:n2g - Ng]
    if world == 1:
        bot_ghost.copy_(top_inner)
        top_ghost.copy_(bot_inner)
        return
    up = dist.get_global_rank(group, (rank + 1) % world) if group is not None else (rank + 1) % world
    down = dist.get_global_rank(group, (rank - 1) % world) if group is not None else (rank - 1) % world
    ops = [dist.P2POp(dist.isend, top_inner.contiguous(), up, group),
           dist.P2POp(dist.irecv, bot_ghost, down, group),
           dist.P2POp(dist.isend, bot_inner.contiguous(), down, group),
           dist.P2POp(dist.irecv, top_ghost, up, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def slab_of(N_q2, q2_start, q2_end, rank, world):
    """(local N_q2, local q2_start, local q2_end) of rank's slab."""
    if N_q2 % world:
        raise ValueError('N_q2 = %d is not divisible by %d ranks' % (N_q2, world))
    n = N_q2 // world
    dq2 = (q2_end - q2_start) / N_q2
    return n, q2_start + rank * n * dq2, q2_start + (rank + 1) * n * dq2


class SlabSolver(object):
    """nonlinear_solver of this rank's q2 slab of ``physical_system``'s domain
    (q2 periodic in the global problem), stepped stage by stage with halo
    exchanges.  Exposes the local solver as ``.local``.  ``slab=(rank, world)``
    builds that slab without a process group (several slabs in one process,
    stepped in lockstep through begin_step / stage_input / stage / end_step)."""

    def __init__(self, physical_system, group=None, slab=None):
        from .physical_system import physical_system as PS
        from .nonlinear_solver import nonlinear_solver
        ps = physical_system
        bc = ps.boundary_conditions
        if bc.in_q2_bottom != 'periodic' or bc.in_q2_top != 'periodic':
            raise NotImplementedError('the q2 slabs split a periodic q2 axis')
        if getattr(ps.params, 'fields_enabled', False):
            raise NotImplementedError('fields are not distributed')
        self.group = group
        self.rank, self.world = slab if slab is not None else _group_info(group)
        dom = types.ModuleType('domain')
        for k in ('N_q1', 'q1_start', 'q1_end', 'N_p1', 'N_p2', 'N_p3', 'N_ghost'):
            setattr(dom, k, getattr(ps, k))
        for k in ('p1_start', 'p1_end', 'p2_start', 'p2_end', 'p3_start', 'p3_end'):
            setattr(dom, k, list(getattr(ps, k)))
        n, lo, hi = slab_of(ps.N_q2, ps.q2_start, ps.q2_end, self.rank, self.world)
        if n < ps.N_ghost:
            raise ValueError('a slab of %d rows is thinner than N_ghost = %d' % (n, ps.N_ghost))
        dom.N_q2, dom.q2_start, dom.q2_end = n, lo, hi
        lbc = types.ModuleType('boundary_conditions')
        lbc.__dict__.update({k: v for k, v in vars(bc).items() if not k.startswith('__')})
        lbc.in_q2_bottom = lbc.in_q2_top = 'external'
        # a solver built on ps.params has turned mass and charge into (1, N_s)
        # arrays (as the reference's does); the slab's solver starts from lists
        lp = types.ModuleType('params')
        lp.__dict__.update({k: v for k, v in vars(ps.params).items() if not k.startswith('__')})
        for k in ('mass', 'charge'):
            v = getattr(lp, k)
            if hasattr(v, 'reshape'):
                setattr(lp, k, [float(x) for x in v.reshape(-1).tolist()])
        local = PS(dom, lbc, lp, ps.initial_conditions, ps.advection_term,
                   ps.source, ps.moments)
        self.local = nonlinear_solver(local)
        self.Ng = self.local.N_ghost
        self.time_elapsed = 0.0

    def stage_count(self):
        return self.local.stage_count()

    def begin_step(self):
        self.local._sync_external_edits()

    def stage_input(self, k):
        return self.local.stage_input(k)

    def stage(self, k, dt):
        self.local.stage(k, dt)

    def end_step(self, dt):
        self.local.time_elapsed += dt
        self.time_elapsed += dt
        self.local.check_divergence()

    def strang_timestep(self, dt):
        """One step of the whole distributed run (every rank calls it)."""
        self.begin_step()
        for k in range(self.stage_count()):
            exchange_q2_halos(self.stage_input(k), self.Ng, self.group)
            self.stage(k, dt)
        self.end_step(dt)

    lie_timestep = swss_timestep = jia_timestep = strang_timestep
