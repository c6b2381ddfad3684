"""q-block decomposition of one run over the ranks of a torch.distributed group.

Bolt distributes a run over MPI ranks with a PETSc DMDA that cuts the q-grid
along q1 and q2, and refreshes the halos with communicate_f before every df/dt
evaluation (nonlinear_solver.py:251-280, communicate.py:8-38).  Here the
ranks form a P1 x P2 grid (rank = r1 + P1 r2, one process per GPU) and each
owns an equal block of the q-grid.  An axis cut into several blocks must be
periodic in the global problem; in the block's own solver it is
``BOLT_BC_EXTERNAL``.  Before every RK stage the N_g halo layers of the stage
input are exchanged with the neighbouring blocks (periodic over the grid), by
point-to-point sends and receives -- NCCL over NVLink between GPUs, gloo
between CPU processes:

* q2 rows, the slowest axis of the layout: each message is one contiguous
  block of N_g (N_q1 + 2 N_g) N_s N_p values, sent from and received into the
  stage buffer itself;
* q1 columns: packed into a contiguous buffer, then unpacked.

Corner cells (ghost in both q1 and q2) are not exchanged: no interior update
reads them, because the q1 and q2 stencils are separate.  An axis kept whole
(P = 1) keeps the global problem's boundary condition.

Electrodynamic fields are distributed like f: each block holds the Yee and
cell-centred fields of its q-cells plus ghosts, and the stage that advances
them (RK4: stage 2; RK2: every other stage) runs in three parts with the Yee
ghosts exchanged before parts 1 and 2 -- where the reference's FDTD update
calls communicate_fields (fields.py:169-180, communicate.py:40-77) -- q1
columns first, then q2 rows over the full width, so corner ghosts (read by
the cell-centring of B3) arrive from the diagonal neighbours.  The fields
must be user-defined initially: the FFT solve of the reference runs only in
serial (fft.py:26-27).

Restart files stay those of a single-process run: PETSc writes a DMDA
vector in the natural (q2, q1, dof) order whatever the process grid
(dump.py:121-168, load.py:10-43), so each rank stores and reads its own rows
of the one shared file (write_block_vec, read_block_vec).  The conserved
totals of the whole run are one FP64 all-reduce of the blocks' sums.
"""

import types

import numpy as np
import torch
import torch.distributed as dist


def _group_info(group):
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def _global_rank(group, r):
    return dist.get_global_rank(group, r) if group is not None else r


def _swap(send_lo, send_hi, recv_lo, recv_hi, lo_rank, hi_rank, group):
    """send_hi -> the hi neighbour, send_lo -> the lo neighbour; recv_lo <- the
    lo neighbour's send_hi, recv_hi <- the hi neighbour's send_lo."""
    ops = [dist.P2POp(dist.isend, send_hi, _global_rank(group, hi_rank), group),
           dist.P2POp(dist.irecv, recv_lo, _global_rank(group, lo_rank), group),
           dist.P2POp(dist.isend, send_lo, _global_rank(group, lo_rank), group),
           dist.P2POp(dist.irecv, recv_hi, _global_rank(group, hi_rank), group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def exchange_q2_halos(store, Ng, group=None, neighbours=None):
    """Fill the N_g ghost rows at both ends of dim 0 of ``store`` (this rank's
    block, (N_q2 + 2 N_g, ...)) with the boundary rows of the blocks below and
    above (``neighbours`` = (down, up) ranks, default the ranks before and
    after this one, periodically); with one rank the block wraps onto itself."""
    rank, world = _group_info(group)
    n2g = store.shape[0]
    bot_ghost, top_ghost = store[:Ng], store[n2g - Ng:]
    bot_inner, top_inner = store[Ng:2 * Ng], store[n2g - 2 * Ng:n2g - Ng]
    down, up = neighbours if neighbours is not None else \
        ((rank - 1) % world, (rank + 1) % world)
    if down == rank and up == rank:
        bot_ghost.copy_(top_inner)
        top_ghost.copy_(bot_inner)
        return
    _swap(bot_inner.contiguous(), top_inner.contiguous(), bot_ghost, top_ghost, down, up, group)


def exchange_q1_halos(store, Ng, group=None, neighbours=None):
    """The same along dim 1 (q1 columns of (N_q2g, N_q1 + 2 N_g, ...);
    ``neighbours`` = (left, right) ranks): the columns travel packed in
    contiguous buffers."""
    rank, world = _group_info(group)
    n1g = store.shape[1]
    left, right = neighbours if neighbours is not None else \
        ((rank - 1) % world, (rank + 1) % world)
    lo_inner, hi_inner = store[:, Ng:2 * Ng], store[:, n1g - 2 * Ng:n1g - Ng]
    if left == rank and right == rank:
        store[:, :Ng].copy_(hi_inner)
        store[:, n1g - Ng:].copy_(lo_inner)
        return
    recv_lo = hi_inner.contiguous().clone()
    recv_hi = lo_inner.contiguous().clone()
    _swap(lo_inner.contiguous(), hi_inner.contiguous(), recv_lo, recv_hi, left, right, group)
    store[:, :Ng].copy_(recv_lo)
    store[:, n1g - Ng:].copy_(recv_hi)


def exchange_field_halos(yee, Ng, external, group=None, q1_neighbours=None,
                         q2_neighbours=None):
    """Yee ghosts of a block's external axes from its neighbours, in place:
    ``yee`` is (..., N_q2 + 2 N_g, N_q1 + 2 N_g); q1 columns over every row
    first, then q2 rows over every column (corners from the diagonal
    neighbours).  ``external`` = (q1 cut, q2 cut); neighbours as for f."""
    rank, world = _group_info(group)
    n2g, n1g = yee.shape[-2], yee.shape[-1]
    if external[0]:
        left, right = q1_neighbours if q1_neighbours is not None else \
            ((rank - 1) % world, (rank + 1) % world)
        lo_in, hi_in = yee[..., Ng:2 * Ng], yee[..., n1g - 2 * Ng:n1g - Ng]
        if left == rank and right == rank:
            yee[..., :Ng], yee[..., n1g - Ng:] = hi_in.clone(), lo_in.clone()
        else:
            recv_lo, recv_hi = torch.empty_like(lo_in.contiguous()), torch.empty_like(hi_in.contiguous())
            _swap(lo_in.contiguous(), hi_in.contiguous(), recv_lo, recv_hi, left, right, group)
            yee[..., :Ng], yee[..., n1g - Ng:] = recv_lo, recv_hi
    if external[1]:
        down, up = q2_neighbours if q2_neighbours is not None else \
            ((rank - 1) % world, (rank + 1) % world)
        lo_in, hi_in = yee[..., Ng:2 * Ng, :], yee[..., n2g - 2 * Ng:n2g - Ng, :]
        if down == rank and up == rank:
            yee[..., :Ng, :], yee[..., n2g - Ng:, :] = hi_in.clone(), lo_in.clone()
        else:
            recv_lo, recv_hi = torch.empty_like(lo_in.contiguous()), torch.empty_like(hi_in.contiguous())
            _swap(lo_in.contiguous(), hi_in.contiguous(), recv_lo, recv_hi, down, up, group)
            yee[..., :Ng, :], yee[..., n2g - Ng:, :] = recv_lo, recv_hi


def _barrier(group):
    if dist.is_available() and dist.is_initialized():
        dist.barrier(group=group)


def write_block_vec(path, block, corner, shape, group=None, create=True, block_size=None,
                    collective=None):
    """Collective write of one PETSc binary Vec holding a whole q-grid array in
    natural order (q2, q1, dof), dof fastest -- what PETSc's VecView writes for
    a DMDA global vector whatever the process grid (dump.py:121-168).

    ``block`` is this rank's interior part, (n2, n1, dof) FP64, starting at
    global interior cell ``corner`` = (j0, i0); ``shape`` = (N_q2, N_q1, dof).
    The creating rank (rank 0 of ``group``) writes the header (int32 class id
    1211214, int32 length, big-endian) and sizes the file; after a barrier
    every rank stores its rows at their offsets.  ``collective=False`` (several
    blocks written from one process; default: whether torch.distributed is
    initialised) skips the barriers: ``create`` then says which call makes the
    file, and that call must come first."""
    rank, _ = _group_info(group)
    N2, N1, dof = (int(x) for x in shape)
    n2, n1 = block.shape[0], block.shape[1]
    j0, i0 = int(corner[0]), int(corner[1])
    if block.shape[2] != dof or j0 < 0 or i0 < 0 or j0 + n2 > N2 or i0 + n1 > N1:
        raise ValueError('block %s at %s does not fit %s' % (block.shape, corner, shape))
    total = N2 * N1 * dof
    if total >= 2 ** 31:
        raise ValueError('a PETSc binary Vec holds fewer than 2^31 values')
    if collective is None:
        collective = dist.is_available() and dist.is_initialized()
    if (rank == 0) if collective else create:
        with open(path, 'wb') as fh:
            np.array([1211214, total], dtype='>i4').tofile(fh)
            fh.truncate(8 + 8 * total)
        with open(path + '.info', 'w') as fh:
            fh.write('-vecload_block_size %d\n' % (block_size or dof))
    if collective:
        _barrier(group)
    mm = np.memmap(path, dtype='>f8', mode='r+', offset=8, shape=(N2, N1, dof))
    mm[j0:j0 + n2, i0:i0 + n1] = block
    mm.flush()
    del mm
    if collective:
        _barrier(group)


def read_block_vec(path, corner, block_shape, shape):
    """This rank's (n2, n1, dof) FP64 part, starting at global interior cell
    ``corner``, of a PETSc binary Vec holding a (N_q2, N_q1, dof) q-grid array
    in natural order (load.py:10-43: PETSc's VecLoad scatters the file to the
    DMDA's ranks; each rank here reads its own rows)."""
    N2, N1, dof = (int(x) for x in shape)
    n2, n1 = int(block_shape[0]), int(block_shape[1])
    j0, i0 = int(corner[0]), int(corner[1])
    with open(path, 'rb') as fh:
        hdr = np.fromfile(fh, dtype='>i4', count=2)
    if hdr.size != 2 or int(hdr[0]) != 1211214:
        raise IOError('%s is not a PETSc binary Vec' % path)
    if int(hdr[1]) != N2 * N1 * dof:
        raise IOError('%s holds %d values, the grid %d' % (path, int(hdr[1]), N2 * N1 * dof))
    mm = np.memmap(path, dtype='>f8', mode='r', offset=8, shape=(N2, N1, dof))
    out = np.array(mm[j0:j0 + n2, i0:i0 + n1], dtype=np.float64)
    del mm
    return out


def slab_of(N_q, q_start, q_end, rank, world):
    """(local N_q, local q_start, local q_end) of block ``rank`` of ``world``
    equal blocks along one axis."""
    if N_q % world:
        raise ValueError('N_q = %d is not divisible by %d blocks' % (N_q, world))
    n = N_q // world
    dq = (q_end - q_start) / N_q
    return n, q_start + rank * n * dq, q_start + (rank + 1) * n * dq


class BlockSolver(object):
    """nonlinear_solver of this rank's q-block of ``physical_system``'s domain,
    on a ``dims`` = (P1, P2) grid of ranks (rank = r1 + P1 r2), stepped stage by
    stage with halo exchanges.  Exposes the local solver as ``.local``.
    ``block=(r1, r2)`` builds that block without a process group (several
    blocks in one process, stepped in lockstep through begin_step /
    stage_input / stage / end_step)."""

    def __init__(self, physical_system, dims, group=None, block=None, external=None,
                 overlap=True):
        from .physical_system import physical_system as PS
        from .nonlinear_solver import nonlinear_solver
        ps = physical_system
        bc = ps.boundary_conditions
        P1, P2 = int(dims[0]), int(dims[1])
        self.dims = (P1, P2)
        # axes whose halos come from exchange(): every cut axis, or as given
        ext1, ext2 = external if external is not None else (P1 > 1, P2 > 1)
        self.external = (bool(ext1), bool(ext2))
        self.group = group
        if block is not None:
            r1, r2 = block
            self.rank = r1 + P1 * r2
        else:
            self.rank, world = _group_info(group)
            if world != P1 * P2:
                raise ValueError('%d ranks for a %d x %d block grid' % (world, P1, P2))
            r1, r2 = self.rank % P1, self.rank // P1
        self.coords = (r1, r2)
        self._collective = block is None and dist.is_available() and dist.is_initialized()
        if ext1 and (bc.in_q1_left != 'periodic' or bc.in_q1_right != 'periodic'):
            raise NotImplementedError('a q1 cut into blocks must be periodic')
        if ext2 and (bc.in_q2_bottom != 'periodic' or bc.in_q2_top != 'periodic'):
            raise NotImplementedError('a q2 cut into blocks must be periodic')
        if getattr(ps.params, 'fields_enabled', False) and (ext1 or ext2):
            # the FFT solves of the reference run only in serial (fft.py:26-27)
            if getattr(ps.params, 'fields_type', 'electrodynamic') != 'electrodynamic':
                raise NotImplementedError('electrostatic fields are solved by a serial FFT')
            if getattr(ps.params, 'fields_initialize', 'fft') != 'user-defined':
                raise NotImplementedError('a run cut into blocks needs user-defined initial '
                                          'fields (the FFT solve is serial)')
        dom = types.ModuleType('domain')
        for k in ('N_p1', 'N_p2', 'N_p3', 'N_ghost'):
            setattr(dom, k, getattr(ps, k))
        for k in ('p1_start', 'p1_end', 'p2_start', 'p2_end', 'p3_start', 'p3_end'):
            setattr(dom, k, list(getattr(ps, k)))
        n1, lo1, hi1 = slab_of(ps.N_q1, ps.q1_start, ps.q1_end, r1, P1)
        n2, lo2, hi2 = slab_of(ps.N_q2, ps.q2_start, ps.q2_end, r2, P2)
        for n, e in ((n1, ext1), (n2, ext2)):
            if e and n < ps.N_ghost:
                raise ValueError('a block of %d cells is thinner than N_ghost = %d'
                                 % (n, ps.N_ghost))
        dom.N_q1, dom.q1_start, dom.q1_end = n1, lo1, hi1
        dom.N_q2, dom.q2_start, dom.q2_end = n2, lo2, hi2
        lbc = types.ModuleType('boundary_conditions')
        lbc.__dict__.update({k: v for k, v in vars(bc).items() if not k.startswith('__')})
        if ext1:
            lbc.in_q1_left = lbc.in_q1_right = 'external'
        if ext2:
            lbc.in_q2_bottom = lbc.in_q2_top = 'external'
        # a solver built on ps.params has turned mass and charge into (1, N_s)
        # arrays (as the reference's does); the block's solver starts from lists
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
        self._peer = False          # peer halos off: exchange before every stage
        self._halos_ready = False
        # exchange on a side stream beside the stage's inner tiles (see
        # overlapped_stage); False: exchange, then the whole stage
        self.overlap = bool(overlap)
        self._comm = None
        # neighbour ranks: (left, right) along q1, (down, up) along q2
        at = lambda a, b: (a % P1) + P1 * (b % P2)
        self.q1_neighbours = (at(r1 - 1, r2), at(r1 + 1, r2))
        self.q2_neighbours = (at(r1, r2 - 1), at(r1, r2 + 1))

    # ---- peer halos: the stage kernels write the neighbours' ghost cells -----
    def peer_buffers(self):
        """Device pointers of this block's f store and RK stage buffers 0, 1
        (what a neighbour passes to bolt_set_peer_halos)."""
        lib, ctx = self.local._lib, self.local._ctx
        return (self.local._fstore.data_ptr(), lib.bolt_stage_buffer(ctx, 0) or 0,
                lib.bolt_stage_buffer(ctx, 1) or 0)

    def set_peer_halos(self, below, above, left=None, right=None):
        """The stage kernels store their boundary rows straight into the lower
        / upper neighbours' buffers (``below`` / ``above``) and their boundary
        columns into the left / right neighbours' (``left`` / ``right``): each
        the neighbour's peer_buffers(), mapped into this process.  Every cut
        axis needs its pair, so that a stage needs no exchange beforehand --
        only an ordering between the blocks' stages.  ``below=None`` switches
        it off."""
        from . import _native as N
        lib, ctx = self.local._lib, self.local._ctx
        if below is None and left is None:
            N.check(lib.bolt_set_peer_halos(ctx, None, None), 'bolt_set_peer_halos')
            N.check(lib.bolt_set_peer_halos_q1(ctx, None, None), 'bolt_set_peer_halos_q1')
            self._peer = False
            return
        if (below is not None) != self.external[1] or (left is not None) != self.external[0]:
            raise ValueError('peer halos: one pair of neighbours per cut axis, none for the others')
        arr = N.ctypes.c_void_p * 3
        if below is not None:
            N.check(lib.bolt_set_peer_halos(ctx, arr(*below), arr(*above)),
                    'bolt_set_peer_halos')
        if left is not None:
            N.check(lib.bolt_set_peer_halos_q1(ctx, arr(*left), arr(*right)),
                    'bolt_set_peer_halos_q1')
        self._peer = True
        self._halos_ready = False

    def enable_peer_halos(self):
        """Collective: map the neighbouring ranks' f and stage buffers into
        this process (CUDA IPC: torch's for f, bolt_ipc_* for the library's
        stage buffers) and switch the peer halos on.  One process per GPU,
        peer access between the GPUs (NVLink)."""
        import ctypes
        from torch.multiprocessing.reductions import reduce_tensor
        from . import _native as N
        lib, ctx = self.local._lib, self.local._ctx
        handles = []
        for i in range(2):
            h = ctypes.create_string_buffer(64)
            N.check(lib.bolt_ipc_get(lib.bolt_stage_buffer(ctx, i), h), 'bolt_ipc_get')
            handles.append(h.raw)
        mine = (reduce_tensor(self.local._fstore), handles)
        _, world = _group_info(self.group)
        every = [None] * world
        dist.all_gather_object(every, mine, group=self.group)
        self._mapped = getattr(self, '_mapped', {})

        def mapped(r):
            if r == self.rank:                              # one slab: its own buffers
                return self.peer_buffers()
            if r not in self._mapped:
                (fn, args), hs = every[r]
                ft = fn(*args)                              # keeps the mapping alive
                ptrs = []
                for h in hs:
                    p = ctypes.c_void_p()
                    N.check(lib.bolt_ipc_open(h, ctypes.byref(p)), 'bolt_ipc_open')
                    ptrs.append(p.value)
                self._mapped[r] = (ft, ptrs)
            ft, ptrs = self._mapped[r]
            return (ft.data_ptr(), ptrs[0], ptrs[1])
        down, up = self.q2_neighbours
        lft, rgt = self.q1_neighbours
        self.set_peer_halos(mapped(down) if self.external[1] else None,
                            mapped(up) if self.external[1] else None,
                            mapped(lft) if self.external[0] else None,
                            mapped(rgt) if self.external[0] else None)

    def disable_peer_halos(self):
        self.set_peer_halos(None, None)
        for _, ptrs in getattr(self, '_mapped', {}).values():
            for p in ptrs:
                self.local._lib.bolt_ipc_close(p)
        self._mapped = {}

    def stage_count(self):
        return self.local.stage_count()

    def begin_step(self):
        self.local._sync_external_edits()

    def stage_input(self, k):
        return self.local.stage_input(k)

    def stage(self, k, dt):
        self.local.stage(k, dt)

    def stage_region(self, k, region, dt):
        """Region 0 (the q-tiles that read no ghost cell of a cut axis), 1 (the
        other tiles) or 2 (the stage's end, after both) of stage k; False when
        the stage cannot be split (nothing was run)."""
        return self.local.stage_region(k, region, dt)

    def overlapped_stage(self, k, dt):
        """Stage k with its input's halo exchange overlapped: the exchange runs
        on a side stream (after everything already queued on the solver's
        stream) and is followed there by the outer tiles, while the tiles
        whose stencils stay inside the block run on the solver's stream, so
        the outer tiles also fill the inner launch's last wave; the solver's
        stream then waits for the side stream and finishes the stage.  Falls
        back to exchange-then-stage when the stage cannot be split (fields,
        the scalar kernel, the first stage after f was set from outside)."""
        loc = self.local
        main = torch.cuda.current_stream(loc.device)
        if self._comm is None:
            self._comm = torch.cuda.Stream(loc.device)
        comm = self._comm
        comm.wait_stream(main)
        with torch.cuda.stream(comm):
            self.exchange(self.stage_input(k))
        split = self.stage_region(k, 0, dt)
        if split:
            with torch.cuda.stream(comm):
                self.stage_region(k, 1, dt)
            main.wait_stream(comm)
            self.stage_region(k, 2, dt)
        else:
            main.wait_stream(comm)
            self.stage(k, dt)
        return split

    def stage_parts(self, k):
        """Parts of stage k: 3 when it advances the fields (the Yee ghosts of
        the cut axes exchanged before parts 1 and 2), else 1."""
        return int(self.local._lib.bolt_stage_parts(self.local._ctx, int(k)))

    def stage_part(self, k, part, dt):
        from . import _native as N
        loc = self.local
        loc.dt = dt
        N.check(loc._lib.bolt_stage_part(loc._ctx, loc._fstore.data_ptr(), float(dt), int(k),
                                         int(part), loc._stream()), 'bolt_stage_part')
        loc._seen_version = loc._fstore._version

    def fields_yee(self):
        """The block's Yee-grid fields on the device, (6, N_q2g, N_q1g) FP64."""
        from . import _native as N
        loc = self.local
        n = 6 * loc.N_q2_local_with_Ng * loc.N_q1_local_with_Ng
        ptr = loc._lib.bolt_fields_yee(loc._ctx)
        t = torch.as_tensor(N.DeviceArray(ptr, n, '<f8'), device=loc.device)
        return t.view(6, loc.N_q2_local_with_Ng, loc.N_q1_local_with_Ng)

    def exchange_fields(self):
        """The Yee ghosts of the cut axes from the neighbouring blocks (every
        rank calls it between the parts of a field-advancing stage)."""
        exchange_field_halos(self.fields_yee(), self.Ng, self.external, self.group,
                             self.q1_neighbours, self.q2_neighbours)

    def end_step(self, dt):
        self.local.time_elapsed += dt
        self.time_elapsed += dt
        self.local.check_divergence()

    def needs_exchange(self, k):
        """Whether stage k's input needs exchange() first: always, unless peer
        halos are on and the halos of f were made current once (the stages
        then keep them current themselves)."""
        return not (self._peer and (k > 0 or self._halos_ready))

    def exchange(self, store):
        """The halo exchanges of one stage input (every rank calls it)."""
        if self.external[1]:
            exchange_q2_halos(store, self.Ng, self.group, self.q2_neighbours)
        if self.external[0]:
            exchange_q1_halos(store, self.Ng, self.group, self.q1_neighbours)
        if self._peer:
            self._halos_ready = True

    def refresh_halos(self):
        """Make the halos of f current (collective): after f was written by
        anything other than the stages."""
        self._halos_ready = False

    def _stage_barrier(self):
        # every rank's stage k has finished (and written the neighbours'
        # ghost rows) before any rank's stage k+1 reads them: a one-element
        # all-reduce ordered on the stream after the stage kernel
        if self.group is not None or (dist.is_available() and dist.is_initialized()):
            if getattr(self, '_token', None) is None:
                self._token = torch.zeros(1, device=self.local.device)
            dist.all_reduce(self._token, group=self.group)

    def strang_timestep(self, dt):
        """One step of the whole distributed run (every rank calls it)."""
        self.begin_step()
        for k in range(self.stage_count()):
            parts = self.stage_parts(k)
            if self.overlap and parts == 1 and self.needs_exchange(k):
                self.overlapped_stage(k, dt)
            else:
                if self.needs_exchange(k):
                    self.exchange(self.stage_input(k))
                for part in range(parts):
                    if part:
                        self.exchange_fields()
                    self.stage_part(k, part, dt)
            if self._peer:
                self._stage_barrier()
        self.end_step(dt)

    lie_timestep = swss_timestep = jia_timestep = strang_timestep

    # ---- the whole run's restart files and totals ----------------------------
    def _grid(self, dof):
        loc = self.local
        corner = (self.coords[1] * loc.N_q2, self.coords[0] * loc.N_q1)
        shape = (self.dims[1] * loc.N_q2, self.dims[0] * loc.N_q1, dof)
        return corner, shape

    def _dof(self):
        loc = self.local
        return loc.N_species * loc.N_p1 * loc.N_p2 * loc.N_p3

    def dump_distribution_function(self, file_name):
        """The whole run's interior f as one PETSc binary Vec, the file a
        single-process run writes (collective; without a process group call
        the blocks in rank order)."""
        data = self.local._interior_store().to(torch.float64).cpu().numpy()
        corner, shape = self._grid(self._dof())
        write_block_vec(file_name + '.bin', data.reshape(data.shape[0], data.shape[1], -1),
                        corner, shape, self.group, create=self.rank == 0,
                        collective=self._collective)

    def load_distribution_function(self, file_name):
        """This block's part of a whole-run f file (dump_distribution_function,
        or a single-process run's); the halos are refreshed before the next
        stage."""
        loc = self.local
        corner, shape = self._grid(self._dof())
        vals = read_block_vec(file_name + '.bin', corner, (loc.N_q2, loc.N_q1), shape)
        loc._load_interior(vals)
        self.refresh_halos()

    def dump_moments(self, file_name):
        """The whole run's dump_moments file (collective, as
        dump_distribution_function)."""
        arr = self.local._moments_interior()
        corner, shape = self._grid(arr.shape[2])
        write_block_vec(file_name + '.bin', arr, corner, shape, self.group,
                        create=self.rank == 0, collective=self._collective)

    def conserved_totals(self):
        """Integrals over the whole q-domain of each species' density, bulk
        momenta (v1, v2, v3) and energy, FP64 (5, N_s): this block's interior
        sums, all-reduced over the group (collective; without a process group
        the block's own share)."""
        loc, g = self.local, self.Ng
        rows = []
        for name in ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy'):
            m = loc._moment_store(name)
            rows.append(m[g:m.shape[0] - g, g:m.shape[1] - g].sum(dim=(0, 1)))
        t = torch.stack(rows) * (float(loc.dq1) * float(loc.dq2))
        if self._collective:
            dist.all_reduce(t, group=self.group)
        return t


class SlabSolver(BlockSolver):
    """BlockSolver cutting q2 only, one slab per rank (``slab=(rank, world)``
    builds that slab without a process group).  With one rank the slab is the
    whole domain and its q2 halo wraps onto itself."""

    def __init__(self, physical_system, group=None, slab=None, overlap=True):
        if slab is not None:
            rank, world = slab
            super(SlabSolver, self).__init__(physical_system, (1, world), group,
                                             block=(0, rank), external=(False, True),
                                             overlap=overlap)
        else:
            _, world = _group_info(group)
            super(SlabSolver, self).__init__(physical_system, (1, world), group,
                                             external=(False, True), overlap=overlap)
        self.world = world
