"""q2 slabs on one GPU: bolt_b200.distributed.SlabSolver against the
periodic nonlinear_solver on the whole domain.

(a) One slab (world 1, no process group): the halo exchange wraps the slab onto
itself, so the run is the periodic run with the q2 ghost rows supplied by a
host-side copy instead of the kernels' periodic images -- equal to the bit.
(b) Two and four slabs in one process, stepped in lockstep with the halo rows
copied between their stage buffers before every RK stage (what the send/recv
exchange does between ranks): interior cells equal the whole-domain run to a
few ulps (the slabs' FP64 moment partial sums may be split differently over
p).  The slabs are 8 rows, so FP32 runs the paired kernel with external q2
ghosts.  Mirror walls along q1 (filled by the ghost pass after every stage)
are covered as well."""

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver

pytestmark = pytest.mark.gpu


def _spec(N_q2, integrator, bc_q1='periodic'):
    return C.make(N_q1=24, N_q2=N_q2, N_p1=8, N_p2=8, N_p3=4, bc_q1=bc_q1,
                  p1_start=[-5.0, -3.0], p1_end=[5.0, 3.0], p2_start=[-5.0, -3.0],
                  p2_end=[5.0, 3.0], p3_start=[-5.0, -3.0], p3_end=[5.0, 3.0],
                  mass=[1.0, 4.0], charge=[0.0, 0.0], p_dim=3, tau=0.01, dt=1e-3,
                  steps=4, integrator=integrator,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=2, u=[0.2, -0.1, 0.05], T=[1.0, 1.5, 0.8]))


def _interior(f, Ng):
    return f[:, :, Ng:-Ng, Ng:-Ng]


def _exchange(slabs, k):
    """Halo rows between slabs held in one process (periodic over the slabs)."""
    Ng = slabs[0].Ng
    xs = [s.stage_input(k) for s in slabs]
    W, n = len(xs), xs[0].shape[0]
    bot = [xs[(r - 1) % W][n - 2 * Ng:n - Ng].clone() for r in range(W)]
    top = [xs[(r + 1) % W][Ng:2 * Ng].clone() for r in range(W)]
    for r in range(W):
        xs[r][:Ng].copy_(bot[r])
        xs[r][n - Ng:].copy_(top[r])


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
@pytest.mark.parametrize('integrator,bc_q1', [('RK4', 'periodic'), ('RK2', 'periodic'),
                                              ('RK4', 'mirror')])
def test_single_slab_equals_periodic_run(precision, integrator, bc_q1):
    from bolt_b200.distributed import SlabSolver
    spec = _spec(16, integrator, bc_q1)
    whole = make_solver(spec, precision)
    slab = SlabSolver(whole.physical_system)
    slab.local.f = whole.f.clone()
    for _ in range(spec['steps']):
        whole.strang_timestep(spec['dt'])
        slab.strang_timestep(spec['dt'])
    Ng = spec['N_ghost']
    assert torch.equal(_interior(slab.local.f, Ng), _interior(whole.f, Ng))
    assert slab.time_elapsed == pytest.approx(whole.time_elapsed)


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-13), ('fp32', 2e-6)])
@pytest.mark.parametrize('world,integrator,bc_q1', [(2, 'RK4', 'periodic'), (4, 'RK4', 'periodic'),
                                                    (2, 'RK2', 'periodic'), (2, 'RK4', 'mirror')])
def test_slabs_in_lockstep_equal_whole_domain(world, integrator, bc_q1, precision, tol):
    from bolt_b200.distributed import SlabSolver
    spec = _spec(8 * world, integrator, bc_q1)
    whole = make_solver(spec, precision)
    slabs = [SlabSolver(whole.physical_system, slab=(r, world)) for r in range(world)]
    Ng, n = spec['N_ghost'], 8
    for r, s in enumerate(slabs):
        s.local.f = whole.f[:, :, :, r * n:r * n + n + 2 * Ng].clone()
    dt = spec['dt']
    for _ in range(spec['steps']):
        whole.strang_timestep(dt)
        for s in slabs:
            s.begin_step()
        for k in range(slabs[0].stage_count()):
            _exchange(slabs, k)
            for s in slabs:
                s.stage(k, dt)
        for s in slabs:
            s.end_step(dt)
    got = torch.cat([_interior(s.local.f, Ng) for s in slabs], dim=3).double()
    ref = _interior(whole.f, Ng).double()
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < tol, err
    # the moments of the slabs, stitched, are the whole domain's
    m = torch.cat([_interior(s.local.compute_moments('density'), Ng) for s in slabs], dim=3)
    mref = _interior(whole.compute_moments('density'), Ng)
    assert float(((m - mref).abs().max() / mref.abs().max())) < tol


def _exchange_blocks(blocks, dims, k):
    """Halo rows, then halo columns, between blocks held in one process."""
    P1, P2 = dims
    Ng = blocks[0].Ng
    xs = [b.stage_input(k) for b in blocks]
    at = lambda a, c: (a % P1) + P1 * (c % P2)
    if P2 > 1:
        n = xs[0].shape[0]
        bot = [xs[at(i % P1, i // P1 - 1)][n - 2 * Ng:n - Ng].clone() for i in range(len(xs))]
        top = [xs[at(i % P1, i // P1 + 1)][Ng:2 * Ng].clone() for i in range(len(xs))]
        for i, x in enumerate(xs):
            x[:Ng].copy_(bot[i])
            x[n - Ng:].copy_(top[i])
    if P1 > 1:
        n = xs[0].shape[1]
        lft = [xs[at(i % P1 - 1, i // P1)][:, n - 2 * Ng:n - Ng].clone() for i in range(len(xs))]
        rgt = [xs[at(i % P1 + 1, i // P1)][:, Ng:2 * Ng].clone() for i in range(len(xs))]
        for i, x in enumerate(xs):
            x[:, :Ng].copy_(lft[i])
            x[:, n - Ng:].copy_(rgt[i])


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-13), ('fp32', 2e-6)])
@pytest.mark.parametrize('dims', [(2, 2), (3, 1)])
def test_blocks_in_lockstep_equal_whole_domain(dims, precision, tol):
    """A P1 x P2 grid of q-blocks (external q1 columns and q2 rows) stepped in
    lockstep on one GPU equals the whole-domain run."""
    from bolt_b200.distributed import BlockSolver
    P1, P2 = dims
    spec = C.make(N_q1=8 * P1, N_q2=8 * P2, N_p1=8, N_p2=8, N_p3=4,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.02, dt=1e-3, steps=4, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=2, u=[0.3, -0.2, 0.05], T=[1.0, 1.4, 0.8]))
    whole = make_solver(spec, precision)
    blocks = [BlockSolver(whole.physical_system, dims, block=(i % P1, i // P1))
              for i in range(P1 * P2)]
    Ng, n = spec['N_ghost'], 8
    for i, b in enumerate(blocks):
        r1, r2 = i % P1, i // P1
        b.local.f = whole.f[:, :, r1 * n:r1 * n + n + 2 * Ng, r2 * n:r2 * n + n + 2 * Ng].clone()
    dt = spec['dt']
    for _ in range(spec['steps']):
        whole.strang_timestep(dt)
        for b in blocks:
            b.begin_step()
        for k in range(blocks[0].stage_count()):
            _exchange_blocks(blocks, dims, k)
            for b in blocks:
                b.stage(k, dt)
        for b in blocks:
            b.end_step(dt)
    cols = [torch.cat([_interior(blocks[r1 + P1 * r2].local.f, Ng) for r2 in range(P2)], dim=3)
            for r1 in range(P1)]
    got = torch.cat(cols, dim=2).double()
    ref = _interior(whole.f, Ng).double()
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < tol, err


def _read_vec(path):
    from bolt_b200.nonlinear_solver import _read_petsc_vec
    return _read_petsc_vec(path)


def _raw(path):
    with open(path, 'rb') as fh:
        return fh.read()


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-13), ('fp32', 2e-6)])
def test_block_grid_restart_files_and_totals(precision, tol, tmp_path):
    """A 2 x 2 block grid writes one whole-run f file and one moments file
    (each block its own rows; blocks called in rank order), loads a
    whole-domain run's f file back block by block, and all-reduces the
    conserved totals: the files hold the blocks' interiors in natural order
    to the bit and equal the whole-domain run's files to the run's
    tolerance; the loaded blocks continue the whole-domain run."""
    from bolt_b200.distributed import BlockSolver
    dims, (P1, P2) = (2, 2), (2, 2)
    spec = C.make(N_q1=16, N_q2=16, N_p1=8, N_p2=8, N_p3=4,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.02, dt=1e-3, steps=2, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=2, u=[0.3, -0.2, 0.05], T=[1.0, 1.4, 0.8]))
    whole = make_solver(spec, precision)
    mk = lambda: [BlockSolver(whole.physical_system, dims, block=(i % P1, i // P1))
                  for i in range(P1 * P2)]
    blocks = mk()
    Ng, n = spec['N_ghost'], 8
    for i, b in enumerate(blocks):
        r1, r2 = i % P1, i // P1
        b.local.f = whole.f[:, :, r1 * n:r1 * n + n + 2 * Ng, r2 * n:r2 * n + n + 2 * Ng].clone()

    def step(bs):
        for b in bs:
            b.begin_step()
        for k in range(bs[0].stage_count()):
            _exchange_blocks(bs, dims, k)
            for b in bs:
                b.stage(k, spec['dt'])
        for b in bs:
            b.end_step(spec['dt'])

    for _ in range(spec['steps']):
        whole.strang_timestep(spec['dt'])
        step(blocks)
    for b in blocks:
        b.dump_distribution_function(str(tmp_path / 'bf'))
        b.dump_moments(str(tmp_path / 'bm'))
    whole.dump_distribution_function(str(tmp_path / 'wf'))
    whole.dump_moments(str(tmp_path / 'wm'))
    # the file holds the blocks' own interiors, natural order, to the bit
    got = _read_vec(str(tmp_path / 'bf.bin')).reshape(16, 16, -1)
    for b in blocks:
        r1, r2 = b.coords
        mine = b.local._interior_store().double().cpu().numpy()
        assert np.array_equal(got[r2 * n:r2 * n + n, r1 * n:r1 * n + n],
                              mine.reshape(n, n, -1))
    assert _raw(str(tmp_path / 'bf.bin'))[:8] == _raw(str(tmp_path / 'wf.bin'))[:8]
    for a, c in (('bf', 'wf'), ('bm', 'wm')):
        x, y = _read_vec(str(tmp_path / (a + '.bin'))), _read_vec(str(tmp_path / (c + '.bin')))
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= tol * np.abs(y).max()
    # conserved totals: the blocks' shares add up to the whole domain's
    one = BlockSolver(whole.physical_system, (1, 1), block=(0, 0))
    one.local.f = whole.f.clone()
    tot = sum(b.conserved_totals() for b in blocks)
    ref = one.conserved_totals()
    assert tot.shape == (5, 1)
    assert float((tot - ref).abs().max()) <= tol * float(ref.abs().max())
    dens = _interior(whole.compute_moments('density'), Ng).sum() * whole.dq1 * whole.dq2
    assert abs(float(ref[0, 0]) - float(dens)) <= 1e-12 * abs(float(dens))
    # load the whole-domain file into fresh blocks and continue together
    fresh = mk()
    for b in fresh:
        b.load_distribution_function(str(tmp_path / 'wf'))
    wf = _interior(whole.f, Ng)
    for b in fresh:
        r1, r2 = b.coords
        assert torch.equal(_interior(b.local.f, Ng),
                           wf[:, :, r1 * n:r1 * n + n, r2 * n:r2 * n + n])
    whole.strang_timestep(spec['dt'])
    step(fresh)
    cols = [torch.cat([_interior(fresh[r1 + P1 * r2].local.f, Ng) for r2 in range(P2)], dim=3)
            for r1 in range(P1)]
    err = float((torch.cat(cols, dim=2).double() - _interior(whole.f, Ng).double()).abs().max()
                / _interior(whole.f, Ng).double().abs().max())
    assert err < tol, err


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-13), ('fp32', 2e-6)])
@pytest.mark.parametrize('world,integrator', [(2, 'RK4'), (3, 'RK4'), (2, 'RK2')])
def test_peer_halo_slabs_equal_whole_domain(world, integrator, precision, tol):
    """Slabs whose stage kernels store their boundary rows straight into the
    neighbours' buffers (bolt_set_peer_halos; the neighbours are other
    contexts on the same GPU here, their buffers at plain device pointers):
    only the first stage input is exchanged, and the run equals the whole
    domain.  FP32 runs the paired kernel's peer images, FP64 the scalar
    kernel's."""
    from bolt_b200.distributed import SlabSolver
    spec = _spec(8 * world, integrator)
    whole = make_solver(spec, precision)
    slabs = [SlabSolver(whole.physical_system, slab=(r, world)) for r in range(world)]
    Ng, n = spec['N_ghost'], 8
    for r, s in enumerate(slabs):
        s.local.f = whole.f[:, :, :, r * n:r * n + n + 2 * Ng].clone()
    for r, s in enumerate(slabs):
        s.set_peer_halos(slabs[(r - 1) % world].peer_buffers(),
                         slabs[(r + 1) % world].peer_buffers())
    dt = spec['dt']
    exchanges = 0
    for _ in range(spec['steps']):
        whole.strang_timestep(dt)
        for s in slabs:
            s.begin_step()
        for k in range(slabs[0].stage_count()):
            if slabs[0].needs_exchange(k):
                _exchange(slabs, k)
                exchanges += 1
                for s in slabs:
                    s._halos_ready = True
            for s in slabs:
                s.stage(k, dt)
        for s in slabs:
            s.end_step(dt)
    assert exchanges == 1
    got = torch.cat([_interior(s.local.f, Ng) for s in slabs], dim=3).double()
    ref = _interior(whole.f, Ng).double()
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < tol, err


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-13), ('fp32', 2e-6)])
@pytest.mark.parametrize('dims,integrator', [((2, 2), 'RK4'), ((3, 1), 'RK4'), ((2, 2), 'RK2')])
def test_peer_halo_blocks_equal_whole_domain(dims, integrator, precision, tol):
    """A P1 x P2 block grid whose stage kernels store their boundary rows and
    columns straight into the neighbours' buffers (bolt_set_peer_halos and
    bolt_set_peer_halos_q1; the neighbours are other contexts on the same
    GPU): only the first stage input is exchanged, and the run equals the
    whole domain.  With P2 = 1 the q2 axis stays periodic inside each block."""
    from bolt_b200.distributed import BlockSolver
    P1, P2 = dims
    spec = C.make(N_q1=8 * P1, N_q2=8 * P2, N_p1=8, N_p2=8, N_p3=4,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.02, dt=1e-3, steps=4, integrator=integrator,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=2, u=[0.3, -0.2, 0.05], T=[1.0, 1.4, 0.8]))
    whole = make_solver(spec, precision)
    blocks = [BlockSolver(whole.physical_system, dims, block=(i % P1, i // P1))
              for i in range(P1 * P2)]
    Ng, n = spec['N_ghost'], 8
    for i, b in enumerate(blocks):
        r1, r2 = i % P1, i // P1
        b.local.f = whole.f[:, :, r1 * n:r1 * n + n + 2 * Ng, r2 * n:r2 * n + n + 2 * Ng].clone()
    if P2 > 1:
        with pytest.raises(ValueError):          # a cut axis without its neighbours
            blocks[0].set_peer_halos(None, None, blocks[1].peer_buffers(),
                                     blocks[1].peer_buffers())
    for b in blocks:
        nb = lambda r: blocks[r].peer_buffers()
        (lft, rgt), (dn, up) = b.q1_neighbours, b.q2_neighbours
        b.set_peer_halos(nb(dn) if P2 > 1 else None, nb(up) if P2 > 1 else None,
                         nb(lft), nb(rgt))
    dt = spec['dt']
    exchanges = 0
    for _ in range(spec['steps']):
        whole.strang_timestep(dt)
        for b in blocks:
            b.begin_step()
        for k in range(blocks[0].stage_count()):
            if blocks[0].needs_exchange(k):
                _exchange_blocks(blocks, dims, k)
                exchanges += 1
                for b in blocks:
                    b._halos_ready = True
            for b in blocks:
                b.stage(k, dt)
        for b in blocks:
            b.end_step(dt)
    assert exchanges == 1
    cols = [torch.cat([_interior(blocks[r1 + P1 * r2].local.f, Ng) for r2 in range(P2)], dim=3)
            for r1 in range(P1)]
    got = torch.cat(cols, dim=2).double()
    ref = _interior(whole.f, Ng).double()
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < tol, err
    for b in blocks:
        b.set_peer_halos(None, None)
        assert b.needs_exchange(1)


def test_peer_halos_through_a_process_group(monkeypatch, tmp_path):
    """The collective set-up and the per-stage ordering of the peer halos on a
    one-rank NCCL group (the single slab is its own neighbour): the IPC handle
    export, all_gather_object, the stage-ordering all-reduce -- equal to the
    periodic run.  (Mapping another process's buffers needs a second GPU.)"""
    import socket
    import torch.distributed as dist
    from bolt_b200.distributed import SlabSolver
    with socket.socket() as sk:
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    monkeypatch.setenv('MASTER_ADDR', '127.0.0.1')
    monkeypatch.setenv('MASTER_PORT', str(port))
    dist.init_process_group('nccl', rank=0, world_size=1)
    try:
        spec = _spec(16, 'RK4')
        whole = make_solver(spec, 'fp32')
        slab = SlabSolver(whole.physical_system)
        slab.local.f = whole.f.clone()
        slab.enable_peer_halos()
        for _ in range(spec['steps']):
            whole.strang_timestep(spec['dt'])
            slab.strang_timestep(spec['dt'])
        Ng = spec['N_ghost']
        assert torch.equal(_interior(slab.local.f, Ng), _interior(whole.f, Ng))
        # the collective restart file (barriers over NCCL) and totals
        slab.dump_distribution_function(str(tmp_path / 's'))
        whole.dump_distribution_function(str(tmp_path / 'w'))
        assert _raw(str(tmp_path / 's.bin')) == _raw(str(tmp_path / 'w.bin'))
        tot = slab.conserved_totals()
        assert tot.device.type == 'cuda' and tot.shape == (5, 2)
        slab.load_distribution_function(str(tmp_path / 'w'))
        slab.strang_timestep(spec['dt'])
        whole.strang_timestep(spec['dt'])
        assert torch.equal(_interior(slab.local.f, Ng), _interior(whole.f, Ng))
        slab.disable_peer_halos()
    finally:
        dist.destroy_process_group()


def _exchange_fields_blocks(blocks, dims):
    """Yee ghosts between blocks held in one process: q1 columns over all rows,
    then q2 rows over all columns (corners from the diagonal neighbours), what
    exchange_field_halos does between ranks."""
    P1, P2 = dims
    Ng = blocks[0].Ng
    ys = [b.fields_yee() for b in blocks]
    at = lambda a, c: (a % P1) + P1 * (c % P2)
    if P1 > 1:
        n = ys[0].shape[2]
        lft = [ys[at(i % P1 - 1, i // P1)][..., n - 2 * Ng:n - Ng].clone() for i in range(len(ys))]
        rgt = [ys[at(i % P1 + 1, i // P1)][..., Ng:2 * Ng].clone() for i in range(len(ys))]
        for i, y in enumerate(ys):
            y[..., :Ng].copy_(lft[i])
            y[..., n - Ng:].copy_(rgt[i])
    if P2 > 1:
        n = ys[0].shape[1]
        bot = [ys[at(i % P1, i // P1 - 1)][:, n - 2 * Ng:n - Ng].clone() for i in range(len(ys))]
        top = [ys[at(i % P1, i // P1 + 1)][:, Ng:2 * Ng].clone() for i in range(len(ys))]
        for i, y in enumerate(ys):
            y[:, :Ng].copy_(bot[i])
            y[:, n - Ng:].copy_(top[i])


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-12), ('fp32', 2e-6)])
@pytest.mark.parametrize('dims,integrator', [((2, 2), 'RK4'), ((2, 1), 'RK2'), ((1, 3), 'RK4')])
def test_field_blocks_in_lockstep_equal_whole_domain(dims, integrator, precision, tol):
    """FDTD-coupled q-blocks on one GPU (user-defined initial E and B): f
    exchanged before every stage, the Yee ghosts between the three parts of
    the field-advancing stage; f, the Yee-grid and the cell-centred fields
    equal the whole-domain run (the blocks evaluate the initial field
    functions at their own coordinates, which differ from the whole grid's
    in the last bits, hence 1e-12 in FP64)."""
    from bolt_b200.distributed import BlockSolver
    P1, P2 = dims
    spec = C.make(N_q1=8 * P1, N_q2=8 * P2, N_p1=8, N_p2=6, N_p3=1,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
                  fields_enabled=True, fields_initialize='user-defined', field_init='E_B',
                  tau=0.1, dt=1e-3, steps=3, integrator=integrator,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.05, k1=1, k2=1, T=[1.0, 1.2, 1.0]))
    whole = make_solver(spec, precision)
    blocks = [BlockSolver(whole.physical_system, dims, block=(i % P1, i // P1))
              for i in range(P1 * P2)]
    Ng, n = spec['N_ghost'], 8
    for i, b in enumerate(blocks):
        r1, r2 = i % P1, i // P1
        b.local.f = whole.f[:, :, r1 * n:r1 * n + n + 2 * Ng, r2 * n:r2 * n + n + 2 * Ng].clone()
    dt = spec['dt']
    for _ in range(spec['steps']):
        whole.strang_timestep(dt)
        for b in blocks:
            b.begin_step()
        for k in range(blocks[0].stage_count()):
            _exchange_blocks(blocks, dims, k)
            parts = blocks[0].stage_parts(k)
            assert all(b.stage_parts(k) == parts for b in blocks)
            for part in range(parts):
                if part:
                    _exchange_fields_blocks(blocks, dims)
                for b in blocks:
                    b.stage_part(k, part, dt)
        for b in blocks:
            b.end_step(dt)
    torch.cuda.synchronize()

    def stitched(arrs):
        rows = [torch.cat([arrs[r1 + P1 * r2] for r1 in range(P1)], dim=-1) for r2 in range(P2)]
        return torch.cat(rows, dim=-2)
    # f as (q2, q1, ...) interiors
    fs = [b.local._fstore[Ng:Ng + n, Ng:Ng + n].double().permute(2, 3, 0, 1) for b in blocks]
    got = stitched(fs)
    ref = whole._fstore[Ng:-Ng, Ng:-Ng].double().permute(2, 3, 0, 1)
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < tol, ('f', err)
    yw = whole.fields_solver.yee_grid_EM_fields[:, 0].permute(0, 2, 1)[:, Ng:-Ng, Ng:-Ng]
    yb = stitched([b.fields_yee()[:, Ng:Ng + n, Ng:Ng + n] for b in blocks])
    ftol = 1e-12 if precision == 'fp64' else 1e-4
    err = float((yb - yw).abs().max() / yw.abs().max())
    assert err < ftol, ('yee', err)


# ---------------------------------------------------------------------------
# Exchange overlapped with the inner tiles (bolt_stage_region)
# ---------------------------------------------------------------------------
def _poison_ghosts(blocks, dims, k):
    """NaN into the cut axes' ghost cells of every block's stage-k input: a
    region-0 update that read any of them would carry the NaN into f."""
    P1, P2 = dims
    Ng = blocks[0].Ng
    for b in blocks:
        x = b.stage_input(k)
        if P2 > 1:
            x[:Ng] = float('nan')
            x[x.shape[0] - Ng:] = float('nan')
        if P1 > 1:
            x[:, :Ng] = float('nan')
            x[:, x.shape[1] - Ng:] = float('nan')


@pytest.mark.parametrize('precision,tol', [('fp32', 2e-6), ('fp64-fast', 1e-12)])
@pytest.mark.parametrize('dims,integrator', [((1, 2), 'RK4'), ((2, 2), 'RK4'), ((1, 3), 'RK2')])
def test_inner_tiles_need_no_ghosts(dims, integrator, precision, tol):
    """Blocks of 24x24 q-cells (3x3 tiles) in lockstep: per stage, the cut axes'
    ghost cells of every stage input are set to NaN, region 0 runs, then the
    halos are exchanged and regions 1 and 2 run -- what a rank does while its
    exchange is in flight.  After three steps the blocks equal the
    whole-domain run, so region 0 read no ghost cell; every stage after the
    first step split."""
    from bolt_b200.distributed import BlockSolver
    P1, P2 = dims
    n = 24
    spec = C.make(N_q1=n * P1, N_q2=n * P2, N_p1=8, N_p2=8, N_p3=4,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=1e-3, steps=3, integrator=integrator,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=1, u=[0.2, -0.1, 0.05]))
    whole = make_solver(spec, precision)
    Ng = spec['N_ghost']
    blocks = [BlockSolver(whole.physical_system, dims, block=(r % P1, r // P1))
              for r in range(P1 * P2)]
    for r, b in enumerate(blocks):
        r1, r2 = r % P1, r // P1
        b.local.f = whole.f[:, :, r1 * n:r1 * n + n + 2 * Ng, r2 * n:r2 * n + n + 2 * Ng].clone()
    dt = spec['dt']
    split = []
    for step in range(spec['steps']):
        whole.strang_timestep(dt)
        for b in blocks:
            b.begin_step()
        for k in range(blocks[0].stage_count()):
            _poison_ghosts(blocks, dims, k)
            done = [b.stage_region(k, 0, dt) for b in blocks]
            _exchange_blocks(blocks, dims, k)
            for b, d in zip(blocks, done):
                if d:
                    assert b.stage_region(k, 1, dt) and b.stage_region(k, 2, dt)
                else:
                    b.stage(k, dt)
            if step > 0:
                split += done
        for b in blocks:
            b.end_step(dt)
    assert split and all(split)
    cols = [torch.cat([_interior(blocks[r1 + P1 * r2].local.f, Ng) for r2 in range(P2)], dim=3)
            for r1 in range(P1)]
    got = torch.cat(cols, dim=2).double()
    ref = _interior(whole.f, Ng).double()
    err = float((got - ref).abs().max() / ref.abs().max())
    assert err < tol, err


@pytest.mark.parametrize('precision', ['fp32', 'fp64-fast'])
@pytest.mark.parametrize('bc_q1', ['periodic', 'mirror'])
def test_overlapped_single_slab_equals_periodic_run(precision, bc_q1):
    """One slab (no process group) stepped by strang_timestep with the exchange
    and then the outer tiles on a side stream beside the inner tiles: the run
    equals the periodic solver to the bit, and the stages after the first
    split."""
    from bolt_b200.distributed import SlabSolver
    spec = _spec(24, 'RK4', bc_q1)
    whole = make_solver(spec, precision)
    slab = SlabSolver(whole.physical_system)
    assert slab.overlap
    slab.local.f = whole.f.clone()
    calls = []
    orig = slab.overlapped_stage
    slab.overlapped_stage = lambda k, dt: calls.append(orig(k, dt))
    for _ in range(spec['steps']):
        whole.strang_timestep(spec['dt'])
        slab.strang_timestep(spec['dt'])
    torch.cuda.synchronize()
    Ng = spec['N_ghost']
    assert torch.equal(_interior(slab.local.f, Ng), _interior(whole.f, Ng))
    assert len(calls) == 4 * spec['steps'] and calls[0] is False and all(calls[1:])


def test_stage_region_refuses_fp64_reference_order():
    """The FP64 reference-order kernel has no tile regions: region 0 returns
    False (nothing run) and the stage runs whole after the exchange."""
    from bolt_b200.distributed import SlabSolver
    spec = _spec(24, 'RK4')
    whole = make_solver(spec, 'fp64')
    slab = SlabSolver(whole.physical_system)
    slab.local.f = whole.f.clone()
    for _ in range(2):
        whole.strang_timestep(spec['dt'])
        slab.strang_timestep(spec['dt'])
    assert not slab.stage_region(1, 0, spec['dt'])
    Ng = spec['N_ghost']
    assert torch.equal(_interior(slab.local.f, Ng), _interior(whole.f, Ng))
