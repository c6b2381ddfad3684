"""q2-slab decomposition on the CPU with two gloo ranks (127.0.0.1):
bolt_b200.distributed.exchange_q2_halos fills each slab's ghost rows from the
neighbouring slabs (periodic over the ranks), and the oracle advanced slab by
slab -- q2 as 'external', halos exchanged before every RK stage exactly where
SlabSolver exchanges them -- equals the oracle advanced on the whole domain."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _spec():
    import cases as C
    return C.make(N_q1=8, N_q2=16, N_p1=8, N_p2=4, N_p3=4,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-5.0], p3_end=[5.0], mass=[1.0], charge=[0.0], p_dim=3,
                  tau=0.05, dt=1e-3, steps=3, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.1, k1=1, k2=2, noise=1e-3, seed=3, u=[0.2, -0.1, 0.05]))


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    sys.path[:0] = [ROOT, HERE, os.path.join(HERE, 'golden')]
    import torch
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from bolt_b200.distributed import exchange_q2_halos, slab_of
        # 1) the exchange itself: rows hold (rank, row) labels
        Ng, n = 3, 4
        t = torch.zeros((n + 2 * Ng, 5), dtype=torch.float64)
        for j in range(n):
            t[Ng + j] = 100 * rank + j
        exchange_q2_halos(t, Ng)
        down, up = (rank - 1) % world, (rank + 1) % world
        ok_ex = all(float(t[g, 0]) == 100 * down + (n - Ng + g) for g in range(Ng)) and \
            all(float(t[n + Ng + g, 0]) == 100 * up + g for g in range(Ng))
        # 2) the oracle advanced slab by slab
        import cases as C
        from oracle.bolt_oracle import Oracle
        spec = _spec()
        fg = C.initial_f(spec)
        nloc, lo, hi = slab_of(spec['N_q2'], spec['q2_start'], spec['q2_end'], rank, world)
        local = dict(spec, N_q2=nloc, q2_start=lo, q2_end=hi, bc_q2='external')
        f0 = fg[rank * nloc: rank * nloc + nloc + 2 * Ng].copy()
        o = Oracle(local, f0)

        def exchange(x):
            x = np.ascontiguousarray(x)
            exchange_q2_halos(torch.from_numpy(x), Ng)
            return x
        o.exchange = exchange
        for _ in range(spec['steps']):
            o.step(spec['dt'])
        out.put((rank, ok_ex, o.f[Ng:Ng + nloc, Ng:-Ng].copy()))
    finally:
        dist.destroy_process_group()


def test_slabs_over_two_gloo_ranks_equal_the_whole_domain():
    import sys
    sys.path[:0] = [ROOT, HERE, os.path.join(HERE, 'golden')]
    import cases as C
    from oracle.bolt_oracle import Oracle
    world = 2
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((out.get(timeout=300) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[1] for r in res), 'halo rows'
    spec = _spec()
    o = Oracle(spec, C.initial_f(spec))
    for _ in range(spec['steps']):
        o.step(spec['dt'])
    Ng = spec['N_ghost']
    whole = o.f[Ng:Ng + spec['N_q2'], Ng:-Ng]     # interior cells
    slabs = np.concatenate([r[2] for r in res], axis=0)
    assert np.max(np.abs(slabs - whole)) <= 1e-15 * np.max(np.abs(whole))


def _block_rank_main(rank, dims, port, out):
    import datetime
    import sys
    sys.path[:0] = [ROOT, HERE, os.path.join(HERE, 'golden')]
    import torch
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    P1, P2 = dims
    dist.init_process_group('gloo', rank=rank, world_size=P1 * P2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from bolt_b200.distributed import exchange_q1_halos, exchange_q2_halos, slab_of
        import cases as C
        from oracle.bolt_oracle import Oracle
        spec = _spec()
        Ng = spec['N_ghost']
        r1, r2 = rank % P1, rank // P1
        at = lambda a, b: (a % P1) + P1 * (b % P2)
        n1, lo1, hi1 = slab_of(spec['N_q1'], spec['q1_start'], spec['q1_end'], r1, P1)
        n2, lo2, hi2 = slab_of(spec['N_q2'], spec['q2_start'], spec['q2_end'], r2, P2)
        local = dict(spec, N_q1=n1, q1_start=lo1, q1_end=hi1, N_q2=n2, q2_start=lo2,
                     q2_end=hi2)
        if P1 > 1:
            local['bc_q1'] = 'external'
        if P2 > 1:
            local['bc_q2'] = 'external'
        fg = C.initial_f(spec)
        f0 = fg[r2 * n2:r2 * n2 + n2 + 2 * Ng, r1 * n1:r1 * n1 + n1 + 2 * Ng].copy()
        o = Oracle(local, f0)

        def exchange(x):
            x = np.ascontiguousarray(x)
            t = torch.from_numpy(x)
            if P2 > 1:
                exchange_q2_halos(t, Ng, None, (at(r1, r2 - 1), at(r1, r2 + 1)))
            if P1 > 1:
                exchange_q1_halos(t, Ng, None, (at(r1 - 1, r2), at(r1 + 1, r2)))
            return x
        o.exchange = exchange
        for _ in range(spec['steps']):
            o.step(spec['dt'])
        out.put((rank, o.f[Ng:Ng + n2, Ng:Ng + n1].copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('dims', [(2, 2), (2, 1)])
def test_blocks_over_gloo_ranks_equal_the_whole_domain(dims):
    """A P1 x P2 grid of q-blocks (q1 columns exchanged packed, q2 rows in
    place), the oracle advanced block by block equals the whole domain."""
    import sys
    sys.path[:0] = [ROOT, HERE, os.path.join(HERE, 'golden')]
    import cases as C
    from oracle.bolt_oracle import Oracle
    P1, P2 = dims
    world = P1 * P2
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_block_rank_main, args=(r, dims, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    spec = _spec()
    o = Oracle(spec, C.initial_f(spec))
    for _ in range(spec['steps']):
        o.step(spec['dt'])
    Ng = spec['N_ghost']
    whole = o.f[Ng:Ng + spec['N_q2'], Ng:Ng + spec['N_q1']]
    rows = [np.concatenate([res[r1 + P1 * r2] for r1 in range(P1)], axis=1) for r2 in range(P2)]
    blocks = np.concatenate(rows, axis=0)
    assert np.max(np.abs(blocks - whole)) <= 1e-15 * np.max(np.abs(whole))


def _field_spec(integrator):
    """User-defined E and B (the only initial fields a run cut into blocks can
    have: the reference's FFT solve is serial), FDTD-coupled 2D2V with BGK."""
    import cases as C
    return C.make(N_q1=8, N_q2=8, N_p1=8, N_p2=6, N_p3=1,
                  p1_start=[-5.0], p1_end=[5.0], p2_start=[-5.0], p2_end=[5.0],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
                  fields_enabled=True, fields_initialize='user-defined', field_init='E_B',
                  tau=0.1, dt=1e-3, steps=3, integrator=integrator,
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.05, k1=1, k2=1, T=[1.0, 1.2, 1.0]))


def _field_block_rank_main(rank, dims, integrator, port, out):
    import datetime
    import sys
    sys.path[:0] = [ROOT, HERE, os.path.join(HERE, 'golden')]
    import torch
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    P1, P2 = dims
    dist.init_process_group('gloo', rank=rank, world_size=P1 * P2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from bolt_b200.distributed import (exchange_q1_halos, exchange_q2_halos,
                                           exchange_field_halos, slab_of)
        import cases as C
        from oracle.bolt_oracle import Oracle
        spec = _field_spec(integrator)
        Ng = spec['N_ghost']
        r1, r2 = rank % P1, rank // P1
        at = lambda a, b: (a % P1) + P1 * (b % P2)
        q1_nb, q2_nb = (at(r1 - 1, r2), at(r1 + 1, r2)), (at(r1, r2 - 1), at(r1, r2 + 1))
        n1, lo1, hi1 = slab_of(spec['N_q1'], spec['q1_start'], spec['q1_end'], r1, P1)
        n2, lo2, hi2 = slab_of(spec['N_q2'], spec['q2_start'], spec['q2_end'], r2, P2)
        local = dict(spec, N_q1=n1, q1_start=lo1, q1_end=hi1, N_q2=n2, q2_start=lo2,
                     q2_end=hi2)
        if P1 > 1:
            local['bc_q1'] = 'external'
        if P2 > 1:
            local['bc_q2'] = 'external'
        fg = C.initial_f(spec)
        f0 = fg[r2 * n2:r2 * n2 + n2 + 2 * Ng, r1 * n1:r1 * n1 + n1 + 2 * Ng].copy()
        o = Oracle(local, f0, field_functions=C.field_functions('E_B', np.sin, np.cos))

        def exchange(x):
            x = np.ascontiguousarray(x)
            t = torch.from_numpy(x)
            if P2 > 1:
                exchange_q2_halos(t, Ng, None, q2_nb)
            if P1 > 1:
                exchange_q1_halos(t, Ng, None, q1_nb)
            return x

        def exchange_fields(y):
            y = np.ascontiguousarray(y)
            exchange_field_halos(torch.from_numpy(y), Ng, (P1 > 1, P2 > 1), None, q1_nb, q2_nb)
            return y
        o.exchange = exchange
        o.fields.exchange = exchange_fields
        for _ in range(spec['steps']):
            o.step(spec['dt'])
        sl = (slice(Ng, Ng + n2), slice(Ng, Ng + n1))
        out.put((rank, o.f[sl].copy(), o.fields.yee[(slice(None),) + sl].copy(),
                 o.fields.cell[(slice(None),) + sl].copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('dims,integrator', [((2, 2), 'RK4'), ((2, 1), 'RK2'), ((1, 2), 'RK4')])
def test_field_blocks_over_gloo_ranks_equal_the_whole_domain(dims, integrator):
    """FDTD-coupled blocks: f exchanged before every stage, the Yee ghosts
    between the parts of the field update (q1 columns, then q2 rows), the
    oracle advanced block by block equals the whole domain in f, the Yee-grid
    and the cell-centred fields (1e-13: the blocks evaluate the initial field
    functions at their own coordinates, which differ from the whole grid's in
    the last bits)."""
    import sys
    sys.path[:0] = [ROOT, HERE, os.path.join(HERE, 'golden')]
    import cases as C
    from oracle.bolt_oracle import Oracle
    P1, P2 = dims
    world = P1 * P2
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_field_block_rank_main, args=(r, dims, integrator, port, out))
             for r in range(world)]
    for p in procs:
        p.start()
    res = {r[0]: r[1:] for r in (out.get(timeout=300) for _ in range(world))}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    spec = _field_spec(integrator)
    o = Oracle(spec, C.initial_f(spec), field_functions=C.field_functions('E_B', np.sin, np.cos))
    for _ in range(spec['steps']):
        o.step(spec['dt'])
    Ng = spec['N_ghost']
    sl = (slice(Ng, Ng + spec['N_q2']), slice(Ng, Ng + spec['N_q1']))

    def joined(i, lead):
        rows = [np.concatenate([res[r1 + P1 * r2][i] for r1 in range(P1)], axis=lead + 1)
                for r2 in range(P2)]
        return np.concatenate(rows, axis=lead)
    for i, whole, lead in ((0, o.f[sl], 0), (1, o.fields.yee[(slice(None),) + sl], 1),
                           (2, o.fields.cell[(slice(None),) + sl], 1)):
        got = joined(i, lead)
        assert np.max(np.abs(got - whole)) <= 1e-13 * np.max(np.abs(whole)), i
