"""Restart files of a run split into q-blocks, on the CPU with gloo ranks
(127.0.0.1): every rank reads its block of a PETSc binary Vec that the
unmodified reference wrote (tests/golden/dumps, made by make_dump_golden.py)
with bolt_b200.distributed.read_block_vec, and the ranks write the blocks
back together with write_block_vec.  The result is the reference's file, byte
for byte, for every block grid: PETSc's DMDA VecView writes the natural
(q2, q1, dof) order whatever the process grid (file_io/dump.py:121-168), and
VecLoad scatters it back (file_io/load.py:10-43)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DUMPS = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'dumps')

# (file, N_q2, N_q1, dof) of the reference-written dumps
FILES = [('c3_2d3v_weno5_rk4_small_f.bin', 8, 8, 512),
         ('c3_2d3v_weno5_rk4_small_moments.bin', 8, 8, 11),
         ('two_species_2d2v_fields_f.bin', 4, 6, 96)]


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _raw(path):
    with open(path, 'rb') as fh:
        return fh.read()


def _rank_main(rank, dims, port, src, shape, out_path, q):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    P1, P2 = dims
    dist.init_process_group('gloo', rank=rank, world_size=P1 * P2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from bolt_b200.distributed import read_block_vec, write_block_vec
        N2, N1, dof = shape
        r1, r2 = rank % P1, rank // P1
        n2, n1 = N2 // P2, N1 // P1
        corner = (r2 * n2, r1 * n1)
        block = read_block_vec(src, corner, (n2, n1), shape)
        write_block_vec(out_path, block, corner, shape)
        q.put((rank, corner, block))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('name,N2,N1,dof,dims', [FILES[0] + ((2, 2),), FILES[0] + ((1, 2),),
                                                  FILES[1] + ((2, 2),), FILES[2] + ((2, 1),)])
def test_block_grid_rewrites_reference_dump(name, N2, N1, dof, dims, tmp_path):
    import sys
    sys.path.insert(0, ROOT)
    from bolt_b200.nonlinear_solver import _read_petsc_vec
    P1, P2 = dims
    src = os.path.join(DUMPS, name)
    out_path = str(tmp_path / 'out.bin')
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main,
                         args=(r, dims, port, src, (N2, N1, dof), out_path, q))
             for r in range(P1 * P2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = _read_petsc_vec(src).reshape(N2, N1, dof)
    for _, (j0, i0), block in res:
        assert np.array_equal(block, whole[j0:j0 + block.shape[0], i0:i0 + block.shape[1]])
    assert _raw(out_path) == _raw(src)
    with open(out_path + '.info') as fh:
        assert fh.read() == '-vecload_block_size %d\n' % dof


def test_blocks_written_in_rank_order_without_a_group(tmp_path):
    """Without a process group the creating block is written first and the
    others fill their rows in."""
    import sys
    sys.path.insert(0, ROOT)
    from bolt_b200.distributed import read_block_vec, write_block_vec
    name, N2, N1, dof = FILES[0]
    src = os.path.join(DUMPS, name)
    out_path = str(tmp_path / 'out.bin')
    for r in range(4):
        corner = ((r // 2) * 4, (r % 2) * 4)
        write_block_vec(out_path, read_block_vec(src, corner, (4, 4), (N2, N1, dof)),
                        corner, (N2, N1, dof), create=r == 0, collective=False)
    assert _raw(out_path) == _raw(src)


def test_blocks_of_one_process_inside_a_process_group(tmp_path):
    """Blocks written one after another by a process that has a process group
    (collective=False): the creating call does not erase the others' rows."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    p = ctx.Process(target=_one_process_blocks, args=(_free_port(), str(tmp_path / 'o.bin'), q))
    p.start()
    ok = q.get(timeout=300)
    p.join(timeout=60)
    assert p.exitcode == 0 and ok


def _one_process_blocks(port, out_path, q):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from bolt_b200.distributed import read_block_vec, write_block_vec
        name, N2, N1, dof = FILES[0]
        src = os.path.join(DUMPS, name)
        for r in range(4):
            corner = ((r // 2) * 4, (r % 2) * 4)
            write_block_vec(out_path, read_block_vec(src, corner, (4, 4), (N2, N1, dof)),
                            corner, (N2, N1, dof), create=r == 0, collective=False)
        q.put(_raw(out_path) == _raw(src))
    finally:
        dist.destroy_process_group()


def test_block_vec_errors(tmp_path):
    import sys
    sys.path.insert(0, ROOT)
    from bolt_b200.distributed import read_block_vec, write_block_vec
    name, N2, N1, dof = FILES[0]
    src = os.path.join(DUMPS, name)
    with pytest.raises(IOError):                      # grid of another size
        read_block_vec(src, (0, 0), (4, 4), (N2, N1, dof + 1))
    bad = tmp_path / 'bad.bin'
    bad.write_bytes(b'\x00' * 16)
    with pytest.raises(IOError):                      # not a Vec
        read_block_vec(str(bad), (0, 0), (1, 1), (1, 1, 1))
    with pytest.raises(ValueError):                   # block past the grid
        write_block_vec(str(tmp_path / 'o.bin'), np.zeros((4, 4, dof)), (6, 0), (N2, N1, dof))
    with pytest.raises(ValueError):                   # wrong dof
        write_block_vec(str(tmp_path / 'o.bin'), np.zeros((4, 4, 3)), (0, 0), (N2, N1, dof))
