"""ctypes wrapper and build recipe of oracle/bolt_oracle_c.c (test/bench
infrastructure).  Built with gcc -O3 -fopenmp -ffp-contract=off into
oracle/_build/liboracle.so."""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'bolt_oracle_c.c')
LIB = os.path.join(HERE, '_build', 'liboracle.so')

_D8 = ctypes.c_double * 8


class OracleGrid(ctypes.Structure):
    _fields_ = [('Nq1', ctypes.c_int), ('Nq2', ctypes.c_int), ('Ng', ctypes.c_int),
                ('Np1', ctypes.c_int), ('Np2', ctypes.c_int), ('Np3', ctypes.c_int),
                ('Ns', ctypes.c_int), ('p_dim', ctypes.c_int),
                ('dq1', ctypes.c_double), ('dq2', ctypes.c_double),
                ('p1_start', _D8), ('p2_start', _D8), ('p3_start', _D8),
                ('dp1', _D8), ('dp2', _D8), ('dp3', _D8), ('mass', _D8),
                ('kB', ctypes.c_double), ('tau', ctypes.c_double),
                ('recon', ctypes.c_int), ('bgk', ctypes.c_int)]


RECON = {'piecewise-constant': 0, 'minmod': 1, 'ppm': 2, 'weno5': 3}


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.run(['gcc', '-O3', '-march=x86-64-v2', '-fopenmp', '-ffp-contract=off', '-fPIC',
                    '-shared', SRC, '-o', LIB, '-lm'], check=True)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.oracle_rk_step.restype = ctypes.c_int
        _lib.oracle_rk_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(OracleGrid),
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int]
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def make_grid(spec):
    g = OracleGrid()
    g.Nq1, g.Nq2, g.Ng = spec['N_q1'], spec['N_q2'], spec['N_ghost']
    g.Np1, g.Np2, g.Np3 = spec['N_p1'], spec['N_p2'], spec['N_p3']
    g.Ns = len(spec['mass'])
    g.p_dim = spec['p_dim']
    g.dq1 = (spec['q1_end'] - spec['q1_start']) / spec['N_q1']
    g.dq2 = (spec['q2_end'] - spec['q2_start']) / spec['N_q2']
    for s in range(g.Ns):
        g.p1_start[s], g.p2_start[s], g.p3_start[s] = spec['p1_start'][s], spec['p2_start'][s], spec['p3_start'][s]
        g.dp1[s] = (spec['p1_end'][s] - spec['p1_start'][s]) / spec['N_p1']
        g.dp2[s] = (spec['p2_end'][s] - spec['p2_start'][s]) / spec['N_p2']
        g.dp3[s] = (spec['p3_end'][s] - spec['p3_start'][s]) / spec['N_p3']
        g.mass[s] = spec['mass'][s]
    g.kB = spec['boltzmann_constant']
    g.tau = spec['tau']
    g.recon = RECON[spec['recon_q']]
    g.bgk = 1 if spec['source_enabled'] else 0
    return g


def rk_step(f, spec, dt, integrator=4, threads=0):
    """One RK step of the ghosted f (numpy float64, C-contiguous) in place."""
    assert f.dtype == np.float64 and f.flags['C_CONTIGUOUS']
    lib = load()
    g = make_grid(spec)
    rc = lib.oracle_rk_step(f.ctypes.data, ctypes.byref(g), float(dt), int(integrator), int(threads))
    if rc != 0:
        raise MemoryError('oracle scratch allocation failed')
    return f


def max_threads():
    return load().oracle_max_threads()
