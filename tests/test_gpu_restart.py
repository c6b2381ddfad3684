"""Restart files compatible with Bolt's (file_io/dump.py, load.py): the dumps
written by the unmodified reference for two cases (tests/golden/dumps, made
by make_dump_golden.py) are loaded into the solver and written back
byte-for-byte; the moments dump of the loaded state equals the reference's to
1e-12; the fields dump after the case's steps (run here from the fixture's
initial state) equals the reference's to 1e-9, with identical headers."""

import os

import numpy as np
import pytest
import torch

import cases as C
from _modules import make_solver, to_layout
from _util import interior, load_golden

pytestmark = pytest.mark.gpu

DUMPS = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'dumps')


def _raw(path):
    with open(path, 'rb') as fh:
        return fh.read()


def _vec(path):
    b = _raw(path)
    hdr = np.frombuffer(b[:8], dtype='>i4')
    return hdr, np.frombuffer(b[8:], dtype='>f8')


@pytest.mark.parametrize('name', ['two_species_2d2v_fields', 'c3_2d3v_weno5_rk4_small'])
def test_load_then_dump_reproduces_reference_files(name, tmp_path):
    spec = C.CASES[name]
    nls = make_solver(spec, 'fp64')
    nls.load_distribution_function(os.path.join(DUMPS, name + '_f'))
    state = np.load(os.path.join(DUMPS, name + '_state.npz'))
    g = spec['N_ghost']
    assert np.array_equal(interior(to_layout(nls.f, spec), g), state['f'])
    out = str(tmp_path / 'f')
    nls.dump_distribution_function(out)
    assert _raw(out + '.bin') == _raw(os.path.join(DUMPS, name + '_f.bin'))
    # moments of the loaded state
    nls.dump_moments(str(tmp_path / 'm'))
    h1, v1 = _vec(str(tmp_path / 'm.bin'))
    h0, v0 = _vec(os.path.join(DUMPS, name + '_moments.bin'))
    assert np.array_equal(h1, h0)
    assert np.linalg.norm(v1 - v0) <= 1e-12 * np.linalg.norm(v0)


def test_fields_dump_matches_reference(tmp_path):
    name = 'two_species_2d2v_fields'
    spec = C.CASES[name]
    G = load_golden(name)
    nls = make_solver(spec, 'fp64')
    from test_gpu_parity import af_from_layout, fields_af
    nls.f = af_from_layout(G['f0_refreshed']).to('cuda')
    nls.fields_solver.cell_centered_EM_fields = fields_af(G['fields_cell0'])
    nls.fields_solver.yee_grid_EM_fields = fields_af(G['fields_yee0'])
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    nls.dump_EM_fields(str(tmp_path / 'e'))
    h1, v1 = _vec(str(tmp_path / 'e.bin'))
    h0, v0 = _vec(os.path.join(DUMPS, name + '_fields.bin'))
    assert np.array_equal(h1, h0)
    assert np.linalg.norm(v1 - v0) <= 1e-9 * np.linalg.norm(v0)
    # and the fields file loads back and dumps identically
    nls.load_EM_fields(os.path.join(DUMPS, name + '_fields'))
    nls.dump_EM_fields(str(tmp_path / 'e2'))
    assert _raw(str(tmp_path / 'e2.bin')) == _raw(os.path.join(DUMPS, name + '_fields.bin'))
