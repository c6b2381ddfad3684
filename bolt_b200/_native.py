"""ctypes binding of the C ABI in include/bolt_b200.h.

The shared library is built in-tree (bolt_b200/build_native.py).  There is no
CPU fallback: if the library is missing or no CUDA device is present, creating
a solver raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_native', 'libbolt_b200.so')

MAX_SPECIES = 8

BOLT_OK = 0
BOLT_ERR_ARG = 1
BOLT_ERR_CUDA = 2
BOLT_ERR_NONFINITE = 3
BOLT_ERR_TIMEOUT = 4
BOLT_ERR_UNSUPPORTED = 5
BOLT_ERR_NOMEM = 6

F64, F32, F64_FAST = 0, 1, 2
RECON = {'piecewise-constant': 0, 'minmod': 1, 'ppm': 2, 'weno5': 3}
FLUX = {'upwind-flux': 0, 'upwind': 0, 'lax-friedrichs': 1, 'llf': 1,
        'local-lax-friedrichs': 1}
BC = {'periodic': 0, 'dirichlet': 1, 'external': 2, 'mirror': 3, 'mirror+dirichlet': 4,
      'shearing-box': 5}
RK = {'RK2': 2, 'RK4': 4}
PGRID = {'cartesian': 0, 'polar2D': 1}
FIELDS = {'electrodynamic': 0, 'electrostatic': 1}
MOMENT_IDS = {'density': 0, 'mom_v1_bulk': 1, 'mom_v2_bulk': 2, 'mom_v3_bulk': 3,
              'energy': 4, 'energy_q1': 5, 'energy_q2': 6, 'energy_q3': 7,
              'q_q1': 8, 'q_q2': 9, 'q_q3': 10}

_D8 = ctypes.c_double * MAX_SPECIES


class BoltGrid(ctypes.Structure):
    _fields_ = [('N_q1', ctypes.c_int), ('N_q2', ctypes.c_int), ('N_ghost', ctypes.c_int),
                ('N_p1', ctypes.c_int), ('N_p2', ctypes.c_int), ('N_p3', ctypes.c_int),
                ('N_s', ctypes.c_int),
                ('q1_start', ctypes.c_double), ('q2_start', ctypes.c_double),
                ('dq1', ctypes.c_double), ('dq2', ctypes.c_double),
                ('p1_start', _D8), ('p2_start', _D8), ('p3_start', _D8),
                ('dp1', _D8), ('dp2', _D8), ('dp3', _D8)]


class BoltParams(ctypes.Structure):
    _fields_ = [('dtype', ctypes.c_int), ('recon_q', ctypes.c_int), ('recon_p', ctypes.c_int),
                ('flux_q', ctypes.c_int), ('flux_p', ctypes.c_int),
                ('bc_q1', ctypes.c_int), ('bc_q2', ctypes.c_int),
                ('integrator', ctypes.c_int), ('source_enabled', ctypes.c_int),
                ('fields_enabled', ctypes.c_int), ('p_dim', ctypes.c_int),
                ('fields_type', ctypes.c_int),
                ('mass', _D8), ('charge', _D8),
                ('boltzmann_constant', ctypes.c_double), ('tau', ctypes.c_double),
                ('eps', ctypes.c_double), ('mu', ctypes.c_double)]


class BoltBatchRun(ctypes.Structure):
    _fields_ = [('N_q1', ctypes.c_int), ('N_p1', ctypes.c_int),
                ('q1_start', ctypes.c_double), ('q1_end', ctypes.c_double),
                ('p1_start', ctypes.c_double), ('p1_end', ctypes.c_double),
                ('p2_center', ctypes.c_double), ('p3_center', ctypes.c_double),
                ('dp2', ctypes.c_double), ('dp3', ctypes.c_double),
                ('mass', ctypes.c_double), ('boltzmann_constant', ctypes.c_double),
                ('tau', ctypes.c_double), ('dt', ctypes.c_double)]


class BoltAdj1DSpec(ctypes.Structure):
    _fields_ = [('N_q1', ctypes.c_int), ('N_p1', ctypes.c_int),
                ('q1_start', ctypes.c_double), ('q1_end', ctypes.c_double),
                ('p1_start', ctypes.c_double), ('p1_end', ctypes.c_double),
                ('dp2', ctypes.c_double), ('dp3', ctypes.c_double),
                ('mass', ctypes.c_double), ('boltzmann_constant', ctypes.c_double),
                ('tau', ctypes.c_double), ('dt', ctypes.c_double), ('recon', ctypes.c_int)]


# exported symbol -> (restype, argtypes); every function of include/bolt_b200.h
_VP = ctypes.c_void_p
SIGNATURES = {
    'bolt_ctx_create': (ctypes.c_int, [ctypes.POINTER(BoltGrid), ctypes.POINTER(BoltParams),
                                       ctypes.POINTER(_VP)]),
    'bolt_ctx_destroy': (None, [_VP]),
    'bolt_set_tau_array': (ctypes.c_int, [_VP, _VP]),
    'bolt_set_dirichlet': (ctypes.c_int, [_VP, ctypes.c_int, _VP]),
    'bolt_fill_ghosts': (ctypes.c_int, [_VP, _VP, _VP]),
    'bolt_set_shear': (ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_double]),
    'bolt_set_p_space_grid': (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_double]),
    'bolt_set_time': (ctypes.c_int, [_VP, ctypes.c_double]),
    'bolt_invalidate': (ctypes.c_int, [_VP]),
    'bolt_dfdt': (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, ctypes.c_double, _VP]),
    'bolt_dfdt_term': (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, _VP]),
    'bolt_step': (ctypes.c_int, [_VP, _VP, ctypes.c_double, _VP]),
    'bolt_run': (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int, _VP]),
    'bolt_stage_count': (ctypes.c_int, [_VP]),
    'bolt_stage_input': (_VP, [_VP, _VP, ctypes.c_int]),
    'bolt_stage': (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int, _VP]),
    'bolt_stage_parts': (ctypes.c_int, [_VP, ctypes.c_int]),
    'bolt_stage_part': (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int, ctypes.c_int, _VP]),
    'bolt_stage_region': (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         _VP]),
    'bolt_asl_advect_q': (ctypes.c_int, [_VP, _VP, ctypes.c_double, _VP]),
    'bolt_asl_source': (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int, _VP]),
    'bolt_fvm_p_step': (ctypes.c_int, [_VP, _VP, ctypes.c_double, _VP]),
    'bolt_asl_advect_q_to': (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_double, _VP]),
    'bolt_asl_source_to': (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_double, ctypes.c_int,
                                          _VP]),
    'bolt_work_buffer': (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    'bolt_fields_yee': (_VP, [_VP]),
    'bolt_set_peer_halos': (ctypes.c_int, [_VP, ctypes.POINTER(_VP), ctypes.POINTER(_VP)]),
    'bolt_set_peer_halos_q1': (ctypes.c_int, [_VP, ctypes.POINTER(_VP), ctypes.POINTER(_VP)]),
    'bolt_fields_evolve': (ctypes.c_int, [_VP, _VP, ctypes.c_double, _VP]),
    'bolt_stage_buffer': (_VP, [_VP, ctypes.c_int]),
    'bolt_ipc_get': (ctypes.c_int, [_VP, ctypes.c_char_p]),
    'bolt_ipc_open': (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
    'bolt_ipc_close': (ctypes.c_int, [_VP]),
    'bolt_moments': (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP]),
    'bolt_fields_set': (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    'bolt_fields_get': (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    'bolt_get_at_n': (ctypes.c_int, [_VP]),
    'bolt_set_at_n': (ctypes.c_int, [_VP, ctypes.c_int]),
    'bolt_divergence_flag': (ctypes.c_int, [_VP]),
    'bolt_clear_divergence_flag': (ctypes.c_int, [_VP]),
    'bolt_status_sync': (ctypes.c_int, [_VP, _VP]),
    'bolt_error_flag': (ctypes.c_int, [_VP]),
    'bolt_clear_error': (ctypes.c_int, [_VP]),
    'bolt_set_wait_budget': (ctypes.c_int, [_VP, ctypes.c_longlong]),
    'bolt_test_stall_waits': (ctypes.c_int, [_VP, ctypes.c_int]),
    'bolt_set_timing': (ctypes.c_int, [_VP, ctypes.c_int]),
    'bolt_timings': (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_double)]),
    'bolt_strerror': (ctypes.c_char_p, [ctypes.c_int]),
    'bolt_launch_count': (ctypes.c_longlong, [_VP]),
    'bolt_paired_launch_count': (ctypes.c_longlong, [_VP]),
    'bolt_split_info': (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    'bolt_scratch_bytes': (ctypes.c_size_t, [_VP]),
    'bolt_dfdt_noalloc': (ctypes.c_int, [ctypes.POINTER(BoltGrid), ctypes.POINTER(BoltParams),
                                         _VP, _VP, _VP]),
    'bolt_noalloc_status': (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
    'bolt_batch_create': (ctypes.c_int, [ctypes.POINTER(BoltBatchRun), ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(_VP)]),
    'bolt_batch_destroy': (None, [_VP]),
    'bolt_batch_f': (_VP, [_VP]),
    'bolt_batch_f_count': (ctypes.c_longlong, [_VP]),
    'bolt_batch_f_offset': (ctypes.c_longlong, [_VP, ctypes.c_int]),
    'bolt_batch_q_offset': (ctypes.c_int, [_VP, ctypes.c_int]),
    'bolt_batch_q_count': (ctypes.c_int, [_VP]),
    'bolt_batch_prepare': (ctypes.c_int, [_VP, _VP]),
    'bolt_batch_run': (ctypes.c_int, [_VP, ctypes.c_int, _VP]),
    'bolt_batch_moments': (ctypes.c_int, [_VP, _VP, _VP]),
    'bolt_batch_divergence_flag': (ctypes.c_int, [_VP]),
    'bolt_batch_set_schedule': (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    'bolt_batch_get_schedule': (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int)]),
    'bolt_adj1d_create': (ctypes.c_int, [ctypes.POINTER(BoltAdj1DSpec), ctypes.c_int,
                                         ctypes.POINTER(_VP)]),
    'bolt_adj1d_destroy': (None, [_VP]),
    'bolt_adj1d_set_tau': (ctypes.c_int, [_VP, ctypes.c_double]),
    'bolt_adj1d_step': (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    'bolt_adj1d_step_adjoint': (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, _VP, _VP]),
    'bolt_adj1d_objective': (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
}

NOALLOC_MAX_QCELLS = 65536
TIMING_NAMES = ('ghosts', 'moments', 'q-stage', 'p-stage', 'fields')

_lib = None


class DeviceArray(object):
    """A device allocation of the library exposed to torch without a copy
    (torch.as_tensor(DeviceArray(ptr, count, '<f4'), device='cuda'))."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {'shape': (int(count),), 'typestr': typestr,
                                         'data': (int(ptr), False), 'version': 3,
                                         'strides': None}


class BoltError(RuntimeError):
    def __init__(self, code, where=''):
        self.code = code
        msg = strerror(code) if _lib is not None else str(code)
        super().__init__('%s failed: %s (code %d)' % (where, msg, code))


def load():
    """Load (building first if it is missing) the native library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build_native
        build_native.build()
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def strerror(code):
    return load().bolt_strerror(int(code)).decode()


def check(rc, where):
    if rc != BOLT_OK:
        if rc == BOLT_ERR_NONFINITE:
            raise SystemExit('Solver Diverging!')
        raise BoltError(rc, where)
