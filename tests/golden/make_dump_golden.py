"""Generate the restart-file fixtures: run the unmodified Bolt source (over the
numpy stand-ins of tests/golden/refshim, as make_golden.py does) for a case,
advance it by the case's steps and write its dump files with Bolt's own
dump_distribution_function / dump_moments / dump_EM_fields (file_io/dump.py).
The PETSc binary Vec format of those files is the stand-in viewer's: the
big-endian int32 Vec class id 1211214, the int32 length, then big-endian
float64 values.  Test infrastructure, run in the container with the reference:

    python tests/golden/make_dump_golden.py /path/to/reference [case ...]
    (or the reference root in $BOLT_REFERENCE_DIR)

writes tests/golden/dumps/<case>_{f,moments,fields}.bin and <case>_state.npz
(the interior f the dumps were made from, in (q2, q1, s, p3, p2, p1) order).
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'refshim'))
sys.path.insert(0, HERE)

import cases as C  # noqa: E402
import make_golden as G  # noqa: E402

CASES = ('two_species_2d2v_fields', 'c3_2d3v_weno5_rk4_small')


def dump_case(name):
    import arrayfire as af
    from bolt.lib.physical_system import physical_system
    from bolt.lib.nonlinear.nonlinear_solver import nonlinear_solver
    import bolt.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt.src.nonrelativistic_boltzmann.moments as mom
    import bolt.lib.nonlinear.nonlinear_solver as nsmod
    spec = C.CASES[name]
    G.patch_reference()
    nsmod.bandwidth_test = lambda n_evals: 0.0
    dom, bc, params, initialize = G.build_modules(spec, af)
    system = physical_system(dom, bc, params, initialize, adv, col.BGK, mom)
    nls = nonlinear_solver(system)
    for _ in range(spec['steps']):
        nls.strang_timestep(spec['dt'])
    out = os.path.join(HERE, 'dumps')
    os.makedirs(out, exist_ok=True)
    base = os.path.join(out, name)
    nls.dump_distribution_function(base + '_f')
    nls.dump_moments(base + '_moments')
    if spec['fields_enabled']:
        nls.dump_EM_fields(base + '_fields')
    np.savez_compressed(base + '_state.npz',
                        f=G.interior(G.af_to_layout(nls.f, spec), spec),
                        time_elapsed=np.array(nls.time_elapsed))
    print('wrote', base)


def main(argv):
    ref, names = G.reference_dir(argv)
    sys.path.insert(1, ref)
    for name in names or CASES:
        dump_case(name)


if __name__ == '__main__':
    main(sys.argv[1:])
