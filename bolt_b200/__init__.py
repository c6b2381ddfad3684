"""bolt_b200 - Bolt's nonlinear finite-volume kinetic update on NVIDIA B200.

Drop-in for the FVM path of QuazarTech/Bolt:

    from bolt_b200.physical_system import physical_system
    from bolt_b200.nonlinear_solver import nonlinear_solver
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as advection_terms
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as collision_operator
    import bolt_b200.src.nonrelativistic_boltzmann.moments as moments

The compute path is the CUDA library bolt_b200/_native/libbolt_b200.so
(C ABI: include/bolt_b200.h); build it with ``python -m bolt_b200.build_native``.
"""

__version__ = '0.1.0'
