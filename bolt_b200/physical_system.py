"""physical_system: the description of a kinetic problem (drop-in for
bolt/lib/physical_system.py:8-283).

Same constructor arguments, the same validation and the same derived
quantities (dq1, dq2, per-species dp1/dp2/dp3 lists, N_species) as the
reference.  The MPI communicator of the reference is replaced by the
torch.distributed world (if initialised), since this build runs one process
per GPU.
"""

import types


class physical_system(object):

    def __init__(self, domain, boundary_conditions, params, initial_conditions,
                 advection_term, source, moments):
        # type checks (physical_system.py:67-110)
        attributes = [a for a in dir(boundary_conditions) if not a.startswith('__')]
        for name in attributes:
            val = getattr(boundary_conditions, name)
            if not (isinstance(val, (str, float, bool, types.FunctionType, types.ModuleType))):
                raise TypeError('Expected attributes of boundary_conditions '
                                'to be of type string or functions')
        if not isinstance(initial_conditions, types.ModuleType):
            raise TypeError('Expected initial_conditions to be of type function')
        if not isinstance(source, types.FunctionType):
            raise TypeError('Expected source_or_sink to be of type function')
        for name in [a for a in dir(advection_term) if not a.startswith('_')]:
            if not isinstance(getattr(advection_term, name), (types.FunctionType, types.ModuleType)):
                raise TypeError('Expected attributes of advection_term '
                                'to be of type function or module')
        for name in [a for a in dir(moments) if not a.startswith('_')]:
            if not isinstance(getattr(moments, name), (types.FunctionType, types.ModuleType)):
                raise TypeError('Expected attributes of moment_defs '
                                'to be of type function or module')

        # species (physical_system.py:112-144)
        N_species = len(params.charge)
        self.N_species = N_species
        if len(params.mass) != len(params.charge):
            raise Exception('Inconsistenty in number of species. Mismatch between '
                            'the number of species mentioned in charge and mass inputs')
        if getattr(params, 'hybrid_model_enabled', False) and N_species != 1:
            raise Exception('Only ions are to be initialized when using the hybrid model')
        for k in ('p1_start', 'p2_start', 'p3_start', 'p1_end', 'p2_end', 'p3_end'):
            if type(getattr(domain, k)) != list:
                raise Exception('p-domain start and end points need to be specified in a list')
            if len(getattr(domain, k)) != N_species:
                raise Exception('Inconsistency in definition of p-space resolution '
                                'with number of species')

        self.N_q1, self.q1_start, self.q1_end = domain.N_q1, domain.q1_start, domain.q1_end
        self.N_q2, self.q2_start, self.q2_end = domain.N_q2, domain.q2_start, domain.q2_end
        self.N_p1, self.p1_start, self.p1_end = domain.N_p1, domain.p1_start, domain.p1_end
        self.N_p2, self.p2_start, self.p2_end = domain.N_p2, domain.p2_start, domain.p2_end
        self.N_p3, self.p3_start, self.p3_end = domain.N_p3, domain.p3_start, domain.p3_end

        if (self.N_q1 < 0 or self.N_q2 < 0 or self.N_p1 < 0 or self.N_p2 < 0 or
                self.N_p3 < 0 or domain.N_ghost < 0):
            raise Exception('Grid resolution for the phase space cannot be negative')
        if (self.q1_start > self.q1_end or self.q2_start > self.q2_end or
                self.p1_start > self.p1_end or self.p2_start > self.p2_end or
                self.p3_start > self.p3_end):
            raise Exception('Start point cannot be placed after the end point')

        # resolution (physical_system.py:176-187)
        self.dq1 = (self.q1_end - self.q1_start) / self.N_q1
        self.dq2 = (self.q2_end - self.q2_start) / self.N_q2
        self.dp1, self.dp2, self.dp3 = [], [], []
        for i in range(N_species):
            self.dp1.append((self.p1_end[i] - self.p1_start[i]) / self.N_p1)
            self.dp2.append((self.p2_end[i] - self.p2_start[i]) / self.N_p2)
            self.dp3.append((self.p3_end[i] - self.p3_start[i]) / self.N_p3)

        self.N_ghost = domain.N_ghost
        self.boundary_conditions = boundary_conditions
        self.params = params
        self.initial_conditions = initial_conditions
        self.A_q = advection_term.A_q
        self.C_q = advection_term.C_q
        self.A_p = advection_term.A_p
        self.C_p = advection_term.C_p
        self.advection_term = advection_term
        self.source = source
        self.moments = moments
        self.mpi_communicator = _World()

        if params.fields_type == 'electrodynamic':
            if params.fields_solver.upper() != 'FDTD':
                raise Exception("Solver specified isn't an electrodynamic solver")
        if params.fields_type == 'electrostatic':
            if params.fields_solver.upper() not in ('SNES', 'FFT'):
                raise Exception("Solver specified isn't an electrostatic solver")


class _World(object):
    """rank/size of the torch.distributed world (one process per GPU)."""

    @property
    def rank(self):
        try:
            import torch.distributed as dist
            return dist.get_rank() if dist.is_initialized() else 0
        except Exception:
            return 0

    @property
    def size(self):
        try:
            import torch.distributed as dist
            return dist.get_world_size() if dist.is_initialized() else 1
        except Exception:
            return 1
