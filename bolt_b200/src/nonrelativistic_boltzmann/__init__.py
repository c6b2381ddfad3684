"""Nonrelativistic Boltzmann plug-ins (advection terms, BGK source, moments).

The nonlinear solver recognises these modules by identity and evaluates them
in its CUDA kernels; the Python functions here state the same mathematics on
torch tensors (AF-ordered shapes: p-grids (Np, Ns, 1, 1), q-grids
(1, 1, Nq1g, Nq2g)) for users and for documentation.
"""
