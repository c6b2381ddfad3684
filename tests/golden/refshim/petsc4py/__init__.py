"""Single-rank stand-in for the petsc4py subset used by Bolt's nonlinear path
(DMDA halo exchange, Vecs, binary viewer, printing).  Test infrastructure for
golden-fixture generation only.

DMDA.globalToLocal: interior copied; ghost cells of a 'periodic' axis are
filled by wrap-around (box stencil, so corners too); ghost cells on a
'ghosted' axis keep the local vector's previous contents (zero after creation),
which is what PETSc does for DM_BOUNDARY_GHOSTED on one rank.
"""


def init(args=None):
    return None
