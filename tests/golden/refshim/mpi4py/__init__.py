"""Single-rank stand-in for the mpi4py subset used by Bolt (test infrastructure)."""
