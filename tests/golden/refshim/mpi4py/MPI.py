"""Single-rank stand-in for mpi4py.MPI (test infrastructure)."""

import numpy as np

SUM = 'sum'
MAX = 'max'
MIN = 'min'


class _Comm(object):
    rank = 0
    size = 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Reduce(self, send, recv, op=SUM, root=0):
        recv[...] = np.asarray(send)

    def Allreduce(self, send, recv, op=SUM):
        recv[...] = np.asarray(send)

    def allreduce(self, x, op=SUM):
        return x

    def Barrier(self):
        pass

    barrier = Barrier


COMM_WORLD = _Comm()
