"""Single-rank numpy stand-in for petsc4py.PETSc (see package docstring)."""

import numpy as np

DECIDE = -1


class _Comm(object):
    rank = 0
    size = 1

    def tompi4py(self):
        import mpi4py.MPI as MPI
        return MPI.COMM_WORLD

    def getRank(self):
        return 0

    def getSize(self):
        return 1


COMM_WORLD = _Comm()


class Sys(object):
    @staticmethod
    def Print(*args, **kw):
        pass

    @staticmethod
    def syncPrint(*args, **kw):
        pass

    @staticmethod
    def syncFlush(*args, **kw):
        pass


class Object(object):
    @staticmethod
    def setName(obj, name):
        obj._name = name


class Vec(object):
    def __init__(self, n, da=None, local=False):
        self._arr = np.zeros(n, dtype=np.float64)
        self._da = da
        self._local = local
        self._name = ''

    def getArray(self):
        return self._arr

    def getSize(self):
        return self._arr.size

    def setRandom(self, rand=None):
        self._arr[:] = np.random.default_rng(0).random(self._arr.size)

    def max(self):
        i = int(np.argmax(self._arr))
        return (i, float(self._arr[i]))

    def set(self, v):
        self._arr[:] = v

    def load(self, viewer):
        data = viewer._read()
        self._arr[:] = data

    def setName(self, name):
        self._name = name


class DMDA(object):
    def create(self, sizes, dof=1, stencil_width=1, boundary_type=None,
               proc_sizes=None, stencil_type=None, comm=None):
        self.N1, self.N2 = sizes
        self.dof = dof
        self.sw = stencil_width
        bt = boundary_type or ('ghosted', 'ghosted')
        self.bt = tuple(bt)
        self.g1 = 0 if self.bt[0] == 'none' else stencil_width
        self.g2 = 0 if self.bt[1] == 'none' else stencil_width
        return self

    def getCorners(self):
        return ((0, 0), (self.N1, self.N2))

    def getGhostCorners(self):
        return ((-self.g1, -self.g2), (self.N1 + 2 * self.g1, self.N2 + 2 * self.g2))

    def createGlobalVec(self):
        return Vec(self.N1 * self.N2 * self.dof, self)

    def createLocalVec(self):
        return Vec((self.N1 + 2 * self.g1) * (self.N2 + 2 * self.g2) * self.dof, self, True)

    def globalToLocal(self, gvec, lvec, addv=None):
        g = gvec._arr.reshape(self.N2, self.N1, self.dof)
        n1g, n2g = self.N1 + 2 * self.g1, self.N2 + 2 * self.g2
        loc = lvec._arr.reshape(n2g, n1g, self.dof)
        per1 = self.bt[0] == 'periodic'
        per2 = self.bt[1] == 'periodic'
        for jj in range(n2g):
            j = jj - self.g2
            if j < 0 or j >= self.N2:
                if not per2:
                    continue
                j %= self.N2
            for ii in range(n1g):
                i = ii - self.g1
                if i < 0 or i >= self.N1:
                    if not per1:
                        continue
                    i %= self.N1
                loc[jj, ii, :] = g[j, i, :]


class _Mode(object):
    READ = 'r'
    WRITE = 'w'


class Viewer(object):
    Mode = _Mode

    def createBinary(self, name, mode='w', comm=None):
        self._name = name
        self._mode = mode
        return self

    def __call__(self, vec):
        # PETSc binary Vec: big-endian int32 class id 1211214, int32 length,
        # then big-endian float64 values.
        with open(self._name, 'wb') as fh:
            np.array([1211214, vec._arr.size], dtype='>i4').tofile(fh)
            vec._arr.astype('>f8').tofile(fh)

    def _read(self):
        with open(self._name, 'rb') as fh:
            hdr = np.fromfile(fh, dtype='>i4', count=2)
            return np.fromfile(fh, dtype='>f8', count=int(hdr[1])).astype(np.float64)
