"""Single-process numpy stand-in for the subset of ArrayFire's Python API that
Bolt's nonlinear FVM path calls.  It exists only so that the unmodified Bolt
sources can be imported and executed on the CPU to generate golden fixtures
(tests/golden/make_golden.py); nothing in the product imports it.

Semantics emulated (ArrayFire 3.x, arrayfire-python):
  * arrays are 4-D, column-major; ``.shape`` trims trailing unit dims;
  * integer indices keep their dimension (``a[0]`` of (6,1,N,M) is (1,1,N,M));
  * ``a[...] = b`` modifies the Python object in place, so aliases see it;
  * ``shift(a, x, y, z, w)``: out[i] = a[(i - x) mod n] per axis (circular);
  * ``sign(x)`` is 1 where x < 0 and 0 elsewhere;
  * ``moddims``/``flat`` reinterpret in column-major order;
  * ``sum(a, d)`` keeps the reduced dim; ``sum(a)``/``mean(a)`` give scalars;
  * ``ifft2(a, scale=1)`` is the unnormalised inverse transform;
  * ``broadcast`` is the identity decorator (numpy broadcasts natively).
"""

import time as _time
import numpy as np


class Dtype(object):
    f32 = np.float32
    f64 = np.float64
    c32 = np.complex64
    c64 = np.complex128
    b8 = np.bool_
    s32 = np.int32
    s64 = np.int64


class INTERP(object):
    NEAREST = 0
    LINEAR = 1
    BILINEAR = 2
    CUBIC = 3
    LOWER = 4
    LINEAR_COSINE = 5
    BILINEAR_COSINE = 6
    BICUBIC = 7
    CUBIC_SPLINE = 8
    BICUBIC_SPLINE = 9


def _as4(a):
    a = np.asarray(a)
    if a.ndim > 4:
        raise ValueError('more than 4 dims')
    return a.reshape(a.shape + (1,) * (4 - a.ndim))


def _unwrap(x):
    return x._a if isinstance(x, Array) else x


def _numdims(shape4):
    nd = 4
    while nd > 1 and shape4[nd - 1] == 1:
        nd -= 1
    return nd


def _seq_bound(b):
    """A slice bound as ArrayFire's af_seq takes it: integral floats index
    like ints; fractional bounds are refused."""
    if b is None or isinstance(b, (int, np.integer)):
        return b
    if float(b) != int(b):
        raise NotImplementedError('fractional slice bound %r' % (b,))
    return int(b)


class Array(object):
    __array_priority__ = 1000

    def __init__(self, src=None, dims=None, dtype=None):
        if src is None:
            self._a = np.zeros((0, 1, 1, 1))
        elif isinstance(src, Array):
            self._a = src._a.copy()
        else:
            a = np.array(src, dtype=dtype)
            if a.ndim == 0:
                a = a.reshape(1)
            if dims is not None:
                a = a.reshape(tuple(dims), order='F')
            self._a = _as4(a)

    @staticmethod
    def _wrap(a):
        out = Array.__new__(Array)
        out._a = _as4(a)
        return out

    # -- metadata -------------------------------------------------------
    @property
    def shape(self):
        nd = _numdims(self._a.shape)
        return tuple(self._a.shape[:nd])

    def dims(self):
        return self.shape

    def numdims(self):
        return _numdims(self._a.shape)

    def elements(self):
        return int(self._a.size)

    def type(self):
        return self._a.dtype

    def dtype(self):
        return self._a.dtype

    def copy(self):
        return Array._wrap(self._a.copy())

    def __array__(self, dtype=None, copy=None):
        out = self._a.reshape(self.shape)
        return out.astype(dtype) if dtype is not None else out.copy()

    def to_ndarray(self, output=None):
        flat = self._a.reshape(-1, order='F')
        if output is None:
            return self._a.reshape(self.shape).copy()
        output.reshape(-1)[:] = flat.astype(output.dtype)
        return output

    def __len__(self):
        return self._a.shape[0]

    def __float__(self):
        return float(self._a.reshape(-1)[0])

    def __repr__(self):
        return 'af.Array(shape=%s)' % (self.shape,)

    # -- indexing (ArrayFire keeps indexed dims) --------------------------
    # ArrayFire's Python indexing turns a slice into an af_seq, whose bounds
    # are doubles, so a float bound such as N_theta/2 (boundaries.py:345)
    # indexes like the integer of the same value; _seq_bound accepts those
    # and refuses fractional ones, whose af_seq meaning is not restated here
    def _key(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        out = []
        for k in key:
            if isinstance(k, (int, np.integer)):
                out.append(slice(int(k), int(k) + 1 if int(k) != -1 else None))
            elif isinstance(k, Array):
                out.append(np.asarray(k._a).reshape(-1))
            elif isinstance(k, slice):
                out.append(slice(_seq_bound(k.start), _seq_bound(k.stop), _seq_bound(k.step)))
            else:
                out.append(k)
        while len(out) < 4:
            out.append(slice(None))
        return tuple(out)

    def __getitem__(self, key):
        return Array._wrap(self._a[self._key(key)].copy())

    def __setitem__(self, key, val):
        k = self._key(key)
        v = _unwrap(val)
        tgt = self._a[k]
        v = np.asarray(v)
        if v.size == tgt.size and v.shape != tgt.shape:
            v = v.reshape(tgt.shape, order='F') if v.ndim == 1 else _as4(v).reshape(tgt.shape)
        if not np.can_cast(v.dtype, self._a.dtype, casting='same_kind') and \
           self._a.dtype != np.bool_:
            self._a = self._a.astype(np.result_type(self._a.dtype, v.dtype))
        new = self._a.copy()
        new[k] = v
        self._a = new

    # -- arithmetic --------------------------------------------------------
    def _bin(self, other, op):
        return Array._wrap(op(self._a, _unwrap(other)))

    def _rbin(self, other, op):
        return Array._wrap(op(_unwrap(other), self._a))

    def __add__(self, o): return self._bin(o, np.add)
    def __radd__(self, o): return self._rbin(o, np.add)
    def __sub__(self, o): return self._bin(o, np.subtract)
    def __rsub__(self, o): return self._rbin(o, np.subtract)
    def __mul__(self, o): return self._bin(o, np.multiply)
    def __rmul__(self, o): return self._rbin(o, np.multiply)
    def __truediv__(self, o): return self._bin(o, np.true_divide)
    def __rtruediv__(self, o): return self._rbin(o, np.true_divide)
    def __pow__(self, o): return self._bin(o, np.power)
    def __rpow__(self, o): return self._rbin(o, np.power)
    def __neg__(self): return Array._wrap(-self._a)
    def __pos__(self): return self
    def __lt__(self, o): return self._bin(o, np.less)
    def __le__(self, o): return self._bin(o, np.less_equal)
    def __gt__(self, o): return self._bin(o, np.greater)
    def __ge__(self, o): return self._bin(o, np.greater_equal)
    def __eq__(self, o): return self._bin(o, np.equal)
    def __ne__(self, o): return self._bin(o, np.not_equal)
    def __and__(self, o): return self._bin(o, np.logical_and)
    def __or__(self, o): return self._bin(o, np.logical_or)

    def __iadd__(self, o):
        self._a = self._a + _unwrap(o)
        return self

    def __isub__(self, o):
        self._a = self._a - _unwrap(o)
        return self

    def __imul__(self, o):
        self._a = self._a * _unwrap(o)
        return self

    def __itruediv__(self, o):
        self._a = self._a / _unwrap(o)
        return self

    __hash__ = object.__hash__


# -- construction ------------------------------------------------------------
def to_array(x):
    if isinstance(x, Array):
        return x.copy()
    return Array._wrap(np.array(x, dtype=np.result_type(np.asarray(x).dtype, np.float64)
                                if np.asarray(x).dtype.kind in 'iub' else None))


def constant(val, d0, d1=1, d2=1, d3=1, dtype=Dtype.f32):
    return Array._wrap(np.full((d0, d1, d2, d3), val, dtype=dtype))


def randu(d0, d1=1, d2=1, d3=1, dtype=Dtype.f32):
    return Array._wrap(np.random.default_rng(0).random((d0, d1, d2, d3)).astype(dtype))


# -- elementwise -------------------------------------------------------------
def _un(f):
    def g(a):
        return Array._wrap(f(_unwrap(a))) if isinstance(a, Array) else f(a)
    return g


abs = _un(np.abs)
exp = _un(np.exp)
sqrt = _un(np.sqrt)
sin = _un(np.sin)
cos = _un(np.cos)
log = _un(np.log)
real = _un(np.real)
imag = _un(np.imag)
isinf = _un(np.isinf)
isnan = _un(np.isnan)


def sign(a):
    return Array._wrap((_unwrap(a) < 0).astype(np.float64))


def minof(a, b):
    return Array._wrap(np.minimum(_unwrap(a), _unwrap(b)))


def maxof(a, b):
    return Array._wrap(np.maximum(_unwrap(a), _unwrap(b)))


def select(cond, a, b):
    return Array._wrap(np.where(_unwrap(cond), _unwrap(a), _unwrap(b)))


# -- data movement -------------------------------------------------------------
def shift(a, x, y=0, z=0, w=0):
    arr = _unwrap(a)
    for ax, s in enumerate((x, y, z, w)):
        if s:
            arr = np.roll(arr, s, axis=ax)
    return Array._wrap(arr.copy())


def moddims(a, d0, d1=1, d2=1, d3=1):
    return Array._wrap(_unwrap(a).reshape((d0, d1, d2, d3), order='F'))


def flat(a):
    return Array._wrap(_unwrap(a).reshape(-1, order='F'))


def tile(a, d0, d1=1, d2=1, d3=1):
    return Array._wrap(np.tile(_unwrap(a), (d0, d1, d2, d3)))


def reorder(a, d0=1, d1=0, d2=2, d3=3):
    return Array._wrap(np.transpose(_unwrap(a), (d0, d1, d2, d3)).copy())


def join(dim, a, b, c=None, d=None):
    arrs = [_unwrap(x) for x in (a, b, c, d) if x is not None]
    return Array._wrap(np.concatenate(arrs, axis=dim))


def flip(a, dim=0):
    return Array._wrap(np.flip(_unwrap(a), axis=dim).copy())


# -- reductions ------------------------------------------------------------------
def sum(a, dim=None):
    arr = _unwrap(a)
    if dim is None:
        return arr.sum().item()
    return Array._wrap(arr.sum(axis=dim, keepdims=True))


def mean(a, dim=None):
    arr = _unwrap(a)
    if dim is None:
        return arr.mean().item()
    return Array._wrap(arr.mean(axis=dim, keepdims=True))


def max(a, dim=None):
    arr = _unwrap(a)
    if dim is None:
        return arr.max().item()
    return Array._wrap(arr.max(axis=dim, keepdims=True))


def min(a, dim=None):
    arr = _unwrap(a)
    if dim is None:
        return arr.min().item()
    return Array._wrap(arr.min(axis=dim, keepdims=True))


def any_true(a, dim=None):
    return bool(np.any(_unwrap(a)))


def all_true(a, dim=None):
    return bool(np.all(_unwrap(a)))


# -- FFT (over the first two dims) ----------------------------------------------------
def fft2(a, dim0=None, dim1=None, scale=None):
    return Array._wrap(np.fft.fft2(_unwrap(a), axes=(0, 1)))


def ifft2(a, dim0=None, dim1=None, scale=None):
    arr = _unwrap(a)
    out = np.fft.ifft2(arr, axes=(0, 1))
    if scale is not None:
        out = out * (arr.shape[0] * arr.shape[1]) * scale
    return Array._wrap(out)


# -- runtime ---------------------------------------------------------------------
def broadcast(func, *args):
    if args:
        return func(*args)
    return func


def eval(*args):
    return None


def sync(device=None):
    return None


def time():
    return _time.time()


def info_str(verbose=False):
    return 'numpy stand-in (CPU)'


def info():
    return None


def set_device(n):
    return None


def get_device():
    return 0


def set_backend(name):
    return None


class _ArrayModule(object):
    Array = Array


array = _ArrayModule()


# -- interpolation ---------------------------------------------------------------
def _catmull_rom(t):
    """Weights of the Catmull-Rom cubic through samples at -1, 0, 1, 2 for a
    point at t in [0, 1) past sample 0 (Catmull and Rom 1974)."""
    t2, t3 = t * t, t * t * t
    return (0.5 * (-t + 2 * t2 - t3), 0.5 * (2 - 5 * t2 + 3 * t3),
            0.5 * (t + 4 * t2 - 3 * t3), 0.5 * (t3 - t2))


def approx2(signal, pos0, pos1, method=INTERP.LINEAR, off_grid=0.0, xp=None, yp=None):
    """Interpolation of dims 0 and 1 of ``signal`` at (pos0, pos1), batched over
    dims 2 and 3 (ArrayFire's approx2).  Positions are sample indices; with xp
    (yp) the positions are coordinates on the uniform grid xp[:, 0, 0, 0]
    (yp[0, :, 0, 0]) and are first mapped to indices, (x - xp0) / dxp.  Only
    BICUBIC_SPLINE is restated: ArrayFire documents it as bicubic
    interpolation with Catmull-Rom splines, here the tensor product of the 1-D
    Catmull-Rom cubic; the neighbouring samples are clamped to the signal and a
    position outside [0, n - 1] on either dim takes ``off_grid``.  (ArrayFire
    itself is not available here: this stands in for its kernel.)"""
    if method != INTERP.BICUBIC_SPLINE:
        raise NotImplementedError('approx2: only BICUBIC_SPLINE is restated')
    f = _unwrap(signal)
    x = np.array(_unwrap(pos0), dtype=np.float64)
    y = np.array(_unwrap(pos1), dtype=np.float64)
    if xp is not None:
        g = _unwrap(xp)
        x = (x - g[0, 0, 0, 0]) / (g[1, 0, 0, 0] - g[0, 0, 0, 0])
    if yp is not None:
        g = _unwrap(yp)
        y = (y - g[0, 0, 0, 0]) / (g[0, 1, 0, 0] - g[0, 0, 0, 0])
    n0, n1 = f.shape[0], f.shape[1]
    x = np.broadcast_to(x, f.shape[:2] + x.shape[2:]) if x.shape[:2] != f.shape[:2] else x
    shape = np.broadcast_shapes(x.shape, y.shape, (1, 1) + f.shape[2:])
    x = np.broadcast_to(x, shape)
    y = np.broadcast_to(y, shape)
    off = (x < 0) | (x > n0 - 1) | (y < 0) | (y > n1 - 1)
    xs = np.clip(x, 0, n0 - 1)
    ys = np.clip(y, 0, n1 - 1)
    i0 = np.floor(xs).astype(np.int64)
    j0 = np.floor(ys).astype(np.int64)
    wx = _catmull_rom(xs - i0)
    wy = _catmull_rom(ys - j0)
    b2 = np.arange(shape[2]).reshape(1, 1, -1, 1)
    b3 = np.arange(shape[3]).reshape(1, 1, 1, -1)
    b2 = np.broadcast_to(b2 if f.shape[2] > 1 else 0 * b2, shape)
    b3 = np.broadcast_to(b3 if f.shape[3] > 1 else 0 * b3, shape)
    out = np.zeros(shape, dtype=np.result_type(f.dtype, np.float64))
    for b in range(4):
        jj = np.clip(j0 - 1 + b, 0, n1 - 1)
        row = np.zeros(shape)
        for a in range(4):
            ii = np.clip(i0 - 1 + a, 0, n0 - 1)
            row = row + wx[a] * f[ii, jj, b2, b3]
        out = out + wy[b] * row
    out[off] = off_grid
    return Array._wrap(out.astype(f.dtype))
