"""A sequential CPU stand-in for the subset of the ``warp`` module that the
reference package ``xpbd3d`` uses, so that the reference's own kernel and solver
code can be executed in a container that has no ``warp-lang``.

Test infrastructure only: it exists to run the reference (``src/xpbd3d/*.py``)
unmodified and record its outputs as golden fixtures (``make_golden.py``).

Semantics restated here (from Warp's public documentation, not its source):

* ``float`` in a kernel is IEEE fp32; every vec/quat/mat operation rounds to fp32
  after each scalar operation, in the association order written below.
* ``wp.launch(k, dim, inputs, outputs)`` runs thread ids ``0..dim-1`` one after
  another; ``wp.atomic_add`` is then a plain read-modify-write.
* quaternions are ``(x, y, z, w)`` with the Hamilton product; ``quat_inverse`` is
  the conjugate (unit quaternions); ``quat_rotate(q, v) = v(2w²-1) + 2w(u×v) +
  2u(u·v)`` with ``u = (x, y, z)``.
* ``wp.Bvh`` queries return every leaf whose box overlaps the query box, bounds
  inclusive, in ascending leaf order.  ``wp.HashGrid`` queries return every point
  whose cell ``floor(p / cell)`` lies, per axis, within
  ``floor((c - r)/cell) .. floor((c + r)/cell)``, in ascending point order.
  (Warp also folds cells into a 128³ table; points reached only through that
  folding are at least 127 cells away and can never pass the callers' box test.)

The ``while wp.bvh_query_next(query, j):`` idiom writes ``j`` through an output
argument, which Python cannot express; ``make_golden.py`` rewrites that one line
of ``kernels_bvh.py`` / ``kernels_hashgrid.py`` into ``for j in query:`` before
executing them.
"""

from __future__ import annotations

import math
import sys
import types

import numpy as np

f32 = np.float32


def _f(x):
    return f32(x)


# ---------------------------------------------------------------------------
# value types
# ---------------------------------------------------------------------------
class vec3:
    __slots__ = ("v",)
    _n = 3

    def __init__(self, *args):
        if len(args) == 0:
            self.v = np.zeros(3, f32)
        elif len(args) == 1:
            self.v = np.array(args[0], dtype=f32).reshape(3)
        else:
            self.v = np.array([_f(a) for a in args], dtype=f32)

    @classmethod
    def _w(cls, arr):
        o = cls.__new__(cls)
        o.v = arr.astype(f32, copy=False)
        return o

    def __getitem__(self, i):
        return self.v[i]

    def __add__(self, o):
        return vec3._w(self.v + o.v)

    def __sub__(self, o):
        return vec3._w(self.v - o.v)

    def __neg__(self):
        return vec3._w(-self.v)

    def __mul__(self, s):
        if isinstance(s, (vec3, quat, mat33)):
            raise TypeError("vec3 * vector is not defined")
        return vec3._w(self.v * _f(s))

    __rmul__ = __mul__

    def __truediv__(self, s):
        return vec3._w(self.v / _f(s))

    def __repr__(self):
        return f"vec3({self.v[0]}, {self.v[1]}, {self.v[2]})"


class quat:
    __slots__ = ("v",)
    _n = 4

    def __init__(self, *args):
        if len(args) == 0:
            self.v = np.array([0, 0, 0, 1], f32)
        elif len(args) == 1:
            self.v = np.array(args[0], dtype=f32).reshape(4)
        else:
            self.v = np.array([_f(a) for a in args], dtype=f32)

    @classmethod
    def _w(cls, arr):
        o = cls.__new__(cls)
        o.v = arr.astype(f32, copy=False)
        return o

    def __getitem__(self, i):
        return self.v[i]

    def __add__(self, o):
        return quat._w(self.v + o.v)

    def __sub__(self, o):
        return quat._w(self.v - o.v)

    def __neg__(self):
        return quat._w(-self.v)

    def __mul__(self, o):
        if isinstance(o, quat):
            return quat._w(_qmul(self.v, o.v))
        return quat._w(self.v * _f(o))

    def __rmul__(self, s):
        return quat._w(self.v * _f(s))

    def __truediv__(self, s):
        return quat._w(self.v / _f(s))


class mat33:
    __slots__ = ("m",)

    def __init__(self, m):
        self.m = np.array(m, dtype=f32).reshape(3, 3)

    def __getitem__(self, ij):
        return self.m[ij]

    def __mul__(self, o):
        if isinstance(o, vec3):
            m = self.m
            a = o.v
            return vec3(m[0, 0] * a[0] + m[0, 1] * a[1] + m[0, 2] * a[2],
                        m[1, 0] * a[0] + m[1, 1] * a[1] + m[1, 2] * a[2],
                        m[2, 0] * a[0] + m[2, 1] * a[1] + m[2, 2] * a[2])
        raise TypeError("mat33 * non-vec3")


def _qmul(a, b):
    x1, y1, z1, w1 = a
    x2, y2, z2, w2 = b
    return np.array([
        ((w1 * x2 + x1 * w2) + y1 * z2) - z1 * y2,
        ((w1 * y2 - x1 * z2) + y1 * w2) + z1 * x2,
        ((w1 * z2 + x1 * y2) - y1 * x2) + z1 * w2,
        ((w1 * w2 - x1 * x2) - y1 * y2) - z1 * z2,
    ], dtype=f32)


class uint64:  # type marker only
    pass


# ---------------------------------------------------------------------------
# builtins
# ---------------------------------------------------------------------------
def constant(x):
    return x


def init():
    return None


def get_devices():
    return ["cpu"]


def synchronize_device(*_a, **_k):
    return None


_TID = [0]


def tid():
    return _TID[0]


def dot(a, b):
    x, y = a.v, b.v
    return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]


def cross(a, b):
    x, y = a.v, b.v
    return vec3(x[1] * y[2] - x[2] * y[1],
                x[2] * y[0] - x[0] * y[2],
                x[0] * y[1] - x[1] * y[0])


def length(a):
    if isinstance(a, quat):
        q = a.v
        return np.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    return np.sqrt(dot(a, a))


def normalize(a):
    ln = length(a)
    if ln > 0.0:
        return a / ln
    return type(a)._w(np.zeros(a._n, f32))


def abs(x):  # noqa: A001 - mirrors the warp builtin name
    return np.abs(_f(x))


def min(a, b):  # noqa: A001
    return a if a < b else b


def max(a, b):  # noqa: A001
    return a if a > b else b


def where(c, a, b):
    return a if c else b


def quat_rotate(q, v):
    x, y, z, w = q.v
    u = vec3(x, y, z)
    k = (_f(2.0) * w) * w - _f(1.0)
    a = v * k
    b = cross(u, v) * (_f(2.0) * w)
    c = u * (_f(2.0) * dot(u, v))
    return (a + b) + c


def quat_inverse(q):
    return quat._w(np.array([-q.v[0], -q.v[1], -q.v[2], q.v[3]], f32))


def quat_rotate_inv(q, v):
    return quat_rotate(quat_inverse(q), v)


def quat_to_matrix(q):
    x, y, z, w = q.v
    one, two = _f(1.0), _f(2.0)
    return mat33([
        [one - two * (y * y + z * z), two * (x * y - z * w), two * (x * z + y * w)],
        [two * (x * y + z * w), one - two * (x * x + z * z), two * (y * z - x * w)],
        [two * (x * z - y * w), two * (y * z + x * w), one - two * (x * x + y * y)],
    ])


def transpose(m):
    return mat33(m.m.T.copy())


def quat_from_axis_angle(axis, angle):
    s = math.sin(angle * 0.5)
    c = math.cos(angle * 0.5)
    return quat(axis[0] * s, axis[1] * s, axis[2] * s, c)


# ---------------------------------------------------------------------------
# arrays
# ---------------------------------------------------------------------------
class _ArrayType:
    def __init__(self, dtype):
        self.dtype = dtype


def _np_dtype(dtype):
    if dtype is float:
        return f32, ()
    if dtype is int:
        return np.int32, ()
    if dtype is vec3:
        return f32, (3,)
    if dtype is quat:
        return f32, (4,)
    raise TypeError(f"unsupported dtype {dtype}")


class warp_array:
    def __init__(self, data, dtype):
        nd, tail = _np_dtype(dtype)
        a = np.array(data, dtype=nd)
        if tail:
            a = a.reshape((-1,) + tail)
        self.a = a
        self.dtype = dtype

    def __len__(self):
        return self.a.shape[0]

    @property
    def shape(self):
        return (self.a.shape[0],)

    def __getitem__(self, i):
        i = int(i)
        if self.dtype is vec3:
            return vec3._w(self.a[i].copy())
        if self.dtype is quat:
            return quat._w(self.a[i].copy())
        if self.dtype is int:
            return int(self.a[i])
        return self.a[i]

    def __setitem__(self, i, val):
        i = int(i)
        if isinstance(val, (vec3, quat)):
            self.a[i] = val.v
        else:
            self.a[i] = val

    def numpy(self):
        return self.a

    def zero_(self):
        self.a[...] = 0

    def assign(self, src):
        self.a[...] = np.asarray(src).reshape(self.a.shape)


def array(data=None, dtype=float, device=None, **_kw):
    if data is None:
        return _ArrayType(dtype)
    return warp_array(data, dtype)


def zeros(n, dtype=float, device=None):
    nd, tail = _np_dtype(dtype)
    return warp_array(np.zeros((int(n),) + tail, nd), dtype)


def ones(n, dtype=float, device=None):
    nd, tail = _np_dtype(dtype)
    return warp_array(np.ones((int(n),) + tail, nd), dtype)


def atomic_add(arr, i, val):
    old = arr[i]
    if isinstance(val, vec3):
        arr[i] = old + val
    else:
        arr[i] = old + val
    return old


# ---------------------------------------------------------------------------
# kernels and launches
# ---------------------------------------------------------------------------
class _Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.ann = list(fn.__annotations__.items())
        self.__name__ = fn.__name__


def kernel(fn):
    return _Kernel(fn)


def func(fn):
    return fn


def _convert(val, ann):
    if ann is float:
        return _f(val)
    if ann is int:
        return int(val)
    if ann is vec3 and not isinstance(val, vec3):
        return vec3(*val)
    return val


def launch(k, dim, inputs=(), outputs=(), device=None):
    args = list(inputs) + list(outputs)
    anns = [a for name, a in k.ann if name != "return"]
    args = [_convert(v, a) for v, a in zip(args, anns)]
    for t in range(int(dim)):
        _TID[0] = t
        k.fn(*args)


# ---------------------------------------------------------------------------
# spatial queries
# ---------------------------------------------------------------------------
class Bvh:
    def __init__(self, lowers, uppers, constructor=None, device=None):
        self.lowers = lowers
        self.uppers = uppers
        self.id = self

    def rebuild(self):
        return None


def bvh_query_aabb(bvh, lo, hi):
    L = bvh.lowers.a
    U = bvh.uppers.a
    lo = lo.v
    hi = hi.v
    ok = np.all((L <= hi[None, :]) & (U >= lo[None, :]), axis=1)
    return [int(j) for j in np.nonzero(ok)[0]]


class HashGrid:
    def __init__(self, dx, dy, dz, device=None):
        self.pts = np.zeros((0, 3), f32)
        self.cell = 1.0
        self.id = self

    def build(self, points, cell):
        self.pts = points.a.copy()
        self.cell = _f(cell)


def hash_grid_query(grid, p, r):
    c = grid.cell
    lo = np.floor((p.v - _f(r)) / c)
    hi = np.floor((p.v + _f(r)) / c)
    cells = np.floor(grid.pts / c)
    ok = np.all((cells >= lo[None, :]) & (cells <= hi[None, :]), axis=1)
    return [int(j) for j in np.nonzero(ok)[0]]


class ScopedCapture:  # only reached on CUDA devices, which the shim never reports
    def __init__(self, *a, **k):
        raise RuntimeError("graph capture is not available in the CPU shim")


def capture_launch(_g):
    raise RuntimeError("graph capture is not available in the CPU shim")


def install():
    """Register this module as ``warp`` in ``sys.modules``."""
    mod = sys.modules[__name__]
    sys.modules["warp"] = mod
    return mod


TIMING_KERNEL = 0
types_ = types
