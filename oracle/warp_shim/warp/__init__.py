"""A pure-Python stand-in for the parts of NVIDIA Warp (warp-lang 1.13.0,
pinned by the reference's uv.lock:904-915) that avbd3d's Solver6DOF uses --
TEST INFRASTRUCTURE ONLY.

warp-lang is not installed and cannot be installed offline, so the
reference's own source (src/avbd3d/solver_6dof.py and kernels_6dof.py) is run
through this module instead: `import warp as wp` resolves here when
`oracle/warp_shim` comes first on sys.path.  Nothing of the reference is
copied or edited; its kernel functions are executed as written, one thread
index after another (tid = 0, 1, ... dim-1), which is how Warp's CPU device
runs a launch.

Kernel-language semantics that plain Python does not have are supplied by a
source transform applied to every @wp.kernel / @wp.func before its first
call:
  * value semantics of vectors and matrices: `v[i] = x` rebinds `v` to a
    modified copy (vectors are immutable here); on a wp.array the same
    statement writes the element in place;
  * `float(x)`, `int(x)` and float literals are Warp's 32-bit types (numpy
    float32 scalars, so every operation rounds to float32 like the
    reference's float32 arrays and kernels; AVBD_WARP_SHIM_PRECISION=float64
    switches the whole run to float64);
  * C integer arithmetic (int32 wrap-around, truncating `/` and `%`) in
    every function that uses bitwise, shift or modulo operators (the contact
    hash, kernels_6dof.py:2597-2603);
  * `while wp.bvh_query_next(query, j):` assigns the next hit to `j`.

Warp internals that are not part of the reference tree -- the exact
floating-point formulation of quat_rotate, quat_to_matrix, inverse and
normalize, and the BVH query -- are written here in the same form as the
C++ oracle (oracle/avbd_oracle.cpp), so a comparison of the two checks the
reference's kernel logic (axis order, tie breaks, clipping, emission order,
cache, coloring rounds, iteration loop), not those internals.  The BVH query
is a brute-force closed-interval AABB overlap test reporting hits in index
order.
"""

from __future__ import annotations

import ast
import ctypes
import ctypes.util
import inspect
import itertools
import math
import operator
import os
import textwrap
import types as _pytypes

import numpy as np

__version__ = "1.13.0-avbd-shim"

_PREC = os.environ.get("AVBD_WARP_SHIM_PRECISION", "float32")
_S = np.float64 if _PREC == "float64" else np.float32
_F32 = _S is np.float32

# --------------------------------------------------------------------------
# scalar types
# --------------------------------------------------------------------------
float32 = _S
float64 = np.float64
int32 = int
inf = _S(np.inf)
pi = _S(math.pi)


def _to_float(x=0.0):
    return _S(x)


def _to_int(x=0):
    if isinstance(x, U32):
        return x.v
    return int(x)


class U32:
    """uint32 with wrap-around (the coloring kernels' used-color masks)."""
    __slots__ = ("v",)

    def __init__(self, v=0):
        self.v = int(v.v if isinstance(v, U32) else v) & 0xFFFFFFFF

    @staticmethod
    def _o(o):
        return o.v if isinstance(o, U32) else int(o)

    def __or__(self, o): return U32(self.v | self._o(o))
    __ror__ = __or__
    def __and__(self, o): return U32(self.v & self._o(o))
    __rand__ = __and__
    def __xor__(self, o): return U32(self.v ^ self._o(o))
    __rxor__ = __xor__
    def __lshift__(self, o): return U32(self.v << self._o(o))
    def __rshift__(self, o): return U32(self.v >> self._o(o))
    def __add__(self, o): return U32(self.v + self._o(o))
    __radd__ = __add__
    def __sub__(self, o): return U32(self.v - self._o(o))
    def __mul__(self, o): return U32(self.v * self._o(o))
    __rmul__ = __mul__
    def __invert__(self): return U32(~self.v)
    def __eq__(self, o): return self.v == self._o(o)
    def __ne__(self, o): return self.v != self._o(o)
    def __lt__(self, o): return self.v < self._o(o)
    def __gt__(self, o): return self.v > self._o(o)
    def __le__(self, o): return self.v <= self._o(o)
    def __ge__(self, o): return self.v >= self._o(o)
    def __bool__(self): return self.v != 0
    def __int__(self): return self.v
    def __index__(self): return self.v
    def __hash__(self): return hash(self.v)
    def __repr__(self): return f"uint32({self.v})"


uint32 = U32


def uint64(v=0):
    return int(v) & 0xFFFFFFFFFFFFFFFF


def _wrap32(r: int) -> int:
    r &= 0xFFFFFFFF
    return r - 0x100000000 if r >= 0x80000000 else r


def _c_div(a: int, b: int) -> int:
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


_PYOPS = {
    "Add": operator.add, "Sub": operator.sub, "Mult": operator.mul, "Div": operator.truediv,
    "Mod": operator.mod, "FloorDiv": operator.floordiv, "Pow": operator.pow, "LShift": operator.lshift,
    "RShift": operator.rshift, "BitOr": operator.or_, "BitXor": operator.xor, "BitAnd": operator.and_,
    "MatMult": operator.matmul,
}


def _binop(op: str, a, b):
    """One binary operation with Warp's semantics: two (non-bool) Python ints
    are int32 values (wrap-around, truncating division and remainder)."""
    if type(a) is int and type(b) is int:
        if op == "Div" or op == "FloorDiv":
            return _wrap32(_c_div(a, b))
        if op == "Mod":
            return _wrap32(a - b * _c_div(a, b))
        return _wrap32(_PYOPS[op](a, b))
    return _PYOPS[op](a, b)


# --------------------------------------------------------------------------
# vectors, quaternions, matrices (immutable values)
# --------------------------------------------------------------------------
def _new(cls, c):
    o = object.__new__(cls)
    o.c = c
    return o


class _Vec:
    __slots__ = ("c",)
    __array_ufunc__ = None  # numpy scalars defer to our reflected operators
    _n = 3
    _int = False

    def __init__(self, *a):
        n = self._n
        conv = int if self._int else _S
        if not a:
            c = (conv(0),) * n
        elif len(a) == 1:
            x = a[0]
            if isinstance(x, _Vec):
                c = tuple(conv(v) for v in x.c)
            elif isinstance(x, (list, tuple, np.ndarray)):
                c = tuple(conv(v) for v in x)
            else:
                c = (conv(x),) * n
        else:
            c = tuple(conv(v) for v in a)
        if len(c) != n:
            raise ValueError(f"{type(self).__name__} needs {n} components, got {len(c)}")
        self.c = c

    def __len__(self):
        return self._n

    def __iter__(self):
        return iter(self.c)

    def __getitem__(self, i):
        return self.c[i]

    def _set(self, i, v):
        c = list(self.c)
        c[int(i)] = int(v) if self._int else _S(v)
        return _new(type(self), tuple(c))

    def __add__(self, o):
        return _new(type(self), tuple(a + b for a, b in zip(self.c, o.c)))

    def __sub__(self, o):
        return _new(type(self), tuple(a - b for a, b in zip(self.c, o.c)))

    def __neg__(self):
        return _new(type(self), tuple(-a for a in self.c))

    def __pos__(self):
        return self

    def __mul__(self, s):
        if isinstance(s, (_Vec, _Mat)):
            return NotImplemented
        return _new(type(self), tuple(a * s for a in self.c))

    def __rmul__(self, s):
        if isinstance(s, (_Vec, _Mat)):
            return NotImplemented
        return _new(type(self), tuple(s * a for a in self.c))

    def __truediv__(self, s):
        return _new(type(self), tuple(a / s for a in self.c))

    def __eq__(self, o):
        return isinstance(o, _Vec) and self.c == o.c

    def __hash__(self):
        return hash(self.c)

    def __repr__(self):
        return f"{type(self).__name__}({', '.join(str(v) for v in self.c)})"

    @property
    def x(self):
        return self.c[0]

    @property
    def y(self):
        return self.c[1]

    @property
    def z(self):
        return self.c[2]

    @property
    def w(self):
        return self.c[3]


class vec3(_Vec):
    __slots__ = ()
    _n = 3


class vec4(_Vec):
    __slots__ = ()
    _n = 4


class quat(_Vec):
    """XYZW quaternion; quat * quat is the Hamilton product."""
    __slots__ = ()
    _n = 4

    def __init__(self, *a):
        if not a:
            self.c = (_S(0), _S(0), _S(0), _S(0))
        else:
            super().__init__(*a)

    def __mul__(self, o):
        if isinstance(o, quat):
            return _qmul(self, o)
        return super().__mul__(o)


def _vector_type(length, dtype=float):
    is_int = dtype in (int, int32)
    name = f"vec{length}{'i' if is_int else ''}"
    return type(name, (_Vec,), {"__slots__": (), "_n": int(length), "_int": is_int})


class _Mat:
    """3x3 matrix stored by rows."""
    __slots__ = ("r",)
    __array_ufunc__ = None

    def __init__(self, *a):
        if not a:
            z = _S(0)
            self.r = ((z, z, z), (z, z, z), (z, z, z))
        elif len(a) == 9:
            v = [_S(x) for x in a]
            self.r = (tuple(v[0:3]), tuple(v[3:6]), tuple(v[6:9]))
        elif len(a) == 1 and isinstance(a[0], (np.ndarray, list, tuple)):
            m = np.asarray(a[0]).reshape(3, 3)
            self.r = tuple(tuple(_S(x) for x in row) for row in m)
        else:
            raise ValueError("mat33 takes 0 or 9 scalars")

    @staticmethod
    def _mk(rows):
        o = object.__new__(_Mat)
        o.r = rows
        return o

    def __getitem__(self, ij):
        if isinstance(ij, tuple):
            return self.r[ij[0]][ij[1]]
        return _new(vec3, self.r[ij])

    def _set(self, ij, v):
        rows = [list(r) for r in self.r]
        if isinstance(ij, tuple):
            rows[int(ij[0])][int(ij[1])] = _S(v)
        else:
            rows[int(ij)] = [_S(x) for x in v]
        return _Mat._mk(tuple(tuple(r) for r in rows))

    def __add__(self, o):
        return _Mat._mk(tuple(tuple(a + b for a, b in zip(ra, rb)) for ra, rb in zip(self.r, o.r)))

    def __sub__(self, o):
        return _Mat._mk(tuple(tuple(a - b for a, b in zip(ra, rb)) for ra, rb in zip(self.r, o.r)))

    def __neg__(self):
        return _Mat._mk(tuple(tuple(-a for a in r) for r in self.r))

    def __mul__(self, o):
        if isinstance(o, _Mat):
            return _mm(self, o)
        if isinstance(o, _Vec):
            return _mv(self, o)
        return _Mat._mk(tuple(tuple(a * o for a in r) for r in self.r))

    def __rmul__(self, s):
        if isinstance(s, _Vec):  # row vector times matrix
            v = s.c
            r = self.r
            return _new(vec3, tuple(v[0] * r[0][j] + v[1] * r[1][j] + v[2] * r[2][j] for j in range(3)))
        return _Mat._mk(tuple(tuple(s * a for a in r) for r in self.r))

    def __truediv__(self, s):
        return _Mat._mk(tuple(tuple(a / s for a in r) for r in self.r))

    def __repr__(self):
        return f"mat33({self.r})"


mat33 = _Mat


def _mv(A, v):
    r, c = A.r, v.c
    return _new(vec3, (r[0][0] * c[0] + r[0][1] * c[1] + r[0][2] * c[2],
                       r[1][0] * c[0] + r[1][1] * c[1] + r[1][2] * c[2],
                       r[2][0] * c[0] + r[2][1] * c[1] + r[2][2] * c[2]))


def _mm(A, B):
    a, b = A.r, B.r
    return _Mat._mk(tuple(tuple(a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j] for j in range(3))
                          for i in range(3)))


def _qmul(a, b):
    ax, ay, az, aw = a.c
    bx, by, bz, bw = b.c
    return _new(quat, (aw * bx + bw * ax + (ay * bz - az * by),
                       aw * by + bw * ay + (az * bx - ax * bz),
                       aw * bz + bw * az + (ax * by - ay * bx),
                       aw * bw - (ax * bx + ay * by + az * bz)))


class types:  # noqa: N801  (the wp.types namespace)
    vector = staticmethod(_vector_type)
    float32 = _S
    int32 = int


# --------------------------------------------------------------------------
# built-in functions of the kernel language
# --------------------------------------------------------------------------
def dot(a, b):
    x, y = a.c, b.c
    if len(x) == 3:
        return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]
    return sum(p * q for p, q in zip(x, y))


def cross(a, b):
    x, y = a.c, b.c
    return _new(vec3, (x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]))


def length(a):
    return _S(np.sqrt(dot(a, a)))


def length_sq(a):
    return dot(a, a)


def normalize(a):
    n = length(a)
    if n > _S(0):
        s = _S(1) / n
        return _new(type(a), tuple(v * s for v in a.c))
    return a


def abs(x):  # noqa: A001
    if isinstance(x, _Vec):
        return _new(type(x), tuple(np.abs(v) for v in x.c))
    return np.abs(x) if isinstance(x, np.floating) else (x if x >= 0 else -x)


def min(a, b):  # noqa: A001
    return a if a < b else b


def max(a, b):  # noqa: A001
    return a if a > b else b


def clamp(x, lo, hi):
    return min(max(x, lo), hi)


def where(cond, a, b):
    return a if cond else b


def select(cond, a, b):  # Warp's older spelling: select(cond, if_false, if_true)
    return b if cond else a


def sqrt(x):
    return _S(np.sqrt(_S(x)))


# Transcendentals come from the C math library, as on Warp's CPU device
# (numpy's own float32 sin / cos / atan2 differ from libm in the last bit).
_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")


def _cfun(name1, nargs):
    name = name1 + ("f" if _F32 else "")
    f = getattr(_libm, name)
    t = ctypes.c_float if _F32 else ctypes.c_double
    f.restype = t
    f.argtypes = [t] * nargs
    return f


_sin, _cos, _atan2, _acos, _exp, _log = (_cfun("sin", 1), _cfun("cos", 1), _cfun("atan2", 2), _cfun("acos", 1),
                                         _cfun("exp", 1), _cfun("log", 1))


def sin(x):
    return _S(_sin(float(x)))


def cos(x):
    return _S(_cos(float(x)))


def atan2(y, x):
    return _S(_atan2(float(y), float(x)))


def acos(x):
    return _S(_acos(float(x)))


def exp(x):
    return _S(_exp(float(x)))


def log(x):
    return _S(_log(float(x)))


def floor(x):
    return _S(np.floor(_S(x)))


def sign(x):
    return _S(1) if x >= 0 else _S(-1)


def isnan(x):
    if isinstance(x, _Vec):
        return any(np.isnan(v) for v in x.c)
    return bool(np.isnan(x))


def isfinite(x):
    return bool(np.isfinite(x))


def transpose(m):
    r = m.r
    return _Mat._mk(((r[0][0], r[1][0], r[2][0]), (r[0][1], r[1][1], r[2][1]), (r[0][2], r[1][2], r[2][2])))


def determinant(m):
    r = m.r
    c00 = r[1][1] * r[2][2] - r[1][2] * r[2][1]
    c01 = r[1][2] * r[2][0] - r[1][0] * r[2][2]
    c02 = r[1][0] * r[2][1] - r[1][1] * r[2][0]
    return r[0][0] * c00 + r[0][1] * c01 + r[0][2] * c02


def inverse(m):
    """3x3 inverse by the adjugate; a singular matrix gives zero."""
    r = m.r
    c00 = r[1][1] * r[2][2] - r[1][2] * r[2][1]
    c01 = r[1][2] * r[2][0] - r[1][0] * r[2][2]
    c02 = r[1][0] * r[2][1] - r[1][1] * r[2][0]
    det = r[0][0] * c00 + r[0][1] * c01 + r[0][2] * c02
    if det == _S(0):
        return _Mat()
    i = _S(1) / det
    return _Mat._mk(((c00 * i, (r[0][2] * r[2][1] - r[0][1] * r[2][2]) * i, (r[0][1] * r[1][2] - r[0][2] * r[1][1]) * i),
                     (c01 * i, (r[0][0] * r[2][2] - r[0][2] * r[2][0]) * i, (r[0][2] * r[1][0] - r[0][0] * r[1][2]) * i),
                     (c02 * i, (r[0][1] * r[2][0] - r[0][0] * r[2][1]) * i, (r[0][0] * r[1][1] - r[0][1] * r[1][0]) * i)))


def diag(v):
    z = _S(0)
    return _Mat._mk(((v.c[0], z, z), (z, v.c[1], z), (z, z, v.c[2])))


def outer(a, b):
    return _Mat._mk(tuple(tuple(p * q for q in b.c) for p in a.c))


def mul(a, b):
    return a * b


def quat_inverse(q):
    x, y, z, w = q.c
    return _new(quat, (-x, -y, -z, w))


def quat_identity():
    return _new(quat, (_S(0), _S(0), _S(0), _S(1)))


def quat_rotate(q, v):
    """v' = (2w^2 - 1) v + 2 (q.v) q + 2 w (q x v)."""
    qx, qy, qz, qw = q.c
    vx, vy, vz = v.c
    c = _S(2) * qw * qw - _S(1)
    d = _S(2) * (qx * vx + qy * vy + qz * vz)
    w2 = qw * _S(2)
    return _new(vec3, (vx * c + qx * d + (qy * vz - qz * vy) * w2,
                       vy * c + qy * d + (qz * vx - qx * vz) * w2,
                       vz * c + qz * d + (qx * vy - qy * vx) * w2))


def quat_rotate_inv(q, v):
    return quat_rotate(quat_inverse(q), v)


def quat_to_matrix(q):
    x, y, z, w = q.c
    one, two = _S(1), _S(2)
    return _Mat._mk(((one - two * (y * y + z * z), two * (x * y - z * w), two * (x * z + y * w)),
                     (two * (x * y + z * w), one - two * (x * x + z * z), two * (y * z - x * w)),
                     (two * (x * z - y * w), two * (y * z + x * w), one - two * (x * x + y * y))))


def quat_from_axis_angle(axis, angle):
    h = _S(0.5) * _S(angle)
    s = sin(h)
    return _new(quat, (axis.c[0] * s, axis.c[1] * s, axis.c[2] * s, cos(h)))


# --------------------------------------------------------------------------
# arrays
# --------------------------------------------------------------------------
def _elem_layout(dtype):
    """(numpy dtype, element shape, element kind) of a Warp dtype."""
    if dtype in (float, float32, np.float32, np.float64):
        return _S, (), "f"
    if dtype in (int, int32, np.int32):
        return np.int32, (), "i"
    if dtype is U32:
        return np.uint32, (), "u32"
    if dtype is uint64:
        return np.uint64, (), "u64"
    if dtype is bool:
        return np.bool_, (), "b"
    if dtype is mat33:
        return _S, (3, 3), "m"
    if isinstance(dtype, type) and issubclass(dtype, _Vec):
        return (np.int32 if dtype._int else _S), (dtype._n,), dtype
    raise TypeError(f"warp shim: unsupported dtype {dtype!r}")


class array:  # noqa: N801
    """A Warp array on the CPU device, backed by a numpy array of shape
    (n, *element_shape).  `wp.array(dtype=...)` with no data is the kernel
    argument annotation and holds nothing."""

    def __init__(self, data=None, dtype=float, shape=None, device=None, copy=True, **_kw):
        self.dtype = dtype
        self.device = device or "cpu"
        if data is None and shape is None:
            self._np = None  # annotation only
            return
        npdt, eshape, kind = _elem_layout(dtype)
        self._kind = kind
        if data is None:
            n = shape if isinstance(shape, int) else int(shape[0])
            self._np = np.zeros((n,) + eshape, dtype=npdt)
        else:
            if isinstance(data, array):
                data = data._np
            a = np.array(data, dtype=npdt, copy=True)
            n = a.size // int(np.prod(eshape)) if eshape else a.size
            self._np = a.reshape((n,) + eshape)

    # ---- host-side API used by the reference ----
    @property
    def shape(self):
        return (self._np.shape[0],)

    @property
    def size(self):
        return self._np.shape[0]

    def __len__(self):
        return self._np.shape[0]

    def numpy(self):
        return self._np

    def assign(self, src):
        src = src._np if isinstance(src, array) else np.asarray(src)
        self._np[...] = src.reshape(self._np.shape)

    def zero_(self):
        self._np[...] = 0

    def fill_(self, value):
        if isinstance(value, _Vec):
            self._np[...] = np.asarray(value.c)
        else:
            self._np[...] = value

    def to(self, device):
        return self

    # ---- element access inside kernels ----
    def __getitem__(self, i):
        kind = self._kind
        if kind == "f":
            return self._np[i]
        if kind == "i":
            return int(self._np[i])
        if kind == "m":
            return _Mat._mk(tuple(tuple(row) for row in self._np[i]))
        if kind == "u32":
            return U32(int(self._np[i]))
        if kind in ("u64", "b"):
            return int(self._np[i])
        row = self._np[i]
        if kind._int:
            return _new(kind, tuple(int(v) for v in row))
        return _new(kind, tuple(row))

    def __setitem__(self, i, v):
        kind = self._kind
        if kind == "m":
            self._np[i] = np.asarray(v.r)
        elif isinstance(v, _Vec):
            self._np[i] = v.c
        elif isinstance(v, U32):
            self._np[i] = v.v
        else:
            self._np[i] = v

    def _set(self, i, v):
        self[i] = v
        return self


def zeros(shape, dtype=float, device=None, **_kw):
    return array(None, dtype=dtype, shape=shape, device=device)


def empty(shape, dtype=float, device=None, **_kw):
    return zeros(shape, dtype=dtype, device=device)


def full(shape, value, dtype=float, device=None, **_kw):
    a = zeros(shape, dtype=dtype, device=device)
    a.fill_(value)
    return a


def zeros_like(a):
    return zeros(a.shape[0], dtype=a.dtype, device=a.device)


def clone(a):
    return array(a._np, dtype=a.dtype, device=a.device)


def copy(dest, src, dest_offset=0, src_offset=0, count=0):
    n = count if count else src.shape[0] - src_offset
    dest._np[dest_offset:dest_offset + n] = src._np[src_offset:src_offset + n]


def atomic_add(arr, i, v):
    old = arr[i]
    arr[i] = old + v
    return old


def atomic_sub(arr, i, v):
    old = arr[i]
    arr[i] = old - v
    return old


def atomic_max(arr, i, v):
    old = arr[i]
    if v > old:
        arr[i] = v
    return old


def atomic_min(arr, i, v):
    old = arr[i]
    if v < old:
        arr[i] = v
    return old


def atomic_cas(arr, i, compare, value):
    old = arr[i]
    if old == compare:
        arr[i] = value
    return old


# --------------------------------------------------------------------------
# BVH: brute-force closed-interval overlap, hits in index order
# --------------------------------------------------------------------------
_BVHS: dict = {}
_BVH_IDS = itertools.count(1)


class Bvh:
    def __init__(self, lowers, uppers, constructor=None, **_kw):
        self.lowers, self.uppers = lowers, uppers
        self.id = next(_BVH_IDS)
        _BVHS[self.id] = self
        self.refit()

    def refit(self):
        self._lo = self.lowers._np.copy()
        self._hi = self.uppers._np.copy()

    rebuild = refit


class _BvhQuery:
    __slots__ = ("hits", "k")

    def __init__(self, hits):
        self.hits = hits
        self.k = 0


def bvh_query_aabb(bvh_id, lo, hi):
    b = _BVHS[int(bvh_id)]
    lo, hi = np.asarray(lo.c, dtype=b._lo.dtype), np.asarray(hi.c, dtype=b._hi.dtype)
    m = np.all(b._lo <= hi, axis=1) & np.all(lo <= b._hi, axis=1)
    return _BvhQuery([int(j) for j in np.nonzero(m)[0]])


def _bvh_next(q):
    if q.k < len(q.hits):
        j = q.hits[q.k]
        q.k += 1
        return True, j
    return False, 0


def bvh_query_next(q, _index):  # only reachable untransformed: a programming error here
    raise RuntimeError("bvh_query_next is rewritten by the warp shim's kernel transform")


# --------------------------------------------------------------------------
# kernels, functions and launches
# --------------------------------------------------------------------------
_TID = [0]


def tid():
    return _TID[0]


_INT_OPS = (ast.BitAnd, ast.BitOr, ast.BitXor, ast.LShift, ast.RShift, ast.Mod, ast.FloorDiv)


class _KernelTransform(ast.NodeTransformer):
    def __init__(self, exact_ints: bool):
        self.exact_ints = exact_ints
        self.consts: dict = {}
        self.k = 0

    def _subscript_assign(self, tgt, value):
        base = tgt.value
        if isinstance(base, ast.Name):
            call = ast.Call(func=ast.Name("__wp_set", ast.Load()),
                            args=[ast.Name(base.id, ast.Load()), tgt.slice, value], keywords=[])
            return ast.Assign(targets=[ast.Name(base.id, ast.Store())], value=call)
        if isinstance(base, ast.Subscript) and isinstance(base.value, ast.Name):  # m[i][j] = v
            inner = ast.Call(func=ast.Name("__wp_set", ast.Load()),
                             args=[ast.Subscript(ast.Name(base.value.id, ast.Load()), base.slice, ast.Load()),
                                   tgt.slice, value], keywords=[])
            return self._subscript_assign(ast.Subscript(base.value, base.slice, ast.Store()), inner)
        raise NotImplementedError(f"warp shim: subscript assignment to {ast.dump(base)}")

    def visit_Assign(self, node):
        self.generic_visit(node)
        if len(node.targets) == 1 and isinstance(node.targets[0], ast.Subscript):
            return self._subscript_assign(node.targets[0], node.value)
        return node

    def visit_AnnAssign(self, node):
        self.generic_visit(node)
        if node.value is None:
            return None
        a = ast.Assign(targets=[node.target], value=node.value)
        if isinstance(node.target, ast.Subscript):
            return self._subscript_assign(node.target, node.value)
        return a

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        tgt = node.target
        load = ast.Subscript(tgt.value, tgt.slice, ast.Load()) if isinstance(tgt, ast.Subscript) else \
            ast.Name(tgt.id, ast.Load())
        val = self._binop_node(node.op, load, node.value)
        if isinstance(tgt, ast.Subscript):
            return self._subscript_assign(tgt, val)
        return ast.Assign(targets=[ast.Name(tgt.id, ast.Store())], value=val)

    def _binop_node(self, op, left, right):
        if self.exact_ints:
            return ast.Call(func=ast.Name("__wp_binop", ast.Load()),
                            args=[ast.Constant(type(op).__name__), left, right], keywords=[])
        return ast.BinOp(left=left, op=op, right=right)

    def visit_BinOp(self, node):
        self.generic_visit(node)
        if self.exact_ints:
            return self._binop_node(node.op, node.left, node.right)
        return node

    def visit_Constant(self, node):
        if _F32 and type(node.value) is float:
            name = f"__wpf{self.k}"
            self.k += 1
            self.consts[name] = _S(node.value)
            return ast.Name(name, ast.Load())
        return node

    def visit_While(self, node):
        self.generic_visit(node)
        t = node.test
        if (isinstance(t, ast.Call) and isinstance(t.func, ast.Attribute) and t.func.attr == "bvh_query_next"):
            q, var = t.args
            fetch = ast.Assign(targets=[ast.Tuple([ast.Name("__wp_ok", ast.Store()), ast.Name(var.id, ast.Store())],
                                                  ast.Store())],
                               value=ast.Call(func=ast.Name("__wp_bvh_next", ast.Load()), args=[q], keywords=[]))
            stop = ast.If(test=ast.UnaryOp(ast.Not(), ast.Name("__wp_ok", ast.Load())), body=[ast.Break()], orelse=[])
            return ast.While(test=ast.Constant(True), body=[fetch, stop] + node.body, orelse=node.orelse)
        return node


def _set(obj, i, v):
    return obj._set(i, v)


def _compile(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    for a in fdef.args.args + fdef.args.kwonlyargs:
        a.annotation = None
    fdef.returns = None
    exact = any(isinstance(n, ast.BinOp) and isinstance(n.op, _INT_OPS) for n in ast.walk(fdef))
    tr = _KernelTransform(exact)
    tree = ast.fix_missing_locations(tr.visit(tree))
    g = dict(fn.__globals__)
    g.update(tr.consts)
    g.update({"__wp_set": _set, "__wp_binop": _binop, "__wp_bvh_next": _bvh_next, "float": _to_float,
              "int": _to_int})
    code = compile(tree, filename=inspect.getsourcefile(fn) or "<warp-shim>", mode="exec")
    exec(code, g)
    return g[fdef.name]


class Function:
    def __init__(self, fn):
        self.fn = fn
        self.key = fn.__name__
        self.__name__ = fn.__name__
        self.__doc__ = fn.__doc__
        self._c = None

    def __call__(self, *a, **k):
        c = self._c
        if c is None:
            c = self._c = _compile(self.fn)
        return c(*a, **k)


class Kernel(Function):
    pass


def func(fn=None, **_kw):
    if fn is None:
        return lambda f: Function(f)
    return Function(fn)


def kernel(fn=None, **_kw):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def func_native(snippet=None, adj_snippet=None, **_kw):
    """CUDA-only native snippets (warp shuffles) have no CPU meaning; calling
    one here is an error."""
    def deco(f):
        def native(*_a, **_k):
            raise RuntimeError(f"warp shim: {f.__name__} is a CUDA-only native function")
        native.__name__ = f.__name__
        return native
    return deco


def _launch_arg(a):
    if isinstance(a, float):
        return _S(a)
    if isinstance(a, (bool, np.bool_)):
        return int(a)
    return a


def launch(kernel, dim, inputs=(), outputs=(), device=None, **_kw):  # noqa: A002
    if isinstance(dim, (tuple, list)):
        if len(dim) != 1:
            raise NotImplementedError("warp shim: multi-dimensional launches are CUDA-only paths here")
        dim = dim[0]
    args = [_launch_arg(a) for a in list(inputs) + list(outputs)]
    fn = kernel if not isinstance(kernel, Function) else None
    if fn is None:
        if kernel._c is None:
            kernel._c = _compile(kernel.fn)
        fn = kernel._c
    with np.errstate(all="ignore"):
        for t in range(int(dim)):
            _TID[0] = t
            fn(*args)


def constant(v):
    return _S(v) if isinstance(v, float) else v


def init():
    return None


def set_module_options(*_a, **_k):
    return None


def synchronize(*_a, **_k):
    return None


def get_device(d=None):
    return d or "cpu"


def is_cuda_available():
    return False


class Tape:  # the 3-DOF module names it; AVBD never records one
    def __init__(self, *a, **k):
        raise RuntimeError("warp shim: autodiff tapes are not supported")


config = _pytypes.SimpleNamespace(mode="release", verbose=False, quiet=True)
