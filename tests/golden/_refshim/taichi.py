"""Import-only stand-in for `taichi`, used ONLY by make_golden.py.

It lets the reference's `@ti.func` source (rendering/taichi/*.py,
scene/primitives.py, scene/mesh.py) execute as plain Python with every value
held as a numpy float32 scalar, so the golden vectors are the reference's own
code path evaluated in IEEE float32 one operation at a time.  Vector
semantics follow Taichi's documented Matrix operations: elementwise + - * /,
`dot` as a left-to-right sum of products, `cross` for 3-vectors and
`normalized()` as v * (1 / norm).
"""
import math

import numpy as np

f32 = np.float32
i32 = "i32"
u8 = "u8"
cpu = "cpu"
gpu = "gpu"

_F = np.float32


def init(*args, **kwargs):
    return None


def func(fn):
    return fn


def kernel(fn):
    return fn


def static(x):
    return x


def _is_vec(x):
    return isinstance(x, Vector)


def _f(x):
    if isinstance(x, (int, np.integer)) and not isinstance(x, bool):
        return x
    return _F(x)


class Vector:
    """Small fixed-length vector of float32 (or int) scalars."""

    # make numpy scalars defer to Vector.__rmul__ etc. instead of broadcasting
    __array_ufunc__ = None

    def __init__(self, data, dt=None):
        if dt == "i32":
            self.e = [int(v) for v in data]
        else:
            self.e = [_F(v) for v in data]
        self.dt = dt

    # constructors -------------------------------------------------------
    @staticmethod
    def zero(dtype, n):
        if dtype == "i32":
            return Vector([0] * n, dt="i32")
        return Vector([0.0] * n)

    @staticmethod
    def field(n, dtype=None, shape=None):
        return Field(shape, vec=n, dtype=dtype)

    # element access -----------------------------------------------------
    def __getitem__(self, i):
        return self.e[i]

    def __setitem__(self, i, v):
        self.e[i] = int(v) if self.dt == "i32" else _F(v)

    def __len__(self):
        return len(self.e)

    def __iter__(self):
        return iter(self.e)

    # arithmetic ---------------------------------------------------------
    def _bin(self, o, op):
        if _is_vec(o):
            return Vector([op(a, b) for a, b in zip(self.e, o.e)])
        return Vector([op(a, o) for a in self.e])

    def _rbin(self, o, op):
        return Vector([op(o, a) for a in self.e])

    def __add__(self, o):
        return self._bin(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self._rbin(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._bin(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._rbin(o, lambda a, b: a - b)

    def __mul__(self, o):
        return self._bin(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self._rbin(o, lambda a, b: a * b)

    def __truediv__(self, o):
        return self._bin(o, lambda a, b: a / b)

    def __neg__(self):
        return Vector([-a for a in self.e])

    def dot(self, o):
        prods = [a * b for a, b in zip(self.e, o.e)]
        acc = prods[0]
        for p in prods[1:]:
            acc = acc + p
        return acc

    def sum(self):
        acc = self.e[0]
        for p in self.e[1:]:
            acc = acc + p
        return acc

    def cross(self, o):
        a, b = self.e, o.e
        return Vector([
            a[1] * b[2] - a[2] * b[1],
            a[2] * b[0] - a[0] * b[2],
            a[0] * b[1] - a[1] * b[0],
        ])

    def norm(self):
        return np.sqrt(self.dot(self))

    def normalized(self, eps=0):
        invlen = _F(1.0) / (self.norm() + _F(eps))
        return invlen * self

    def cast(self, dtype):
        return Vector([_F(v) for v in self.e])

    def to_list(self):
        return [float(v) for v in self.e]


class _Types:
    @staticmethod
    def vector(n, dtype):
        return ("vector", n, dtype)


types = _Types()


class Field:
    """numpy-backed stand-in for ti.field / ti.Vector.field."""

    def __init__(self, shape, vec=None, dtype=None):
        self.shape = shape if isinstance(shape, tuple) else ((shape,) if shape is not None else ())
        self.vec = vec
        self.dtype = dtype
        self.data = None

    def _alloc(self):
        if self.data is None:
            dt = np.int32 if self.dtype == "i32" else (np.uint8 if self.dtype == "u8" else np.float32)
            full = self.shape + ((self.vec,) if self.vec else ())
            if not self.shape:
                self.data = np.zeros(full or (1,), dtype=dt)
            else:
                # large capacities are only touched sparsely: start small, grow on demand
                self.data = {}
        return self.data

    def _key(self, idx):
        if idx is None:
            return 0
        return idx

    def __getitem__(self, idx):
        data = self._alloc()
        k = self._key(idx)
        if isinstance(data, dict):
            v = data.get(k)
            if v is None:
                if self.vec:
                    return Vector([0] * self.vec, dt="i32" if self.dtype == "i32" else None)
                return 0 if self.dtype == "i32" else _F(0.0)
            return v
        if self.vec:
            return Vector(list(data[k]), dt="i32" if self.dtype == "i32" else None)
        v = data[k]
        return int(v) if self.dtype == "i32" else _F(v)

    def __setitem__(self, idx, value):
        data = self._alloc()
        k = self._key(idx)
        if isinstance(data, dict):
            if self.vec:
                vals = value.e if isinstance(value, Vector) else list(value)
                data[k] = Vector(vals, dt="i32" if self.dtype == "i32" else None)
            else:
                data[k] = int(value) if self.dtype == "i32" else _F(value)
        else:
            data[k] = value.e if isinstance(value, Vector) else value

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if len(self.shape) > 1:
            # multi-index field (texture texels): keep the dense array
            self.data = arr.astype(np.uint8 if self.dtype == "u8" else arr.dtype, copy=True)
            return
        n = arr.shape[0]
        d = {}
        used = n
        # only keep rows that carry data (capacity arrays are zero-padded)
        if self.vec:
            nz = np.nonzero(np.any(arr.reshape(n, -1) != 0, axis=1))[0]
        else:
            nz = np.nonzero(arr != 0)[0]
        for i in nz:
            if self.vec:
                d[int(i)] = Vector(list(arr[i]), dt="i32" if self.dtype == "i32" else None)
            else:
                d[int(i)] = int(arr[i]) if self.dtype == "i32" else _F(arr[i])
        self.data = d
        self.used = used

    def to_numpy(self):
        raise NotImplementedError("to_numpy is not used by the golden generator")


def field(dtype=None, shape=None):
    return Field(shape, dtype=dtype)


# scalar math ---------------------------------------------------------------
def abs(x):  # noqa: A001 - mirrors ti.abs
    if _is_vec(x):
        return Vector([np.abs(a) for a in x.e])
    return np.abs(x)


def _scalar(v, a, b):
    both_int = all(isinstance(x, (int, np.integer)) and not isinstance(x, bool) for x in (a, b))
    return v if both_int else _F(v)


def min(a, b):  # noqa: A001
    if _is_vec(a) or _is_vec(b):
        av = a.e if _is_vec(a) else [a] * len(b.e)
        bv = b.e if _is_vec(b) else [b] * len(a.e)
        return Vector([x if x < y else y for x, y in zip(av, bv)])
    return _scalar(a if a < b else b, a, b)


def max(a, b):  # noqa: A001
    if _is_vec(a) or _is_vec(b):
        av = a.e if _is_vec(a) else [a] * len(b.e)
        bv = b.e if _is_vec(b) else [b] * len(a.e)
        return Vector([x if x > y else y for x, y in zip(av, bv)])
    return _scalar(a if a > b else b, a, b)


def sqrt(x):
    return np.sqrt(_F(x))


def sin(x):
    return np.sin(_F(x))


def cos(x):
    return np.cos(_F(x))


def acos(x):
    return np.arccos(_F(x))


def floor(x):
    return np.floor(_F(x))


def cast(x, dtype):
    if dtype == "i32":
        return int(x)
    return _F(x)


class _Ref:
    def __init__(self, fld, idx):
        self.fld = fld
        self.idx = idx


class CounterField(Field):
    """Field whose element reads return a reference usable by atomic_add."""

    def __init__(self):
        super().__init__((), dtype="i32")
        self.value = 0

    def __getitem__(self, idx):
        return _Ref(self, idx)

    def __setitem__(self, idx, value):
        self.value = int(value)


def atomic_add(ref, v):
    if isinstance(ref, _Ref):
        ref.fld.value += int(v)
    return None


# scripted random stream -----------------------------------------------------
_stream = []
_pos = [0]


def set_random_stream(values):
    global _stream
    _stream = [_F(v) for v in values]
    _pos[0] = 0


def consumed():
    return _pos[0]


def random():
    i = _pos[0]
    _pos[0] += 1
    if i < len(_stream):
        return _stream[i]
    return _F(0.5)


def ndrange(*dims):
    import itertools
    return itertools.product(*[range(d) for d in dims])


pi = math.pi
