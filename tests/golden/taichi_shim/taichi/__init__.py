"""A minimal, pure-Python stand-in for the subset of Taichi that the reference
project's adaptive_gimp.py, utils.py and init.py use.

TEST INFRASTRUCTURE ONLY.  Taichi cannot be installed in this environment, so
tests/golden/make_golden.py puts this package first on sys.path and imports the
reference's own source files, which then run serially in Python.  The shim
emulates the semantics the reference relies on:

* kernels and funcs run as plain Python; struct-for loops over a sparse field
  visit the elements active when the loop starts, in sorted index order;
* sparse storage (pointer / bitmasked / dense / dynamic SNodes): an element is
  activated by a write, reading an inactive element returns 0, and
  ``deactivate_all`` frees everything under a pointer;
* f32 arithmetic: float values are numpy float32 and every binary operation
  rounds to f32 (Taichi's default_fp); Python float constants are cast to f32
  where they meet a field value, as Taichi's constant folding does;
* integer casts truncate toward zero; ``//`` and ``%`` follow Python;
* ``ti.svd`` is replaced by a float64 SVD (numpy) with the rotation-variant
  sign convention (det U = det V = +1), rounded to f32.

It does not emulate Taichi's fast-math code generation, its out-of-range
index behaviour, or its parallel scheduling.
"""
from __future__ import annotations

import builtins
import itertools
import types

import numpy as np

f32 = np.float32
f64 = np.float64
i32 = np.int32
i64 = np.int64
u8 = np.uint8

cpu = "cpu"
cuda = "cuda"


def init(*a, **k):
    pass


def _is_float_dt(dt):
    return dt in (float, f32, f64) or getattr(dt, "_is_ti_float", False)


def _np_dt(dt):
    return np.float32 if _is_float_dt(dt) else np.int32


class _FloatCast:
    """Stand-in for the builtin ``float`` inside reference modules: it is both a
    dtype marker (``ti.field(float)``) and a cast that works on vectors."""
    _is_ti_float = True

    def __new__(cls, x=0.0):
        x = _val(x)
        if isinstance(x, Mat):
            return x.cast(float)
        return np.float32(x)


def _val(x):
    if isinstance(x, Ref):
        return x.get()
    return x


def _scal(x):
    """Normalise a scalar operand: Python float -> f32, ints stay ints."""
    x = _val(x)
    if isinstance(x, (bool, np.bool_)):
        return x
    if isinstance(x, float):
        return np.float32(x)
    return x


# ----------------------------------------------------------------------------
def _unwrap_list(a):
    if isinstance(a, Mat):
        return a.a.tolist()
    if isinstance(a, (list, tuple)):
        return [_unwrap_list(e) for e in a]
    return _val(a)


class Mat:
    """Vector (1-D) or matrix (2-D) value with Taichi-like promotion rules."""
    __array_ufunc__ = None  # make numpy scalars defer to the reflected operators

    def __init__(self, a, dt=None):
        a = np.array(_unwrap_list(a))
        if dt is not None:
            a = a.astype(_np_dt(dt))
        elif a.dtype.kind == "f":
            a = a.astype(np.float32)
        elif a.dtype.kind in "iu":
            a = a.astype(np.int64)
        self.a = a

    # -- construction helpers
    @staticmethod
    def _wrap(a):
        m = Mat.__new__(Mat)
        m.a = a
        return m

    # -- container protocol
    def __len__(self):
        return self.a.shape[0]

    def __iter__(self):
        for e in self.a:
            yield e if np.ndim(e) == 0 else Mat._wrap(e)

    def __getitem__(self, k):
        k = _key(k)
        r = self.a[k]
        return Mat._wrap(np.array(r)) if np.ndim(r) else r

    def __setitem__(self, k, val):
        k = _key(k)
        val = _val(val)
        if isinstance(val, Mat):
            val = val.a
        self.a[k] = val

    def __bool__(self):
        return bool(np.all(self.a))

    def __repr__(self):
        return "Mat(%r)" % (self.a,)

    # -- elementwise arithmetic
    def _bin(self, o, fn, rev=False, force_float=False):
        o = _scal(o)
        ob = o.a if isinstance(o, Mat) else o
        fl = force_float or self.a.dtype.kind == "f" or (isinstance(ob, np.ndarray) and ob.dtype.kind == "f") or \
            isinstance(ob, (np.floating, float))
        if fl:
            A = self.a.astype(np.float32)
            B = ob.astype(np.float32) if isinstance(ob, np.ndarray) else np.float32(ob)
        else:
            A = self.a
            B = ob
        r = fn(B, A) if rev else fn(A, B)
        if isinstance(r, np.ndarray) and r.dtype.kind == "f":
            r = r.astype(np.float32)
        return Mat._wrap(np.asarray(r))

    def __add__(self, o): return self._bin(o, np.add)
    def __radd__(self, o): return self._bin(o, np.add, True)
    def __sub__(self, o): return self._bin(o, np.subtract)
    def __rsub__(self, o): return self._bin(o, np.subtract, True)
    def __mul__(self, o): return self._bin(o, np.multiply)
    def __rmul__(self, o): return self._bin(o, np.multiply, True)
    def __truediv__(self, o): return self._bin(o, np.divide, force_float=True)
    def __rtruediv__(self, o): return self._bin(o, np.divide, True, force_float=True)
    def __floordiv__(self, o): return self._bin(o, np.floor_divide)
    def __rfloordiv__(self, o): return self._bin(o, np.floor_divide, True)
    def __mod__(self, o): return self._bin(o, np.mod)
    def __rmod__(self, o): return self._bin(o, np.mod, True)
    def __pow__(self, o): return self._bin(o, np.power)
    def __neg__(self): return Mat._wrap(-self.a)
    def __abs__(self): return Mat._wrap(np.abs(self.a))
    def __lt__(self, o): return self._bin(o, np.less)
    def __le__(self, o): return self._bin(o, np.less_equal)
    def __gt__(self, o): return self._bin(o, np.greater)
    def __ge__(self, o): return self._bin(o, np.greater_equal)
    def __eq__(self, o): return self._bin(o, np.equal)
    def __ne__(self, o): return self._bin(o, np.not_equal)
    __hash__ = None

    def __matmul__(self, o):
        o = _val(o)
        A = self.a.astype(np.float32)
        B = o.a.astype(np.float32)
        if B.ndim == 1:
            r = np.zeros(A.shape[0], np.float32)
            for i in range(A.shape[0]):
                s = np.float32(0)
                for k in range(A.shape[1]):
                    s = np.float32(s + np.float32(A[i, k] * B[k]))
                r[i] = s
            return Mat._wrap(r)
        r = np.zeros((A.shape[0], B.shape[1]), np.float32)
        for i in range(A.shape[0]):
            for j in range(B.shape[1]):
                s = np.float32(0)
                for k in range(A.shape[1]):
                    s = np.float32(s + np.float32(A[i, k] * B[k, j]))
                r[i, j] = s
        return Mat._wrap(r)

    # -- Taichi methods
    def cast(self, dt):
        if _is_float_dt(dt):
            return Mat._wrap(self.a.astype(np.float32))
        return Mat._wrap(np.trunc(self.a).astype(np.int64))

    def dot(self, o):
        o = _val(o)
        r = self * o
        s = r.a.dtype.type(0)
        for e in r.a:
            s = s + e
            if r.a.dtype.kind == "f":
                s = np.float32(s)
        return s

    def outer_product(self, o):
        a = self.a.astype(np.float32)
        b = _val(o).a.astype(np.float32)
        return Mat._wrap(np.array([[np.float32(x * y) for y in b] for x in a], np.float32))

    def transpose(self):
        return Mat._wrap(self.a.T.copy())

    def determinant(self):
        a = self.a.astype(np.float32)
        if a.shape == (2, 2):
            return np.float32(np.float32(a[0, 0] * a[1, 1]) - np.float32(a[0, 1] * a[1, 0]))
        c0 = np.float32(np.float32(a[1, 1] * a[2, 2]) - np.float32(a[1, 2] * a[2, 1]))
        c1 = np.float32(np.float32(a[1, 0] * a[2, 2]) - np.float32(a[1, 2] * a[2, 0]))
        c2 = np.float32(np.float32(a[1, 0] * a[2, 1]) - np.float32(a[1, 1] * a[2, 0]))
        return np.float32(np.float32(np.float32(a[0, 0] * c0) - np.float32(a[0, 1] * c1)) + np.float32(a[0, 2] * c2))

    def max(self):
        return self.a.max()

    def sum(self):
        return self.a.sum()

    def fill(self, v):
        self.a[...] = _val(v)
        return self

    def norm(self):
        return np.float32(np.sqrt(np.sum(self.a.astype(np.float32) ** 2)))

    # -- static constructors
    @staticmethod
    def zero(dt, n, m=None):
        shp = (n,) if m is None else (n, m)
        return Mat._wrap(np.zeros(shp, _np_dt(dt)))

    @staticmethod
    def identity(dt, n):
        return Mat._wrap(np.eye(n, dtype=_np_dt(dt)))

    @staticmethod
    def field(n, m, dtype=None, shape=None):
        if dtype is None:
            m, dtype = None, m
        return Field(dtype, (n,) if m is None else (n, m), shape)


def _key(k):
    if isinstance(k, Mat):
        return tuple(int(e) for e in k.a)
    if isinstance(k, tuple):
        return tuple(_key1(e) for e in k)
    return _key1(k)


def _key1(e):
    e = _val(e)
    if isinstance(e, slice):
        return e
    if isinstance(e, (np.integer, int)):
        return int(e)
    return e


class _VectorNS:
    """``ti.Vector``: constructor plus the static helpers the reference uses."""

    def __call__(self, a, dt=None):
        return Mat(a, dt)

    def zero(self, dt, n):
        return Mat.zero(dt, n)

    def field(self, n, dtype, shape=None):
        return Field(dtype, (n,), shape)


class _MatrixNS:
    def __call__(self, a, dt=None):
        return Mat(np.array([[_val(e) for e in (r.a if isinstance(r, Mat) else r)] for r in a]), dt)

    zero = staticmethod(Mat.zero)
    identity = staticmethod(Mat.identity)

    def field(self, n, m, dtype, shape=None):
        return Field(dtype, (n, m), shape)


Vector = _VectorNS()
Matrix = _MatrixNS()


# ----------------------------------------------------------------------------
class Ref:
    """A scalar field element used as a value or as the target of ti.atomic_*."""
    __slots__ = ("f", "k")
    __array_ufunc__ = None

    def __init__(self, f, k):
        self.f, self.k = f, k

    def get(self):
        v = self.f._load(self.k)
        return int(v) if self.f.dt is np.int32 else v

    def __index__(self): return int(self.get())
    def __int__(self): return int(self.get())
    def __float__(self): return float(self.get())
    def __bool__(self): return bool(self.get())
    def __repr__(self): return "Ref(%r)" % (self.get(),)
    __hash__ = None


def _mk(op):
    def f(self, o):
        return op(self.get(), _scal(o))
    return f


def _mkr(op):
    def f(self, o):
        return op(_scal(o), self.get())
    return f


import operator as _op
for _n, _f in [("add", _op.add), ("sub", _op.sub), ("mul", _op.mul), ("truediv", _op.truediv),
               ("floordiv", _op.floordiv), ("mod", _op.mod), ("pow", _op.pow), ("and", _op.and_),
               ("or", _op.or_), ("xor", _op.xor), ("lshift", _op.lshift), ("rshift", _op.rshift)]:
    setattr(Ref, "__%s__" % _n, _mk(_f))
    setattr(Ref, "__r%s__" % _n, _mkr(_f))
for _n, _f in [("lt", _op.lt), ("le", _op.le), ("gt", _op.gt), ("ge", _op.ge), ("eq", _op.eq), ("ne", _op.ne)]:
    setattr(Ref, "__%s__" % _n, _mk(_f))
Ref.__neg__ = lambda self: -self.get()


class VecView(Mat):
    """Vector/matrix field element; in-place writes go back to the field."""

    def __init__(self, f, k):
        self._f, self._k = f, k
        self.a = f._load(k).copy()

    def __setitem__(self, k, val):
        Mat.__setitem__(self, k, val)
        self._f._store(self._k, self.a.copy())

    def fill(self, v):
        self.a[...] = _val(v)
        self._f._store(self._k, self.a.copy())
        return self


class Field:
    def __init__(self, dtype, elem=(), shape=None):
        self.dt = _np_dt(dtype)
        self.elem = elem
        self.group = None
        self.snode = None
        if shape is not None:
            shape = (shape,) if isinstance(shape, int) else tuple(shape)
            self.dense = np.zeros(shape + elem, self.dt)
        else:
            self.dense = None
            self.store = {}

    def _zero(self):
        return np.zeros(self.elem, self.dt) if self.elem else self.dt(0)

    def _load(self, k):
        if self.dense is not None:
            v = self.dense[k]
            return v if self.elem else self.dt(v)
        return self.store.get(k, self._zero())

    def _store(self, k, v):
        if self.elem:
            v = np.asarray(v).astype(self.dt) if not isinstance(v, Mat) else v.a.astype(self.dt)
        else:
            v = self.dt(_val(v))
        if self.dense is not None:
            self.dense[k] = v
        else:
            self.store[k] = v
            if self.group is not None:
                self.group.activate(k)

    def __getitem__(self, k):
        k = _key(k)
        if not isinstance(k, tuple):
            k = (k,)
        if self.elem:
            return VecView(self, k)
        return Ref(self, k)

    def __setitem__(self, k, v):
        k = _key(k)
        if not isinstance(k, tuple):
            k = (k,)
        self._store(k, v)

    def to_numpy(self):
        return self.dense.copy()

    def from_numpy(self, a):
        self.dense[...] = np.asarray(a).astype(self.dt)

    def parent(self, n=1):
        s = self.snode
        for _ in range(n - 1):
            s = s.parent
        return s

    def _active(self):
        if self.group is not None:
            return sorted(self.group.active)
        return sorted(self.store)


class _Group:
    """Activation set shared by the fields placed under one SNode."""

    def __init__(self):
        self.active = set()
        self.fields = []

    def activate(self, k):
        self.active.add(k)

    def clear(self):
        self.active.clear()
        for f in self.fields:
            f.store.clear()


class SNode:
    def __init__(self, kind, parent=None, shape=None, block=1):
        self.kind, self.parent, self.shape, self.block = kind, parent, shape, block
        self.children = []
        self.group = _Group()
        self.lists = None

    def _child(self, kind, shape=None, block=1):
        c = SNode(kind, self, shape, block)
        self.children.append(c)
        return c

    def pointer(self, axes, shape):
        return self._child("pointer", shape)

    def dense(self, axes, n):
        return self._child("dense", block=n)

    def bitmasked(self, axes, n):
        return self._child("bitmasked", block=n)

    def dynamic(self, axis, n, chunk_size=None):
        c = self._child("dynamic")
        c.lists = {}
        return c

    def place(self, *fields):
        for f in fields:
            f.snode = self
            if self.kind == "dynamic":
                f.dyn = self
            else:
                f.group = self.group
                self.group.fields.append(f)
        return self

    def deactivate_all(self):
        stack = [self]
        while stack:
            s = stack.pop()
            s.group.clear()
            if s.lists is not None:
                s.lists.clear()
            stack.extend(s.children)


root = SNode("root")
ij, ijk = "ij", "ijk"


def axes(*a):
    return a


def field(dtype, shape=None):
    return Field(dtype, (), shape)


# ----------------------------------------------------------------------------
def kernel(fn):
    ann = dict(getattr(fn, "__annotations__", {}))
    names = fn.__code__.co_varnames[:fn.__code__.co_argcount]

    def wrapper(*args):
        args = list(args)
        for i, n in enumerate(names):
            if i < len(args) and ann.get(n) is f32:
                args[i] = np.float32(args[i])
        return fn(*args)

    wrapper.__name__ = fn.__name__
    return wrapper


def func(fn):
    return fn


def data_oriented(cls):
    return cls


def template():
    return None


def static(x, *a):
    return x


def loop_config(**k):
    pass


class ndrange:
    def __init__(self, *rs):
        self.rs = [(0, r) if isinstance(r, int) else tuple(r) for r in rs]

    def __iter__(self):
        return itertools.product(*[range(a, b) for a, b in self.rs])


def grouped(x):
    if isinstance(x, ndrange):
        return [Mat._wrap(np.array(t, np.int64)) for t in x]
    if isinstance(x, Field):
        if getattr(x, "dyn", None) is not None:
            out = []
            for blk in sorted(x.dyn.lists):
                for j in range(len(x.dyn.lists[blk])):
                    out.append(Mat._wrap(np.array(blk + (j,), np.int64)))
            return out
        return [Mat._wrap(np.array(k, np.int64)) for k in x._active()]
    raise TypeError(x)


def atomic_or(ref, v):
    old = ref.get()
    ref.f._store(ref.k, old | _val(v))
    return old


def atomic_add(ref, v):
    old = ref.get()
    ref.f._store(ref.k, old + _val(v))
    return old


def rescale_index(a, b, I):
    return I // 4


def append(dyn, idx, val):
    k = _key(idx)
    if not isinstance(k, tuple):
        k = (k,)
    dyn.lists.setdefault(k, []).append(int(_val(val)))


# dynamic field element read: pid[l][I] with I = (block..., j)
_orig_load = Field._load


def _load_dyn(self, k):
    dyn = getattr(self, "dyn", None)
    if dyn is not None:
        return self.dt(dyn.lists[tuple(k[:-1])][k[-1]])
    return _orig_load(self, k)


Field._load = _load_dyn


def max(*a):
    a = [_val(x) for x in a]
    return builtins.max(a)


def min(*a):
    a = [_val(x) for x in a]
    return builtins.min(a)


def abs(x):
    x = _val(x)
    if isinstance(x, Mat):
        return Mat._wrap(np.abs(x.a))
    return builtins.abs(x)


def svd(F, dt=None):
    A = _val(F).a.astype(np.float64)
    U, S, Vt = np.linalg.svd(A)
    V = Vt.T
    if np.linalg.det(U) < 0:
        U[:, -1] *= -1
        S[-1] *= -1
    if np.linalg.det(V) < 0:
        V[:, -1] *= -1
        S[-1] *= -1
    return (Mat._wrap(U.astype(np.float32)), Mat._wrap(np.diag(S).astype(np.float32)),
            Mat._wrap(V.astype(np.float32)))


def _clamp(x, lo, hi):
    x = _val(x)
    if isinstance(x, Mat):
        return Mat._wrap(np.minimum(np.maximum(x.a, np.float32(lo)), np.float32(hi)).astype(x.a.dtype))
    return builtins.min(builtins.max(x, lo), hi)


math = types.SimpleNamespace(ivec2="ivec2", ivec3="ivec3", vec2="vec2", vec3="vec3", clamp=_clamp)
