"""A NumPy stand-in for the subset of the Taichi API that the reference's
mass-spring path uses, so the reference's own kernel source can be executed
here (Taichi is not installed and there is no network) to generate golden
vectors.

Only the fixture generator (make_golden.py) imports this module.  It is not part
of the product and not used at test time: tests read the committed ``.npz``
fixtures.

Semantics restated from Taichi's public documentation for the primitives the
reference calls (all in float64, like the reference's ``default_fp=ti.f64``):

* fields are dense arrays placed by ``ti.root.dense(...).place(...)``; element
  reads of vector fields return views so ``ti.atomic_add(f[i], v)`` and
  ``f[i][d] = s`` write through, as Taichi's field element references do;
* ``Vector.norm(eps) = sqrt(norm_sqr + eps)``, ``normalized(eps) = v / (norm() + eps)``;
* ``ti.ndrange`` iterates the cartesian product of its ranges in row-major order
  (the reference's atomics make its own order irrelevant to the result up to
  rounding);
* ``ti.random()`` draws U[0,1) from a seeded NumPy generator (the reference's
  stream is time-seeded, ``multitask/taichi_env.py:15``);
* ``ti.ad.Tape`` is a no-op context manager: only forward values are produced.
"""
import itertools
import math
import types

import numpy as np

f64 = np.float64
f32 = np.float32
i32 = np.int32
real = f64
gpu = "gpu"
cpu = "cpu"
cuda = "cuda"

i = ("i",)
j = ("j",)
k = ("k",)
ij = ("i", "j")
ijk = ("i", "j", "k")

_rng = np.random.default_rng(0)


def seed(s):
    global _rng
    _rng = np.random.default_rng(s)


def random(dtype=None):
    return float(_rng.random())


def init(*args, **kwargs):
    return None


def template():
    return None


def ext_arr():
    return None


def data_oriented(cls):
    return cls


def kernel(fn):
    return fn


def func(fn):
    return fn


def static(x, *args):
    return x


def ndrange(*args):
    ranges = []
    for a in args:
        if isinstance(a, (tuple, list)):
            ranges.append(range(int(a[0]), int(a[1])))
        else:
            ranges.append(range(int(a)))
    if len(ranges) == 1:
        return iter(ranges[0])
    return itertools.product(*ranges)


def grouped(field):
    return itertools.product(*[range(s) for s in field.shape])


class TiVec(np.ndarray):
    """ndarray with the Taichi Vector methods the reference calls."""

    def norm(self, eps=0.0):
        return math.sqrt(float(np.sum(np.asarray(self) ** 2)) + eps)

    def norm_sqr(self):
        return float(np.sum(np.asarray(self) ** 2))

    def normalized(self, eps=0.0):
        invlen = 1.0 / (self.norm() + eps)
        return invlen * self

    def outer_product(self, other):
        return np.outer(np.asarray(self), np.asarray(other)).view(TiVec)

    def determinant(self):
        return float(np.linalg.det(np.asarray(self)))

    def __call__(self, *idx):
        # old-style component access v(i) / m(i, j)
        return np.asarray(self)[idx if len(idx) > 1 else idx[0]]


def _vec(values):
    return np.array(values, dtype=np.float64).view(TiVec)


class Field:
    def __init__(self, dtype=f64, n=None, m=None, shape=None):
        self.dtype = dtype
        self.n = n
        self.m = m
        self.arr = None
        self.shape = None
        if shape is not None:
            if isinstance(shape, int):
                shape = (shape,)
            self._alloc(tuple(shape))

    def _alloc(self, shape):
        self.shape = shape
        full = shape
        if self.n is not None:
            full = shape + (self.n,) + ((self.m,) if self.m is not None else ())
        arr = np.zeros(full, dtype=np.int32 if self.dtype is i32 else np.float64)
        self.arr = arr.view(TiVec) if self.n is not None else arr

    @staticmethod
    def _key(idx):
        if idx is None:
            return ()
        if isinstance(idx, tuple):
            out = []
            for e in idx:
                if isinstance(e, np.ndarray):
                    out.extend(int(v) for v in np.asarray(e).ravel())
                else:
                    out.append(int(e))
            return tuple(out)
        return idx

    def __iter__(self):
        # struct-for over all indices of the field
        return itertools.product(*[range(s) for s in self.shape])

    @property
    def grad(self):
        if getattr(self, "_grad", None) is None:
            g = Field(self.dtype, n=self.n, m=self.m)
            g._alloc(self.shape)
            self._grad = g
        return self._grad

    def __getitem__(self, idx):
        return self.arr[self._key(idx)]

    def __setitem__(self, idx, val):
        self.arr[self._key(idx)] = val

    def fill(self, v):
        self.arr[...] = v

    def to_numpy(self):
        return np.array(self.arr)

    def from_numpy(self, a):
        self.arr[...] = a


class _VectorNS:
    @staticmethod
    def field(n, dtype=f64, shape=None):
        return Field(dtype, n=n, shape=shape)

    def __call__(self, values):
        return _vec(values)


class _MatrixNS:
    @staticmethod
    def field(n, m, dtype=f64, shape=None):
        return Field(dtype, n=n, m=m, shape=shape)

    @staticmethod
    def zero(dtype, n, m=None):
        if m is None or m == 1:
            return _vec(np.zeros(n))
        return np.zeros((n, m)).view(TiVec)

    @staticmethod
    def diag(dim, val):
        return (np.eye(dim) * val).view(TiVec)

    def __call__(self, values):
        return np.array(values, dtype=np.float64).view(TiVec)


Vector = _VectorNS()
Matrix = _MatrixNS()


def field(dtype=f64, shape=None):
    return Field(dtype, shape=shape)


class SNode:
    def __init__(self, shape=()):
        self.shape = tuple(shape)

    def dense(self, axes, shape):
        if isinstance(shape, int):
            shape = (shape,)
        return SNode(self.shape + tuple(shape))

    def place(self, *fields):
        for f in fields:
            f._alloc(self.shape)
        return self

    def lazy_grad(self):
        return None


root = SNode()


def atomic_add(ref, val):
    old = np.array(ref)
    ref += val
    return old


def exp(x):
    return np.exp(x)


def sin(x):
    return np.sin(x)


def cos(x):
    return np.cos(x)


def sqrt(x):
    return np.sqrt(x)


def atan2(y, x):
    return np.arctan2(y, x)


def abs(x):  # noqa: A001 - mirrors ti.abs
    return np.abs(x)


def min(a, b):  # noqa: A001 - mirrors ti.min
    return np.minimum(a, b)


def max(a, b):  # noqa: A001 - mirrors ti.max
    return np.maximum(a, b)


def cast(x, dtype):
    if dtype is i32:
        return np.asarray(x).astype(np.int64).view(TiVec) if np.ndim(x) else int(x)
    return np.asarray(x).astype(np.float64).view(TiVec) if np.ndim(x) else float(x)


def polar_decompose(A, dt=None):
    """2D polar decomposition in Taichi's closed form: R from
    (A00 + A11, A10 - A01) normalised, S = R^T A."""
    A = np.asarray(A)
    x, y = A[0, 0] + A[1, 1], A[1, 0] - A[0, 1]
    scale = 1.0 / np.sqrt(x * x + y * y)
    c, s = x * scale, y * scale
    r = np.array([[c, -s], [s, c]]).view(TiVec)
    return r, (np.asarray(r).T @ A).view(TiVec)


class _TapeCtx:
    def __init__(self, *args, **kwargs):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def _grad_replaced(fn):
    return fn


def _grad_for(primal):
    def deco(fn):
        return fn
    return deco


ad = types.SimpleNamespace(Tape=_TapeCtx, grad_replaced=_grad_replaced, grad_for=_grad_for)


class GUI:
    def __init__(self, *args, **kwargs):
        pass

    def __getattr__(self, name):
        return lambda *a, **k: None


def rgb_to_hex(c):
    return 0
