"""A minimal pure-Python stand-in for the parts of NVIDIA Warp that Heatflow-MPM's air path uses, so that the
reference's own kernel source can be executed on the CPU at tiny grid sizes to produce golden vectors.

Test infrastructure only: it is imported by ``make_golden.py`` in the development container (where the reference
checkout is readable and warp-lang is not installed) and never by the product or on a GPU box.

Semantics reproduced (Warp kernel language, fp32):
  * every ``float`` kernel parameter and float literal is IEEE binary32; arithmetic on ``numpy.float32`` scalars with
    NumPy >= 2 weak-scalar promotion gives exactly that (no fused multiply-add, round-to-nearest per operation);
  * ``int / int`` inside a kernel is C integer division (``WInt`` below), ``%`` is C remainder (operands are >= 0);
  * ``wp.tid()`` enumerates the launch dimensions in row-major order; ``wp.atomic_add`` adds sequentially in that
    order (a deterministic stand-in for the order-free GPU atomics).

``warp.optim.linear.cg`` is third-party (warp-lang >= 1.7, README says 1.17; not vendored in the reference).  Its
published algorithm is restated in ``cg`` below: Jacobi-preconditioned CG whose absolute tolerance is
max(tol * ||b||, atol (defaults to tol), eps^(9/4)), iterations run in pairs, the residual test is applied on the
device every iteration (alpha and beta are forced to 0 once r.r <= atol^2, which freezes x) and on the host every
``check_every`` iterations (which is what the returned iteration count reflects).  The inner products and the
alpha/beta scalars are evaluated in float64 and applied to the float32 vectors after rounding to float32: that is
the reduction precision of the CUDA build, chosen so that the fixtures pin the stencil/stage semantics without
reduction-order noise.
"""
from __future__ import annotations

import math
import sys
import types

import numpy as np

_F = np.float32


# ----------------------------------------------------------------------------------------------------------- scalars
class WInt(int):
    """Kernel-side integer: ``/`` is C integer division, and every arithmetic result stays a WInt."""

    def _w(self, v):
        return WInt(v)

    def __truediv__(self, o):
        a, b = int(self), int(o)
        q = abs(a) // abs(b)
        return WInt(q if (a >= 0) == (b >= 0) else -q)

    def __rtruediv__(self, o):
        return WInt(o).__truediv__(self)

    def __floordiv__(self, o):
        return self.__truediv__(o)

    def __mod__(self, o):
        a, b = int(self), int(o)
        return WInt(a - b * int(WInt(a).__truediv__(b)))

    def __add__(self, o):
        return WInt(int(self) + int(o)) if isinstance(o, int) else int(self) + o

    __radd__ = __add__

    def __sub__(self, o):
        return WInt(int(self) - int(o)) if isinstance(o, int) else int(self) - o

    def __rsub__(self, o):
        return WInt(int(o) - int(self)) if isinstance(o, int) else o - int(self)

    def __mul__(self, o):
        return WInt(int(self) * int(o)) if isinstance(o, int) else int(self) * o

    __rmul__ = __mul__

    def __neg__(self):
        return WInt(-int(self))


def _f32(x):
    return _F(x)


class Vec:
    """Small fixed-length vector (wp.vec3 / wp.vec3i) with componentwise arithmetic."""

    __array_ufunc__ = None  # make numpy scalars defer to our reflected operators

    def __init__(self, *c, kind="f"):
        if len(c) == 1 and isinstance(c[0], (list, tuple, np.ndarray)):
            c = tuple(c[0])
        if len(c) == 1:
            c = (c[0],) * 3
        self.kind = kind
        self.c = [(_F(v) if kind == "f" else int(v)) for v in c]

    def __getitem__(self, i):
        return self.c[i]

    def __setitem__(self, i, v):
        self.c[i] = _F(v) if self.kind == "f" else int(v)

    def __len__(self):
        return len(self.c)

    def _bin(self, o, f):
        if isinstance(o, Vec):
            return Vec(*[f(a, b) for a, b in zip(self.c, o.c)], kind=self.kind)
        return Vec(*[f(a, o) for a in self.c], kind=self.kind)

    def __add__(self, o):
        return self._bin(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._bin(o, lambda a, b: a - b)

    def __mul__(self, o):
        return self._bin(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return Vec(*[o * a for a in self.c], kind=self.kind)

    def __truediv__(self, o):
        return self._bin(o, lambda a, b: a / b)

    def __neg__(self):
        return Vec(*[-a for a in self.c], kind=self.kind)

    def __repr__(self):
        return f"Vec{tuple(self.c)}"


def vec3(*c):
    return Vec(*(c if c else (0.0,)), kind="f")


def vec3i(*c):
    return Vec(*c, kind="i")


# ----------------------------------------------------------------------------------------------------------- arrays
class Array:
    """Host-resident stand-in for wp.array: wraps a numpy array; vec3 arrays are (N, 3) float32."""

    def __init__(self, data, dtype):
        self.dtype = dtype
        self.np = data

    @property
    def shape(self):
        return self.np.shape[:1] if self.dtype is vec3 else self.np.shape

    def numpy(self):
        return self.np

    def reshape(self, shape):
        return Array(self.np.reshape(shape), self.dtype)

    def zero_(self):
        self.np[...] = 0

    def fill_(self, v):
        self.np[...] = v

    def kernel_view(self):
        return _Vec3View(self.np) if self.dtype is vec3 else self.np


class _Vec3View:
    def __init__(self, a):
        self.a = a

    def __getitem__(self, t):
        return Vec(*self.a[int(t)], kind="f")

    def __setitem__(self, t, v):
        self.a[int(t)] = np.array([float(x) for x in v.c], np.float32)


def _np_dtype(dtype):
    if dtype is int or dtype == "int32":
        return np.int32
    if dtype is vec3:
        return np.float32
    return np.float32


def zeros(shape, dtype=float, device=None, **kw):
    if isinstance(shape, int):
        shape = (shape,)
    shape = tuple(shape)
    if dtype is vec3:
        shape = shape + (3,)
    return Array(np.zeros(shape, _np_dtype(dtype)), dtype)


def empty(n=None, dtype=float, device=None, shape=None, **kw):
    return zeros(shape if shape is not None else n, dtype)


def full(shape, value, dtype=float, device=None, **kw):
    a = zeros(shape, dtype)
    a.np[...] = value
    return a


def array(data, dtype=float, device=None, **kw):
    a = np.array(data, dtype=_np_dtype(dtype), copy=True)
    return Array(a, dtype)


def clone(a, **kw):
    return Array(a.np.copy(), a.dtype)


# ---------------------------------------------------------------------------------------------------------- kernels
_TID = [None]


def tid():
    return _TID[0]


class Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.__name__ = fn.__name__
        ann = dict(fn.__annotations__)
        self.params = [p for p in fn.__code__.co_varnames[: fn.__code__.co_argcount]]
        self.float_params = {p for p in self.params if str(ann.get(p, "")).strip() == "float"}


def kernel(fn=None, **kw):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def func(fn):
    return fn


def launch(k, dim, inputs, device=None, **kw):
    args = []
    for name, v in zip(k.params, inputs):
        if isinstance(v, Array):
            args.append(v.kernel_view())
        elif name in k.float_params:
            args.append(_F(v))
        else:
            args.append(v)
    if isinstance(dim, int):
        for t in range(dim):
            _TID[0] = WInt(t)
            k.fn(*args)
    else:
        dim = tuple(int(d) for d in dim)
        for idx in np.ndindex(*dim):
            _TID[0] = tuple(WInt(i) for i in idx)
            k.fn(*args)
    _TID[0] = None


def floor(x):
    return np.floor(x)


def min(a, b):  # noqa: A001 - mirrors wp.min
    return a if a < b else b


def max(a, b):  # noqa: A001 - mirrors wp.max
    return a if a > b else b


def clamp(x, lo, hi):
    r = min(max(x, lo), hi)
    return _F(r) if isinstance(x, (np.floating, float)) else r


def atomic_add(a, i, j, k, v):
    a[i, j, k] = a[i, j, k] + _F(v)


def where(c, a, b):
    return a if c else b


def array3d(*a, **k):
    return None


def _array_annot(*a, **k):
    return None


class ScopedDevice:
    def __init__(self, *a, **k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class _Config:
    log_level = 0


config = _Config()
LOG_WARNING = 0
float32 = float
int32 = int
uint64 = int


def init():
    pass


# --------------------------------------------------------------------------------------- warp.optim.linear restated
class LinearOperator:
    def __init__(self, shape, dtype=None, device=None, matvec=None):
        self.shape, self.dtype, self.device, self.matvec = shape, dtype, device, matvec


def aslinearoperator(diag):
    def mv(x, y, z, alpha, beta):
        zn = (_F(alpha) * diag.np) * x.np
        if beta != 0.0:
            zn = zn + _F(beta) * y.np
        z.np[...] = zn

    n = diag.np.shape[0]
    return LinearOperator((n, n), float, None, mv)


def _dot(a, b):
    return float(np.dot(a.np.astype(np.float64), b.np.astype(np.float64)))


CG_LOG = []   # (iterations performed on the device, reported iterations, ||r||, atol) per solve


def cg(A, b, x, tol=None, atol=None, maxiter=0, M=None, callback=None, check_every=10, use_cuda_graph=True):
    n = b.np.shape[0]
    if maxiter == 0:
        maxiter = A.shape[0]
    eps = 1.0e-8
    if tol is None and atol is None:
        tol = atol = eps ** 0.75
    elif tol is None:
        tol = atol
    elif atol is None:
        atol = tol
    bb = _dot(b, b)
    atol = max(max(tol * math.sqrt(bb), atol), eps ** 2.25)
    atol_sq = atol * atol
    r = zeros(n)
    A.matvec(x, b, r, -1.0, 1.0)
    rr = _dot(r, r)
    z = zeros(n)
    M.matvec(r, z, z, 1.0, 0.0)
    rz = _dot(r, z)
    Ap = zeros(n)
    p = clone(z)
    if rr <= atol_sq:
        CG_LOG.append((0, 0, math.sqrt(rr), atol))
        return 0, math.sqrt(rr), atol
    cur, done_at = 0, None
    check_every = check_every if check_every >= 2 else 2
    while True:
        for _ in range(2):
            A.matvec(p, Ap, Ap, 1.0, 0.0)
            pAp = _dot(p, Ap)
            alpha = _F(rz / pAp) if rr > atol_sq else _F(0.0)
            x.np[...] = x.np + alpha * p.np
            r.np[...] = r.np - alpha * Ap.np
            live = rr > atol_sq
            rr = _dot(r, r)
            M.matvec(r, z, z, 1.0, 0.0)
            rz_new = _dot(r, z)
            beta = _F(rz_new / rz) if rr > atol_sq else _F(0.0)
            p.np[...] = z.np + beta * p.np
            rz = rz_new
            if live:
                done_at = (done_at or 0) + 1
        cur += 2
        if cur >= maxiter:
            break
        if cur % check_every < 2 and rr <= atol_sq:
            break
    CG_LOG.append((done_at or 0, cur, math.sqrt(rr), atol))
    return cur, math.sqrt(rr), atol


# ------------------------------------------------------------------------------------------------------ installation
def install():
    """Register ``warp``, ``warp.optim`` and ``warp.optim.linear`` (and a ``trimesh`` placeholder) in sys.modules."""
    wp = types.ModuleType("warp")
    me = sys.modules[__name__]
    for name in ("kernel", "func", "launch", "tid", "floor", "min", "max", "clamp", "atomic_add", "where", "vec3", "vec3i",
                 "zeros", "empty", "full", "array", "clone", "ScopedDevice", "config", "LOG_WARNING", "init", "float32",
                 "int32", "uint64"):
        setattr(wp, name, getattr(me, name))
    wp.array3d = array3d
    _arr = array

    class _ArrayFactory:
        def __call__(self, *a, **k):
            if "dtype" in k and not a:
                return None        # used as a type annotation: wp.array(dtype=float)
            return _arr(*a, **k)

    wp.array = _ArrayFactory()
    optim = types.ModuleType("warp.optim")
    linear = types.ModuleType("warp.optim.linear")
    linear.cg, linear.LinearOperator, linear.aslinearoperator = cg, LinearOperator, aslinearoperator
    optim.linear = linear
    wp.optim = optim
    sys.modules["warp"], sys.modules["warp.optim"], sys.modules["warp.optim.linear"] = wp, optim, linear
    if "trimesh" not in sys.modules:
        tm = types.ModuleType("trimesh")
        tm.Trimesh = object
        sys.modules["trimesh"] = tm
    return wp
