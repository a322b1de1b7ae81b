"""A NumPy stand-in for the subset of the NVIDIA Warp API that EMPM's MPM
simulator uses — used ONLY by tests/golden/make_golden.py to run the
reference's own kernel source on the CPU in FP64 and record golden vectors.

Warp (warp-lang 1.8.1) cannot be installed offline. This module restates
the documented semantics of the builtins the reference calls:
  * ``@wp.kernel`` functions run as plain Python, one call per thread index
    (``wp.launch`` loops over ``dim``; ``wp.tid()`` returns the index);
  * ``wp.vec3`` / ``wp.mat33`` are value types; ``mat * mat`` and
    ``mat * vec`` are matrix products; ``wp.mat33(v0, v1, v2)`` places the
    three vectors as COLUMNS (the semantics under which the reference's
    B-spline tables ``w[axis, offset]`` are correct; the partition-of-unity
    known-answer test pins this);
  * ``wp.svd3`` returns U, V proper rotations with the sign of det(A) on the
    last singular value, computed with LAPACK (numpy.linalg.svd);
  * arithmetic is FP64 throughout (Python floats / float64 arrays).
It is test infrastructure, not a Warp implementation.
"""
from __future__ import annotations

import ctypes
import math
import threading
import types as _pytypes

import builtins as _b

import numpy as np

_F = np.float64
_tls = threading.local()


# --------------------------------------------------------------------------
# value types
# --------------------------------------------------------------------------
def _to_float(x):
    return _b.float(x)


class _Vec:
    __array_ufunc__ = None
    _n = 3
    _type_ = ctypes.c_float

    def __init__(self, *args):
        n = self._n
        if len(args) == 0:
            a = np.zeros(n, _F)
        elif len(args) == 1:
            x = args[0]
            if isinstance(x, _Vec):
                a = x.a.copy()
            elif np.ndim(x) == 0:
                a = np.full(n, _b.float(x), _F)
            else:
                a = np.array([_b.float(t) for t in np.asarray(x, dtype=_F).reshape(-1)], _F)
        else:
            a = np.array([_b.float(t) for t in args], _F)
        assert a.shape == (n,), a.shape
        self.a = a

    def _new(self, a):
        o = self.__class__.__new__(self.__class__)
        o.a = a
        return o

    def __add__(self, o): return self._new(self.a + o.a)
    def __sub__(self, o): return self._new(self.a - o.a)
    def __neg__(self): return self._new(-self.a)
    def __mul__(self, s):
        if isinstance(s, (_Vec, _Mat)):
            raise TypeError("vec * vec/mat is not a Warp operation")
        return self._new(self.a * _b.float(s))
    def __rmul__(self, s): return self._new(_b.float(s) * self.a)
    def __truediv__(self, s): return self._new(self.a / _b.float(s))
    def __getitem__(self, i): return _b.float(self.a[i])
    def __setitem__(self, i, val): self.a[i] = _b.float(val)
    def __len__(self): return self._n
    def __iter__(self): return iter([_b.float(t) for t in self.a])
    def __repr__(self): return f"{self.__class__.__name__}{tuple(self.a)}"


class vec3(_Vec):
    _n = 3
    _shape_ = (3,)


class vec2(_Vec):
    _n = 2
    _shape_ = (2,)


class _Mat:
    __array_ufunc__ = None
    _type_ = ctypes.c_float
    _shape_ = (3, 3)

    def __init__(self, *args):
        if len(args) == 0:
            a = np.zeros((3, 3), _F)
        elif len(args) == 9:
            a = np.array([_b.float(t) for t in args], _F).reshape(3, 3)
        elif len(args) == 3 and all(isinstance(t, _Vec) for t in args):
            a = np.stack([t.a for t in args], axis=1)   # vectors are columns
        elif len(args) == 1:
            x = args[0]
            if isinstance(x, _Mat):
                a = x.a.copy()
            elif np.ndim(x) == 0:
                a = np.full((3, 3), _b.float(x), _F)
            else:
                a = np.asarray(x, _F).reshape(3, 3).copy()
        else:
            raise TypeError(f"unsupported mat33 constructor args: {args}")
        self.a = a

    def _new(self, a):
        o = _Mat.__new__(mat33)
        o.a = a
        return o

    def __add__(self, o): return self._new(self.a + o.a)
    def __sub__(self, o): return self._new(self.a - o.a)
    def __neg__(self): return self._new(-self.a)
    def __mul__(self, o):
        if isinstance(o, _Mat):
            return self._new(self.a @ o.a)
        if isinstance(o, _Vec):
            return vec3(self.a @ o.a)
        return self._new(self.a * _b.float(o))
    def __rmul__(self, s): return self._new(_b.float(s) * self.a)
    def __truediv__(self, s): return self._new(self.a / _b.float(s))
    def __getitem__(self, ij):
        if isinstance(ij, tuple):
            return _b.float(self.a[ij])
        return vec3(self.a[ij])
    def __setitem__(self, ij, val):
        if isinstance(ij, tuple):
            self.a[ij] = _b.float(val)
        else:
            self.a[ij] = val.a
    def __repr__(self): return f"mat33({self.a.tolist()})"


class mat33(_Mat):
    pass


class quat(_Vec):
    _n = 4
    _shape_ = (4,)


float32 = _b.float
int32 = _b.int
float64 = _b.float

# --------------------------------------------------------------------------
# arrays
# --------------------------------------------------------------------------
def _dtype_shape(dtype):
    if dtype in (vec3,):
        return (3,)
    if dtype in (vec2,):
        return (2,)
    if dtype in (mat33,):
        return (3, 3)
    if dtype is quat:
        return (4,)
    return ()


def _np_dtype(dtype):
    return np.int32 if dtype in (_b.int, bool) else _F


class array:
    """Runtime array (data given) or a type annotation (no data)."""

    def __init__(self, data=None, dtype=float, shape=None, ndim=None, device=None, requires_grad=False,
                 grad=None, ptr=None, strides=None, copy=None, owner=None, **kw):
        self.dtype = dtype
        self.ndim = ndim
        self.device = device
        self.requires_grad = requires_grad
        self.grad = grad
        if ptr is not None:
            raise NotImplementedError("raw-pointer arrays are not supported by the shim")
        if data is None:
            self.data = None
            self.shape = shape
            return
        self.data = data
        ds = _dtype_shape(dtype)
        self.shape = tuple(data.shape[: data.ndim - len(ds)]) if ds else tuple(data.shape)

    def _wrap(self, v):
        if self.dtype is vec3:
            return vec3(v)
        if self.dtype is vec2:
            return vec2(v)
        if self.dtype is mat33:
            return mat33(v)
        if self.dtype in (_b.int, bool):
            return _b.int(v)
        return _b.float(v)

    def __getitem__(self, idx):
        return self._wrap(self.data[idx])

    def __setitem__(self, idx, val):
        if isinstance(val, (_Vec, _Mat)):
            self.data[idx] = val.a
        else:
            self.data[idx] = val

    def numpy(self):
        return self.data

    def __len__(self):
        return self.shape[0]


def _alloc(shape, dtype, fill=0):
    if isinstance(shape, (_b.int, np.integer)):
        shape = (shape,)
    shape = tuple(shape)
    return array(np.full(shape + _dtype_shape(dtype), fill, _np_dtype(dtype)), dtype=dtype)


def zeros(shape=None, dtype=float, device=None, requires_grad=False, **kw):
    a = _alloc(shape, dtype, 0)
    a.requires_grad = requires_grad
    return a


def ones(shape=None, dtype=float, device=None, requires_grad=False, **kw):
    return _alloc(shape, dtype, 1)


def zeros_like(a):
    return array(np.zeros_like(a.data), dtype=a.dtype)


def from_numpy(arr, dtype=float, device=None, requires_grad=False, **kw):
    ds = _dtype_shape(dtype)
    data = np.array(arr, dtype=_np_dtype(dtype))
    if ds and data.shape[-len(ds):] != ds:
        data = data.reshape(-1, *ds)
    return array(data, dtype=dtype, requires_grad=requires_grad)


def _torch_to_numpy(t):
    return t.detach().cpu().numpy()


def from_torch(t, dtype=None, requires_grad=None, **kw):
    if dtype is None:
        dtype = _b.int if str(t.dtype).startswith("torch.int") else _b.float
    return from_numpy(_torch_to_numpy(t), dtype=dtype, requires_grad=bool(requires_grad))


def to_torch(a, requires_grad=None):
    import torch

    return torch.from_numpy(a.data)


def clone(a, device=None, requires_grad=False):
    return array(a.data.copy(), dtype=a.dtype, requires_grad=requires_grad)


def copy(dest, src, **kw):
    dest.data[...] = src.data


# --------------------------------------------------------------------------
# kernels
# --------------------------------------------------------------------------
class Kernel:
    def __init__(self, func):
        self.func = func
        self.key = func.__name__


def kernel(f=None, **kw):
    if f is None:
        return lambda g: Kernel(g)
    return Kernel(f)


def func(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


def struct(cls):
    ann = dict(getattr(cls, "__annotations__", {}))

    def _default(t):
        if t in (_b.float,):
            return 0.0
        if t in (_b.int, bool):
            return 0 if t is _b.int else False
        if t in (vec3, vec2, mat33):
            return t()
        return None

    def __init__(self):
        for name, t in ann.items():
            setattr(self, name, _default(t))

    cls.__init__ = __init__
    cls.vars = ann
    return cls


def tid():
    return _tls.tid


def launch(kernel, dim, inputs=(), outputs=(), device=None, **kw):
    f = kernel.func if isinstance(kernel, Kernel) else kernel
    args = list(inputs) + list(outputs)
    if isinstance(dim, (_b.int, np.integer)):
        for i in range(_b.int(dim)):
            _tls.tid = i
            f(*args)
    else:
        for idx in np.ndindex(*[_b.int(d) for d in dim]):
            _tls.tid = tuple(_b.int(t) for t in idx)
            f(*args)


# --------------------------------------------------------------------------
# builtins
# --------------------------------------------------------------------------
float32 = _b.float
int32 = _b.int


def clamp(x, a, b):
    if x < a:
        return a
    if x > b:
        return b
    return x


def max(a, b):  # noqa: A001
    if isinstance(a, _Vec):
        return a._new(np.maximum(a.a, b.a))
    return a if a > b else b


def min(a, b):  # noqa: A001
    if isinstance(a, _Vec):
        return a._new(np.minimum(a.a, b.a))
    return a if a < b else b


def abs(x):  # noqa: A001
    if isinstance(x, _Vec):
        return x._new(np.abs(x.a))
    return _b.abs(x)


def _scalar_np(fn, x):
    with np.errstate(all="ignore"):
        return _b.float(fn(np.float64(x)))


def log(x): return _scalar_np(np.log, x)
def exp(x): return _scalar_np(np.exp, x)
def sqrt(x): return _scalar_np(np.sqrt, x)
def sin(x): return _scalar_np(np.sin, x)
def cos(x): return _scalar_np(np.cos, x)
def acos(x): return _scalar_np(np.arccos, x)


def length(v): return _b.float(np.sqrt(np.dot(v.a, v.a)))
def normalize(v):
    n = length(v)
    return v._new(v.a / n) if n > 0 else v._new(np.zeros_like(v.a))
def dot(a, b): return _b.float(np.dot(a.a, b.a))
def cross(a, b): return vec3(np.cross(a.a, b.a))
def cw_mul(a, b): return a._new(a.a * b.a)
def outer(a, b): return mat33(np.outer(a.a, b.a))
def transpose(m): return mat33(m.a.T.copy())
def determinant(m): return _b.float(np.linalg.det(m.a))
def ddot(a, b): return _b.float(np.sum(a.a * b.a))
def diag(v): return mat33(np.diag(v.a))
def add(a, b): return a + b
def sub(a, b): return a - b
def mul(a, b): return a * b


def svd3(A, U, sig, V):
    u, s, vt = np.linalg.svd(A.a)
    v = vt.T.copy()
    s = s.copy()
    if np.linalg.det(u) < 0:
        u[:, 2] *= -1
        s[2] *= -1
    if np.linalg.det(v) < 0:
        v[:, 2] *= -1
        s[2] *= -1
    U.a[...] = u
    V.a[...] = v
    sig.a[...] = s


def atomic_add(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    arr.data[idx] = arr.data[idx] + (val.a if isinstance(val, (_Vec, _Mat)) else val)


def atomic_sub(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    arr.data[idx] = arr.data[idx] - (val.a if isinstance(val, (_Vec, _Mat)) else val)


class ScopedTimer:
    def __init__(self, name, synchronize=False, print=True, dict=None, **kw):  # noqa: A002
        self.name = name
        self.dict = dict

    def __enter__(self):
        return self

    def __exit__(self, *a):
        if self.dict is not None:
            self.dict.setdefault(self.name, []).append(0.0)


class ScopedDevice:
    def __init__(self, device):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


class Tape:
    def __init__(self):
        self.gradients = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass

    def backward(self, *a, **k):
        raise NotImplementedError("the shim does not differentiate")

    def zero(self):
        pass


def synchronize_device(*a, **k):
    pass


def synchronize(*a, **k):
    pass


def init():
    pass


# submodules referenced as attributes
types = _pytypes.ModuleType("warp.types")
types.array = array
types.float32 = _b.float
types.is_array = lambda a: isinstance(a, array)
context = _pytypes.ModuleType("warp.context")
context.Devicelike = object
codegen = _pytypes.ModuleType("warp.codegen")


class StructInstance:
    pass


codegen.StructInstance = StructInstance


# Warp's scalar casts (wp.int truncates toward zero like a C cast)
def _wp_int(x):
    return _b.int(x)


def _wp_float(x):
    return _b.float(x)


globals()["int"] = _wp_int
globals()["float"] = _wp_float
