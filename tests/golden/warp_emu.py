"""Executor for the subset of the Warp Python DSL (warp-lang 1.12.1) used by
PDE_Module's finite-difference path — TEST INFRASTRUCTURE ONLY.

warp-lang is a dependency of the reference (pinned 1.12.1 in its uv.lock) that is
not installed in this container and cannot be.  tests/golden/make_golden.py
installs this module as ``warp`` so that the reference's own kernel and module
source (FDM/kernel/*.py, FDM/module/*.py, FDM/boundary/functional_boundary.py,
time_step/forwardEuler.py, stencil/*.py) runs unmodified here, to write the
golden fixtures that pin oracle/fdm.py and the CUDA kernels.  Nothing under
pde_module_b200 or on the GPU box uses it.

Semantics reproduced (Warp's documented kernel semantics):
  * scalars are float32 / int32; every arithmetic operation is rounded to
    float32 on its own (no fused multiply-add), as on Warp's CPU device;
  * vectors and matrices are values: reading an array element, assigning a
    variable and passing an argument to a ``wp.func`` copy them;
  * ``arr[i, j, k][c] = v`` stores component c of an array element (the only
    place the reference writes through an element; done by an AST rewrite);
  * ``wp.launch`` runs the kernel once per thread index.  The kernels on this
    path have no write-after-read hazards between threads, so sequential order
    gives the result of any parallel order;
  * ``wp.empty`` fills float storage with NaN so cells a kernel never writes
    are visible as such;
  * NumPy arrays passed to a launch are wrapped without a copy (Warp's CPU
    behaviour), and ``arr[i]`` of a 2-d array is a view of row i;
  * kernel ``assert`` statements are not executed (Warp's default "release"
    mode compiles them out).
Kernel bodies are compiled from their source (``inspect.getsource``) with the
closure variables of the reference's kernel factories bound at first launch,
the same information Warp's own code generator resolves.
"""
from __future__ import annotations

import ast
import inspect
import sys
import textwrap
import types as _pytypes
from typing import Any

import numpy as np

# ------------------------------------------------------------------ scalars --
float32 = np.float32
float64 = np.float64
float16 = np.float16
int32 = np.int32
int64 = np.int64
int8 = np.int8
uint8 = np.uint8
uint32 = np.uint32
bool = np.bool_  # noqa: A001  (Warp's wp.bool)


def _np_dtype(dt):
    if dt is int or dt is np.int32:
        return np.int32
    if dt is float or dt is np.float32:
        return np.float32
    if dt in (np.float64, np.int64, np.int8, np.uint8, np.uint32, np.float16, np.bool_):
        return dt
    raise TypeError(f"unsupported scalar type {dt!r}")


def _is_seq(x):
    return isinstance(x, (list, tuple, np.ndarray, _Vec))


# ------------------------------------------------------------ vector types --
class _Vec:
    __array_ufunc__ = None  # numpy scalars defer to our reflected operators
    _length_ = 0
    _np = np.float32
    _wp_scalar_type_ = np.float32

    def __init__(self, *args):
        n = self._length_
        if len(args) == 0:
            d = np.zeros(n, self._np)
        elif len(args) == 1 and _is_seq(args[0]):
            src = args[0].d if isinstance(args[0], _Vec) else list(args[0])
            assert len(src) == n, f"vector of length {n} from {len(src)} values"
            d = np.array(src, dtype=self._np)
        elif len(args) == 1:
            d = np.full(n, args[0], dtype=self._np)
        else:
            assert len(args) == n, f"vector of length {n} from {len(args)} values"
            d = np.array(args, dtype=self._np)
        self.d = d

    @classmethod
    def _wrap(cls, d):
        o = object.__new__(cls)
        o.d = d
        return o

    def _copy(self):
        return self._wrap(self.d.copy())

    def _scal(self, v):
        return v if self._np is np.int32 else self._np(v)

    def __len__(self):
        return self._length_

    def __getitem__(self, i):
        v = self.d[int(i)]
        return int(v) if self._np is np.int32 else v

    def __setitem__(self, i, v):
        self.d[int(i)] = v

    def __iter__(self):
        return (self[i] for i in range(self._length_))

    def __add__(self, o):
        return self._wrap(self.d + o.d)

    def __sub__(self, o):
        return self._wrap(self.d - o.d)

    def __neg__(self):
        return self._wrap(-self.d)

    def __mul__(self, s):
        if isinstance(s, _Vec):
            return self._wrap(self.d * s.d)
        return self._wrap(self.d * self._scal(s))

    __rmul__ = __mul__

    def __truediv__(self, s):
        return self._wrap(self.d / self._scal(s))

    def __repr__(self):
        return f"{type(self).__name__}({self.d.tolist()})"


_vec_cache: dict = {}


def vector(length, dtype=float):
    key = (int(length), _np_dtype(dtype))
    if key not in _vec_cache:
        _vec_cache[key] = type(f"vec{length}_{key[1].__name__}", (_Vec,),
                               {"_length_": key[0], "_np": key[1], "_wp_scalar_type_": key[1],
                                "_shape_": (key[0],)})
    return _vec_cache[key]


vec2i = vector(2, int)
vec3i = vector(3, int)
vec2 = vector(2, float)
vec3 = vector(3, float)


class _Mat:
    __array_ufunc__ = None
    _shape_ = (0, 0)
    _np = np.float32
    _wp_scalar_type_ = np.float32

    def __init__(self, *args):
        n, m = self._shape_
        if len(args) == 0:
            d = np.zeros((n, m), self._np)
        else:
            d = np.array(args[0] if len(args) == 1 else args, dtype=self._np).reshape(n, m)
        self.d = d

    @classmethod
    def _wrap(cls, d):
        o = object.__new__(cls)
        o.d = d
        return o

    def _copy(self):
        return self._wrap(self.d.copy())

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            a, b = idx
            if isinstance(a, slice):
                return vector(self._shape_[0], self._np)._wrap(self.d[:, int(b)].copy())
            return self.d[int(a), int(b)]
        return vector(self._shape_[1], self._np)._wrap(self.d[int(idx)].copy())

    def __setitem__(self, idx, v):
        if isinstance(idx, tuple):
            a, b = idx
            if isinstance(a, slice):
                self.d[:, int(b)] = v.d
            else:
                self.d[int(a), int(b)] = v
        else:
            self.d[int(idx)] = v.d

    def __add__(self, o):
        return self._wrap(self.d + o.d)

    def __sub__(self, o):
        return self._wrap(self.d - o.d)

    def __mul__(self, s):
        if isinstance(s, (_Vec, _Mat)):
            raise NotImplementedError("matrix products are not on the emulated path")
        return self._wrap(self.d * self._np(s))

    __rmul__ = __mul__


_mat_cache: dict = {}


def matrix(shape, dtype=float):
    key = (tuple(int(s) for s in shape), _np_dtype(dtype))
    if key not in _mat_cache:
        _mat_cache[key] = type(f"mat{key[0][0]}{key[0][1]}", (_Mat,),
                               {"_shape_": key[0], "_np": key[1], "_wp_scalar_type_": key[1]})
    return _mat_cache[key]


def type_is_vector(t):
    return isinstance(t, type) and issubclass(t, _Vec)


def type_is_matrix(t):
    return isinstance(t, type) and issubclass(t, _Mat)


def type_is_float(t):
    return t in (float, np.float32, np.float64, np.float16)


is_float = type_is_float


def types_equal(a, b, **kw):
    if a is b:
        return True
    if type_is_vector(a) and type_is_vector(b):
        return a._length_ == b._length_ and a._np is b._np
    if type_is_matrix(a) and type_is_matrix(b):
        return a._shape_ == b._shape_ and a._np is b._np
    return _np_dtype(a) is _np_dtype(b)


def _elem_shape(dt):
    if type_is_vector(dt):
        return (dt._length_,)
    if type_is_matrix(dt):
        return tuple(dt._shape_)
    return ()


def _storage_np(dt):
    return dt._np if (type_is_vector(dt) or type_is_matrix(dt)) else _np_dtype(dt)


# ------------------------------------------------------------------ arrays --
class _Ann:
    """An array type used only as an annotation (wp.array3d(dtype=...), wp.array1d[...])."""

    def __init__(self, kind, dtype=None):
        self.kind, self.dtype = kind, dtype

    def __getitem__(self, dtype):
        return _Ann(self.kind, dtype)

    def __call__(self, dtype=None, **kw):
        return _Ann(self.kind, dtype)

    def __or__(self, other):
        return Any

    __ror__ = __or__


array1d = _Ann("array1d")
array2d = _Ann("array2d")
array3d = _Ann("array3d")
array4d = _Ann("array4d")


class _Array:
    def __init__(self, st: np.ndarray, dtype, shape: tuple):
        self.st, self.dtype, self.shape = st, dtype, tuple(int(s) for s in shape)
        self.device = "cpu"

    @property
    def size(self):
        return int(np.prod(self.shape)) if self.shape else 1

    @property
    def ndim(self):
        return len(self.shape)

    def __len__(self):
        return self.shape[0]

    def _idx(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        idx = tuple(int(i) for i in idx)
        if len(idx) != len(self.shape):
            raise IndexError(f"{len(idx)} indices for a {len(self.shape)}-d array")
        for i, n in zip(idx, self.shape):
            if i < 0 or i >= n:
                raise IndexError(f"index {idx} out of bounds for shape {self.shape}")
        return idx

    def __getitem__(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        if len(idx) < len(self.shape):  # arr[i] of a 2-d array: a view of row i
            sub = tuple(int(i) for i in idx)
            for i, n in zip(sub, self.shape):
                if i < 0 or i >= n:
                    raise IndexError(f"index {sub} out of bounds for shape {self.shape}")
            return _Array(self.st[sub], self.dtype, self.shape[len(sub):])
        idx = self._idx(idx)
        if type_is_vector(self.dtype) or type_is_matrix(self.dtype):
            return self.dtype._wrap(self.st[idx].copy())
        v = self.st[idx]
        return int(v) if self.st.dtype == np.int32 else v

    def __setitem__(self, idx, v):
        idx = self._idx(idx)
        self.st[idx] = v.d if isinstance(v, (_Vec, _Mat)) else v

    def flatten(self):
        es = _elem_shape(self.dtype)
        return _Array(self.st.reshape((self.size,) + es), self.dtype, (self.size,))

    def numpy(self):
        return self.st

    def fill_(self, v):
        self.st[...] = v.d if isinstance(v, (_Vec, _Mat)) else v

    def zero_(self):
        self.st[...] = 0


def _make_array(data=None, dtype=None, shape=None, device=None, copy=True, **kw):
    if data is None and shape is None:
        return _Ann("array", dtype)
    if dtype is None:
        # Warp takes the element type of a NumPy array; the path's integer and
        # boolean arrays (ImmersedBoundary's type table) keep theirs, others are float32
        src_dt = getattr(data, "dtype", None)
        dtype = src_dt.type if src_dt is not None and src_dt.type in (np.int8, np.int32, np.bool_) else np.float32
    es = _elem_shape(dtype)
    npdt = _storage_np(dtype)
    if data is None:
        return zeros(shape, dtype)
    st = np.array(data.st if isinstance(data, _Array) else data, dtype=npdt)
    if shape is None:
        shape = st.shape[:st.ndim - len(es)] if es else st.shape
    shape = (shape,) if isinstance(shape, int) else tuple(shape)
    st = np.ascontiguousarray(st.reshape(tuple(shape) + es))
    return _Array(st, dtype, shape)


class _ArrayType:
    """wp.array: constructor, annotation (wp.array(dtype=...), wp.array | None)."""

    def __call__(self, *a, **k):
        return _make_array(*a, **k)

    def __getitem__(self, dtype):
        return _Ann("array", dtype)

    def __or__(self, other):
        return Any

    __ror__ = __or__


array = _ArrayType()


def zeros(shape, dtype=float, device=None, **kw):
    shape = (shape,) if isinstance(shape, int) else tuple(shape)
    return _Array(np.zeros(shape + _elem_shape(dtype), _storage_np(dtype)), dtype, shape)


def empty(shape, dtype=float, device=None, **kw):
    a = zeros(shape, dtype)
    if np.issubdtype(a.st.dtype, np.floating):
        a.st[...] = np.nan
    return a


def empty_like(a, **kw):
    return empty(a.shape, a.dtype)


def zeros_like(a, **kw):
    return zeros(a.shape, a.dtype)


def copy(dest, src, **kw):
    dest.st[...] = src.st


# ------------------------------------------------------- kernels, launches --
_TID: Any = 0


def tid():
    return _TID


def static(x):
    return x


def where(c, a, b):
    return a if c else b


def sign(x):
    return type(x)(-1) if x < 0 else type(x)(1)


def min(a, b):  # noqa: A001
    return a if a < b else b


def max(a, b):  # noqa: A001
    return a if a > b else b


def outer(a, b):
    """wp.outer: the matrix a b^T, each product rounded on its own."""
    return matrix((a._length_, b._length_), a._np)._wrap(np.outer(a.d, b.d).astype(a._np))


def argmin(v):
    """wp.argmin: index of the first smallest component."""
    return int(np.argmin(v.d))


def _setc(arr, idx, comp, value):
    e = arr[idx]
    e[comp] = value
    arr[idx] = e


class _StoreRewrite(ast.NodeTransformer):
    """`A[i, j, k][c] = v`  ->  `__wp_setc(A, (i, j, k), c, v)`; kernel ``assert``
    statements are dropped, as Warp's default release mode compiles them out."""

    def visit_Assert(self, node):
        return ast.Pass()

    def visit_Assign(self, node):
        self.generic_visit(node)
        if len(node.targets) == 1:
            t = node.targets[0]
            if isinstance(t, ast.Subscript) and isinstance(t.value, ast.Subscript):
                inner = t.value
                call = ast.Call(func=ast.Name("__wp_setc", ast.Load()),
                                args=[inner.value, inner.slice, t.slice, node.value], keywords=[])
                return ast.copy_location(ast.Expr(call), node)
        return node


def _compile(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    fdef.returns = None
    for a in fdef.args.args + fdef.args.kwonlyargs:
        a.annotation = None
    tree = _StoreRewrite().visit(tree)
    ast.increment_lineno(tree, fn.__code__.co_firstlineno - 1)
    ast.fix_missing_locations(tree)
    ns = dict(fn.__globals__)
    if fn.__closure__:
        for name, cell in zip(fn.__code__.co_freevars, fn.__closure__):
            ns[name] = cell.cell_contents
    ns["__wp_setc"] = _setc
    exec(compile(tree, inspect.getsourcefile(fn) or "<warp_emu>", "exec"), ns)
    return ns[fdef.name]


def _by_value(x):
    return x._copy() if isinstance(x, (_Vec, _Mat)) else x


class Function:
    def __init__(self, fn):
        self.fn, self._c = fn, None
        self.__name__ = fn.__name__

    def __call__(self, *args):
        if self._c is None:
            self._c = _compile(self.fn)
        return self._c(*[_by_value(a) for a in args])


class Kernel:
    def __init__(self, fn):
        self.fn, self._c = fn, None
        self.key = fn.__name__
        self.ann = dict(fn.__annotations__)
        self.params = list(inspect.signature(fn).parameters)

    def compiled(self):
        if self._c is None:
            self._c = _compile(self.fn)
        return self._c


def func(fn=None, **kw):
    return Function(fn) if fn is not None else (lambda f: Function(f))


def kernel(fn=None, **kw):
    return Kernel(fn) if fn is not None else (lambda f: Kernel(f))


def _convert(arg, ann):
    if isinstance(arg, np.ndarray) and isinstance(ann, _Ann):
        # a NumPy array passed to a CPU launch: Warp wraps its memory without a
        # copy, so the kernel's stores land in the caller's array
        dt = ann.dtype if ann.dtype is not None else arg.dtype.type
        if dt is bool:
            dt = np.bool_
        es = _elem_shape(dt)
        assert arg.dtype == np.dtype(_storage_np(dt)), f"{arg.dtype} array for a {dt} parameter"
        return _Array(arg, dt, arg.shape[:arg.ndim - len(es)] if es else arg.shape)
    if isinstance(ann, type) and ann in (np.float32, np.float64, np.int32, np.int8, np.uint8):
        return ann(arg)
    if ann is float:
        return np.float32(arg)
    if ann is int:
        return int(arg)
    return arg


def launch(kernel, dim, inputs=(), outputs=(), device=None, **kw):
    global _TID
    fn = kernel.compiled()
    args = list(inputs) + list(outputs)
    args = [_convert(a, kernel.ann.get(p)) for a, p in zip(args, kernel.params)]
    if isinstance(dim, (int, np.integer)):
        it = range(int(dim))
    else:
        dim = tuple(int(d) for d in dim)
        it = range(dim[0]) if len(dim) == 1 else np.ndindex(*dim)
    for t in it:
        _TID = t if isinstance(t, int) else tuple(int(i) for i in t)
        fn(*args)


# ------------------------------------------------------------ odds and ends --
def init():
    pass


def dtype_from_numpy(dt):
    return np.dtype(dt).type


def dtype_to_numpy(dt):
    return _np_dtype(dt)


class _Config:
    mode = "release"
    verify_cuda = False


config = _Config()


class ScopedTimer:
    def __init__(self, *a, **k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class _Anything:
    """Stand-in for Warp names this path never executes (imported by sibling modules)."""

    def __init__(self, name):
        self._name = name

    def __call__(self, *a, **k):
        return _Anything(self._name)

    def __getattr__(self, n):
        return _Anything(f"{self._name}.{n}")

    def __getitem__(self, k):
        return _Anything(self._name)


def install() -> _pytypes.ModuleType:
    """Register this module as ``warp`` and ``warp.types`` in sys.modules."""
    me = sys.modules[__name__]
    wp = _pytypes.ModuleType("warp")
    for k, v in vars(me).items():
        if not k.startswith("__"):
            setattr(wp, k, v)
    tys = _pytypes.ModuleType("warp.types")
    for k in ("vector", "matrix", "type_is_vector", "type_is_matrix", "type_is_float", "is_float",
              "types_equal", "float32", "float64", "int32", "int8", "uint8"):
        setattr(tys, k, getattr(me, k))
    tys.is_array = lambda a: isinstance(a, _Array)
    tys.array = _Array
    wp.types = tys
    wp.Device = _Anything("Device")
    wp.__getattr__ = lambda n: _Anything(n)
    tys.__getattr__ = lambda n: _Anything(n)
    sys.modules["warp"] = wp
    sys.modules["warp.types"] = tys
    return wp
