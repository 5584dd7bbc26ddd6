"""Sequential numpy stand-in for the small part of the taichi 1.7.4 API that the
reference's FSI hot path uses.

TEST INFRASTRUCTURE ONLY.  taichi is not installed in this container, so the
fixture generator (``make_fixtures.py``) registers this module as ``taichi``
before importing the reference's own ``LBMFluid3D``, ``MPMSolid3D``,
``MPMToLBMProjector3D``, ``PenaltyFSICoupler3D``, ``MovingBoundaryFSICoupler3D``,
``LinkAreaMovingBoundaryCoupler3D`` and ``FSIDriver3D`` classes, so that their
unmodified ``@ti.kernel`` bodies execute as plain Python over numpy storage.

Semantics reproduced (the reference's own tests pin the same single-thread
order: ``ti.init(arch=ti.cpu, cpu_max_num_threads=1)``,
tests/test_step115_lbm_open_boundary_and_force_accumulation_contract.py:29):

* every kernel loop runs sequentially in index order;
* fields are typed numpy arrays (f32 / i32 / i8), every store rounds to the
  field's type, and arithmetic on f32 values stays in f32 (an i32 operand
  mixed with an f32 operand is promoted to f32, as taichi does);
* reading a field element yields a value snapshot (taichi value semantics)
  that still remembers its storage slot, so ``ti.atomic_*`` and element
  assignment (``F[i][s] = v``, ``x[p].z = v``) write through;
* assigning to a local variable (``u = v[i]``, ``w = u``) copies the value and
  drops the storage link, as taichi's local variables do: the bodies of
  ``@ti.kernel`` / ``@ti.func`` functions are recompiled with every plain
  ``name = expr`` assignment wrapped in a copy, so that ``w[0] = ...`` later
  changes neither ``u`` nor the field;
* ``ti.svd`` returns rotations U, V with the sign of the smallest singular
  value flipped when det(F) < 0, so ``R = U @ V.T`` is the proper rotation
  (the value the reference uses, mpm/solid.py:233-234).

What is not reproduced: taichi's fast-math instruction selection and FMA
contraction, so fixtures agree with the reference's f32 arithmetic to within
f32 rounding, not bit for bit.
"""

from __future__ import annotations

import ast
import inspect
import itertools
import textwrap

import numpy as np

f32 = np.float32
f64 = np.float64
i32 = np.int32
i64 = np.int64
i8 = np.int8
u8 = np.uint8
cpu = "cpu"
gpu = "gpu"
cuda = "cuda"
x64 = "x64"


def init(*_args, **_kwargs):
    return None


def reset():
    return None


def data_oriented(cls):
    return cls


def _ti_local(value):
    """The value a taichi local variable holds: a copy without storage link."""
    if isinstance(value, np.ndarray):
        return np.array(value).view(TiArr)
    return value


class _LocalCopies(ast.NodeTransformer):
    def visit_Assign(self, node):
        self.generic_visit(node)
        if all(isinstance(t, ast.Name) for t in node.targets):
            node.value = ast.Call(func=ast.Name(id="_ti_local_copy", ctx=ast.Load()), args=[node.value], keywords=[])
        return node

    def visit_AnnAssign(self, node):
        self.generic_visit(node)
        if isinstance(node.target, ast.Name) and node.value is not None:
            node.value = ast.Call(func=ast.Name(id="_ti_local_copy", ctx=ast.Load()), args=[node.value], keywords=[])
        return node


def _with_local_copies(fn):
    """fn recompiled from its source with local assignments copying (see the
    module docstring); fn itself if its source is not available."""
    try:
        src = textwrap.dedent(inspect.getsource(fn))
        filename = inspect.getsourcefile(fn) or "<taichi_shim>"
        first = inspect.getsourcelines(fn)[1]
    except (OSError, TypeError):
        return fn
    tree = ast.parse(src)
    fdef = tree.body[0]
    if not isinstance(fdef, ast.FunctionDef) or fn.__code__.co_freevars:
        return fn
    fdef.decorator_list = []
    _LocalCopies().visit(tree)
    ast.fix_missing_locations(tree)
    ast.increment_lineno(tree, first - 1)
    glb = fn.__globals__
    glb.setdefault("_ti_local_copy", _ti_local)
    scope = {}
    exec(compile(tree, filename, "exec"), glb, scope)
    new = scope[fdef.name]
    new.__defaults__ = fn.__defaults__
    new.__kwdefaults__ = fn.__kwdefaults__
    new.__qualname__ = fn.__qualname__
    return new


def kernel(fn):
    return _with_local_copies(fn)


def func(fn):
    return _with_local_copies(fn)


def template():
    return None


def static(value, *_rest):
    return value


def _norm_index(idx):
    if idx is None:
        return ()
    if isinstance(idx, np.ndarray):
        return tuple(int(v) for v in np.asarray(idx).reshape(-1))
    if isinstance(idx, tuple):
        out = []
        for v in idx:
            if isinstance(v, np.ndarray):
                out.extend(int(a) for a in np.asarray(v).reshape(-1))
            else:
                out.append(int(v))
        return tuple(out)
    return (int(idx),)


def _is_float(a):
    return np.issubdtype(np.asarray(a).dtype, np.floating)


class TiArr(np.ndarray):
    """A taichi Vector/Matrix/scalar value.  ``_src``/``_idx`` remember the
    field slot the value was read from (write-through target)."""

    def __array_finalize__(self, obj):
        self._src = None
        self._idx = ()

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        args = [np.asarray(a) if isinstance(a, np.ndarray) else a for a in inputs]
        if any(isinstance(a, (np.ndarray, np.generic)) and _is_float(a) for a in args) or any(
            isinstance(a, float) for a in args
        ):
            args = [
                a.astype(np.float32)
                if isinstance(a, (np.ndarray, np.generic)) and np.issubdtype(np.asarray(a).dtype, np.integer)
                else a
                for a in args
            ]
        out = kwargs.get("out")
        if out is not None:
            kwargs["out"] = tuple(np.asarray(o) for o in out)
        result = getattr(ufunc, method)(*args, **kwargs)
        if out is not None:
            # in-place update of a local value: hand back the original objects
            return out[0] if len(out) == 1 else out
        if isinstance(result, np.ndarray):
            if result.ndim == 0:
                return result[()]
            return result.view(TiArr)
        return result

    def __getitem__(self, key):
        value = np.ndarray.__getitem__(np.asarray(self), key)
        if self._src is not None and np.ndim(value) == 0:
            ref = np.array(value).view(TiArr)
            ref._src = self._src
            ref._idx = self._idx + _norm_index(key)
            return ref
        if isinstance(value, np.ndarray):
            return value.view(TiArr)
        return value

    def __setitem__(self, key, value):
        np.ndarray.__setitem__(np.asarray(self), key, np.asarray(value))
        if self._src is not None:
            self._src[self._idx + _norm_index(key)] = np.asarray(value)

    def _get(self, i):
        return self[i]

    def _set(self, i, v):
        self[i] = v

    x = property(lambda self: self._get(0), lambda self, v: self._set(0, v))
    y = property(lambda self: self._get(1), lambda self, v: self._set(1, v))
    z = property(lambda self: self._get(2), lambda self, v: self._set(2, v))

    def dot(self, other):
        a = np.asarray(self)
        b = np.asarray(other)
        if _is_float(a) or _is_float(b):
            a = a.astype(np.float32)
            b = b.astype(np.float32)
        return np.dot(a, b)

    def norm(self):
        a = np.asarray(self).astype(np.float32)
        return np.sqrt(np.sum(a * a))

    def sum(self, *args, **kwargs):
        return np.sum(np.asarray(self), *args, **kwargs)

    def outer_product(self, other):
        return np.outer(np.asarray(self), np.asarray(other)).astype(np.float32).view(TiArr)

    def transpose(self, *axes):
        return np.asarray(self).T.copy().view(TiArr)

    def determinant(self):
        return np.float32(np.linalg.det(np.asarray(self, dtype=np.float64)))

    def inverse(self):
        return np.linalg.inv(np.asarray(self, dtype=np.float64)).astype(np.float32).view(TiArr)

    def to_numpy(self):
        return np.array(self)


def _value(arr):
    return np.array(arr).view(TiArr)


def _elem_dtype(values):
    flat = list(np.asarray(values, dtype=object).reshape(-1))
    if all(isinstance(v, (int, np.integer, bool, np.bool_)) for v in flat):
        return np.int32
    return np.float32


class Field:
    def __init__(self, dtype, shape, elem_shape=()):
        if shape is None:
            shape = ()
        if isinstance(shape, int):
            shape = (shape,)
        self.dtype = dtype
        self.shape = tuple(shape)
        self.elem_shape = tuple(elem_shape)
        self.n = elem_shape[0] if elem_shape else None
        self._data = np.zeros(self.shape + self.elem_shape, dtype=dtype)

    def __getitem__(self, idx):
        key = _norm_index(idx)
        ref = np.array(self._data[key]).view(TiArr)
        ref._src = self._data
        ref._idx = key
        return ref

    def __setitem__(self, idx, value):
        self._data[_norm_index(idx)] = np.asarray(value)

    def __iter__(self):
        for idx in np.ndindex(*self.shape):
            yield idx if len(idx) > 1 else idx[0]

    def to_numpy(self):
        return self._data.copy()

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if arr.shape != self._data.shape:
            raise ValueError(f"from_numpy shape {arr.shape} != field shape {self._data.shape}")
        self._data[...] = arr.astype(self.dtype)

    def fill(self, value):
        self._data[...] = value


def field(dtype, shape=None, **_kwargs):
    return Field(dtype, shape)


class _VectorType:
    def __call__(self, values, dt=None):
        dtype = dt if dt is not None else _elem_dtype(values)
        arr = np.array([np.asarray(v).item() if isinstance(v, np.ndarray) else v for v in values], dtype=dtype)
        return _value(arr)

    @staticmethod
    def field(n, dtype, shape=None, **_kwargs):
        return Field(dtype, shape, (n,))

    @staticmethod
    def zero(dtype, n):
        return _value(np.zeros(n, dtype=dtype))


class _MatrixType:
    def __call__(self, values, dt=None):
        arr = np.asarray(values)
        dtype = dt if dt is not None else (np.int32 if np.issubdtype(arr.dtype, np.integer) else np.float32)
        return _value(arr.astype(dtype))

    @staticmethod
    def field(n, m, dtype, shape=None, **_kwargs):
        return Field(dtype, shape, (n, m))

    @staticmethod
    def zero(dtype, n, m):
        return _value(np.zeros((n, m), dtype=dtype))

    @staticmethod
    def identity(dtype, n):
        return _value(np.eye(n, dtype=dtype))


Vector = _VectorType()
Matrix = _MatrixType()


class _NDRange:
    def __init__(self, *args):
        self.ranges = [range(a[0], a[1]) if isinstance(a, tuple) else range(a) for a in args]

    def __iter__(self):
        for t in itertools.product(*self.ranges):
            yield t if len(t) > 1 else t[0]


def ndrange(*args):
    return _NDRange(*args)


def grouped(obj):
    if isinstance(obj, Field):
        it = np.ndindex(*obj.shape)
    else:
        it = (t if isinstance(t, tuple) else (t,) for t in obj)
    for t in it:
        yield _value(np.array(t, dtype=np.int32))


def cast(value, dtype):
    if np.issubdtype(np.dtype(dtype), np.integer):
        arr = np.asarray(value)
        if np.issubdtype(arr.dtype, np.floating):
            arr = np.trunc(arr)
        out = arr.astype(dtype)
    else:
        out = np.asarray(value).astype(dtype)
    if out.ndim == 0:
        return out[()]
    return out.view(TiArr)


def _plain(v):
    return np.asarray(v)


def abs(value):  # noqa: A001 - taichi name
    r = np.abs(_plain(value))
    return r[()] if np.ndim(r) == 0 else r.view(TiArr)


def max(a, b):  # noqa: A001 - taichi name
    r = np.maximum(_plain(a), _plain(b))
    return r[()] if np.ndim(r) == 0 else r.view(TiArr)


def min(a, b):  # noqa: A001 - taichi name
    r = np.minimum(_plain(a), _plain(b))
    return r[()] if np.ndim(r) == 0 else r.view(TiArr)


def _atomic(dst, val, op):
    if not isinstance(dst, TiArr) or dst._src is None:
        raise TypeError("atomic operation target must be a field element")
    src, idx = dst._src, dst._idx
    old = np.array(src[idx])
    src[idx] = op(old, np.asarray(val)).astype(src.dtype)
    return old[()] if old.ndim == 0 else old.view(TiArr)


def atomic_add(dst, val):
    return _atomic(dst, val, lambda a, b: a + b)


def atomic_sub(dst, val):
    return _atomic(dst, val, lambda a, b: a - b)


def atomic_max(dst, val):
    return _atomic(dst, val, np.maximum)


def atomic_min(dst, val):
    return _atomic(dst, val, np.minimum)


def svd(F, dt=None):
    a = np.asarray(F, dtype=np.float64)
    u, s, vt = np.linalg.svd(a)
    v = vt.T.copy()
    if np.linalg.det(u) < 0.0:
        u[:, 2] *= -1.0
        s[2] *= -1.0
    if np.linalg.det(v) < 0.0:
        v[:, 2] *= -1.0
        s[2] *= -1.0
    return (
        _value(u.astype(np.float32)),
        _value(np.diag(s).astype(np.float32)),
        _value(v.astype(np.float32)),
    )
