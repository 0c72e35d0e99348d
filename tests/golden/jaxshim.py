"""A NumPy stand-in for the subset of ``jax`` that yggdrax's tree-pipeline
modules use, so their own source can run in a container without JAX.

Used only by ``make_golden.py`` to produce golden fixtures from the reference
code.  It reproduces the JAX semantics those modules rely on:

* x64 mode (uint64 / int64 / float64 available; Python scalars are "weak");
* array indexing: negative indices wrap, then out-of-range indices clamp
  (XLA gather clamps start indices);
* ``.at[...]`` scatters: negative indices wrap, out-of-range updates are
  dropped; ``set`` applies updates in order (last writer wins), ``add`` /
  ``max`` / ``min`` accumulate;
* ``jnp.searchsorted`` uses the fixed-step "scan" binary search;
* ``jnp.nextafter`` returns a weak Python float (so ``clip`` keeps float32);
* ``jax.jit`` / ``jax.vmap`` / ``lax`` control flow run eagerly.
"""

from __future__ import annotations

import math
import sys
import types
from functools import partial

import numpy as np


class JArray(np.ndarray):
    """ndarray with JAX index clamping and an ``.at`` property."""

    def __array_finalize__(self, obj):
        pass

    @property
    def at(self):
        return _At(self)

    def __getitem__(self, idx):
        return np.ndarray.__getitem__(self, _jax_index(self, idx))

    def __hash__(self):
        return id(self)


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, JArray):
        return x.view(JArray)
    if isinstance(x, np.generic):
        return np.asarray(x).view(JArray)
    return x


def _is_int_array(i):
    return isinstance(i, np.ndarray) and i.dtype.kind in "iu" and i.dtype != np.bool_


def _norm_clamp(i, n):
    i = np.asarray(i)
    if i.dtype.kind == "u":
        i = i.astype(np.int64)
    i = np.where(i < 0, i + n, i)
    return np.clip(i, 0, max(n - 1, 0)).astype(np.int64)


def _jax_index(arr, idx):
    if isinstance(idx, tuple):
        out = []
        ax = 0
        for it in idx:
            if it is None:
                out.append(it)
                continue
            if it is Ellipsis:
                out.append(it)
                ax = arr.ndim - (len([x for x in idx if x is not None]) - 1 - ax)
                continue
            if _is_int_array(it):
                out.append(_norm_clamp(it, arr.shape[ax]))
            elif isinstance(it, JArray) and it.ndim == 0 and it.dtype.kind in "iu":
                out.append(int(_norm_clamp(it, arr.shape[ax])))
            else:
                out.append(it)
            ax += 1
        return tuple(out)
    if _is_int_array(idx):
        return _norm_clamp(idx, arr.shape[0])
    if isinstance(idx, np.generic) and np.asarray(idx).dtype.kind in "iu":
        return int(_norm_clamp(idx, arr.shape[0]))
    return idx


def _scatter_index(arr, idx):
    """Normalise negatives; return (index tuple, keep mask) for drop mode."""
    if not isinstance(idx, tuple):
        idx = (idx,)
    arrays, keep = [], None
    for ax, it in enumerate(idx):
        if isinstance(it, slice):
            arrays.append(it)
            continue
        it = np.asarray(it)
        if it.dtype == np.bool_:
            arrays.append(it)
            continue
        it = it.astype(np.int64)
        n = arr.shape[ax]
        it = np.where(it < 0, it + n, it)
        ok = (it >= 0) & (it < n)
        keep = ok if keep is None else (keep & ok)
        arrays.append(it)
    return arrays, keep


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self.arr, idx)


class _AtIdx:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def get(self, **kw):
        return _wrap(self.arr[self.idx])

    def _apply(self, values, op):
        out = np.array(self.arr, copy=True)
        idx = self.idx if isinstance(self.idx, tuple) else (self.idx,)
        if any(it is Ellipsis for it in idx) and op == "set" and all(
                it is Ellipsis or isinstance(it, slice) or np.ndim(it) == 0 for it in idx):
            # basic (Ellipsis / slice / scalar) indexing, all in range here
            out[tuple(it if (it is Ellipsis or isinstance(it, slice)) else int(it)
                      for it in idx)] = np.asarray(values)
            return _wrap(out)
        arrays, keep = _scatter_index(out, self.idx)
        if all(isinstance(a, slice) for a in arrays):
            tgt = tuple(arrays)
            if op == "set":
                out[tgt] = values
            elif op == "add":
                out[tgt] = out[tgt] + values
            elif op == "max":
                out[tgt] = np.maximum(out[tgt], values)
            else:
                out[tgt] = np.minimum(out[tgt], values)
            return _wrap(out)
        if any(isinstance(a, slice) for a in arrays):
            if keep is not None and np.ndim(keep) == 0:
                # scalar indices beside slices (x.at[:, 0].set(v))
                if not bool(keep):
                    return _wrap(out)
                tgt = tuple(a if isinstance(a, slice) else int(a) for a in arrays)
                out[tgt] = np.asarray(values)
                return _wrap(out)
            # mixed slice + array: only used with a trailing full slice
            tgt = tuple(a[keep] if (keep is not None and not isinstance(a, slice)) else a
                        for a in arrays)
            vals = np.asarray(values)
            if keep is not None and vals.ndim >= 1 and vals.shape[0] == keep.shape[0]:
                vals = vals[keep]
            out[tgt] = vals
            return _wrap(out)
        shape = np.broadcast_shapes(*[a.shape for a in arrays])
        arrays = [np.broadcast_to(a, shape) for a in arrays]
        keepb = np.ones(shape, bool) if keep is None else np.broadcast_to(keep, shape)
        vals = np.broadcast_to(np.asarray(values), shape + out.shape[len(arrays):])
        sel = tuple(a[keepb] for a in arrays)
        v = vals[keepb]
        if op == "set":
            # in order, last writer wins
            flat = np.ravel_multi_index(sel, out.shape[: len(arrays)]) if len(sel) > 1 else sel[0]
            order = np.arange(flat.shape[0])
            _, last = np.unique(flat[::-1], return_index=True)
            pick = order[::-1][last]
            tgt = tuple(s[pick] for s in sel)
            out[tgt] = v[pick]
        elif op == "add":
            np.add.at(out, sel, v)
        elif op == "max":
            np.maximum.at(out, sel, v)
        else:
            np.minimum.at(out, sel, v)
        return _wrap(out)

    def set(self, values, mode=None, **kw):
        return self._apply(values, "set")

    def add(self, values, mode=None, **kw):
        return self._apply(values, "add")

    def max(self, values, mode=None, **kw):
        return self._apply(values, "max")

    def min(self, values, mode=None, **kw):
        return self._apply(values, "min")


# ---------------------------------------------------------------------------
# jax.numpy


def _mk_jnp():
    jnp = types.ModuleType("jax.numpy")

    def w(f):
        def g(*a, **k):
            return _wrap(f(*a, **k))
        return g

    for name in ["minimum", "maximum", "where", "sign", "sqrt", "rint", "abs", "logical_and",
                 "logical_or", "logical_not", "bitwise_and", "bitwise_or", "bitwise_xor",
                 "left_shift", "right_shift", "floor", "ceil", "exp", "log", "isfinite",
                 "square", "equal", "not_equal", "less", "greater", "invert", "mod",
                 "tile", "repeat", "broadcast_to", "ravel", "reshape", "transpose",
                 "take_along_axis", "flip", "diff", "unique", "isnan", "all", "any",
                 "prod", "floor_divide", "expand_dims", "squeeze", "count_nonzero", "ceil",
                 "argmax", "argmin", "isin", "cumprod", "outer", "meshgrid", "dot",
                 "take", "einsum", "trace"]:
        setattr(jnp, name, w(getattr(np, name)))
    for name in ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64",
                 "float16", "float32", "float64", "bool_", "complex64", "complex128", "iinfo",
                 "finfo", "inf", "nan", "pi", "ndarray", "integer", "floating", "dtype",
                 "newaxis"]:
        setattr(jnp, name, getattr(np, name))

    def asarray(x, dtype=None, copy=None):
        if isinstance(x, (list, tuple)):
            x = [np.asarray(v) for v in x] if any(isinstance(v, np.ndarray) for v in x) else x
        a = np.asarray(x, dtype=dtype)
        return _wrap(np.array(a, copy=True) if a.ndim == 0 else a)
    jnp.asarray = asarray
    jnp.result_type = np.result_type
    jnp.array = lambda x, dtype=None, **k: _wrap(np.array(x, dtype=dtype))
    for name in ["zeros", "ones", "empty", "full", "arange", "zeros_like", "ones_like",
                 "full_like", "empty_like", "linspace", "eye"]:
        setattr(jnp, name, w(getattr(np, name)))

    def sum_(a, axis=None, dtype=None, keepdims=False, **k):
        return _wrap(np.sum(np.asarray(a), axis=axis, dtype=dtype, keepdims=keepdims))
    jnp.sum = sum_

    def _red(f):
        def g(a, axis=None, keepdims=False, initial=None, where=None, **k):
            kw = {}
            if initial is not None:
                kw["initial"] = initial
            if where is not None:
                kw["where"] = where
            return _wrap(f(np.asarray(a), axis=axis, keepdims=keepdims, **kw))
        return g
    jnp.max = _red(np.max)
    jnp.min = _red(np.min)
    jnp.amax = jnp.max
    jnp.amin = jnp.min
    jnp.mean = _red(np.mean)

    def cumsum(a, axis=None, dtype=None):
        a = np.asarray(a)
        return _wrap(np.cumsum(a, axis=0 if axis is None and a.ndim == 1 else axis, dtype=dtype))
    jnp.cumsum = cumsum

    def stack(xs, axis=0):
        return _wrap(np.stack([np.asarray(x) for x in xs], axis=axis))
    jnp.stack = stack

    def concatenate(xs, axis=0):
        return _wrap(np.concatenate([np.asarray(x) for x in xs], axis=axis))
    jnp.concatenate = concatenate

    def argsort(a, axis=-1, kind=None, stable=True, descending=False):
        a = np.asarray(a)
        return _wrap(np.argsort(a, axis=axis, kind="stable").astype(np.int64))
    jnp.argsort = argsort

    def sort(a, axis=-1, **k):
        return _wrap(np.sort(np.asarray(a), axis=axis, kind="stable"))
    jnp.sort = sort

    def lexsort(keys, axis=-1):
        return _wrap(np.lexsort([np.asarray(k) for k in keys], axis=axis).astype(np.int64))
    jnp.lexsort = lexsort

    def clip(a, min=None, max=None, a_min=None, a_max=None):
        lo = min if min is not None else a_min
        hi = max if max is not None else a_max
        x = np.asarray(a)
        if lo is not None:
            x = np.maximum(x, _as_like(lo, x))
        if hi is not None:
            x = np.minimum(x, _as_like(hi, x))
        return _wrap(x)
    jnp.clip = clip

    def nextafter(a, b):
        r = np.nextafter(np.float64(a), np.float64(b))
        return float(r)  # weakly typed like a JAX Python-scalar result
    jnp.nextafter = nextafter

    def bincount(x, weights=None, minlength=0, *, length=None):
        x = np.asarray(x).astype(np.int64)
        L = length if length is not None else max(minlength, int(x.max()) + 1 if x.size else 0)
        keep = (x >= 0) & (x < L)
        if weights is None:
            out = np.zeros(L, np.int64)
            np.add.at(out, x[keep], 1)
        else:
            w_ = np.asarray(weights)
            out = np.zeros(L, w_.dtype if w_.dtype.kind != "b" else np.int64)
            np.add.at(out, x[keep], w_[keep])
        return _wrap(out)
    jnp.bincount = bincount

    def nonzero(a, size=None, fill_value=None):
        idx = np.nonzero(np.asarray(a))
        if size is None:
            return tuple(_wrap(i.astype(np.int64)) for i in idx)
        out = []
        for i in idx:
            o = np.full(size, -1 if fill_value is None else int(fill_value), np.int64)
            m = min(size, i.shape[0])
            o[:m] = i[:m]
            out.append(_wrap(o))
        return tuple(out)
    jnp.nonzero = nonzero

    def searchsorted(a, v, side="left", sorter=None, method="scan"):
        a = np.asarray(a)
        v = np.asarray(v)
        n = a.shape[0]
        levels = int(np.ceil(np.log2(n + 1))) if n > 0 else 0
        lo = np.zeros(v.shape, np.int64)
        hi = np.full(v.shape, n, np.int64)
        for _ in range(levels):
            mid = (lo + hi) // 2
            av = a[np.clip(mid, 0, max(n - 1, 0))]
            go_left = (v <= av) if side == "left" else (v < av)
            lo, hi = np.where(go_left, lo, mid), np.where(go_left, mid, hi)
        return _wrap(hi)
    jnp.searchsorted = searchsorted

    linalg = types.ModuleType("jax.numpy.linalg")

    def norm(x, ord=None, axis=None, keepdims=False):
        x = np.asarray(x)
        return _wrap(np.sqrt(np.sum(x * x, axis=axis, keepdims=keepdims)))
    linalg.norm = norm
    jnp.linalg = linalg
    jnp.result_type = np.result_type
    jnp.shape = np.shape
    jnp.size = np.size
    jnp.ndim = np.ndim
    jnp.issubdtype = np.issubdtype
    return jnp


def _as_like(v, x):
    if isinstance(v, float) and x.dtype.kind == "f":
        return x.dtype.type(v)
    return np.asarray(v)


# ---------------------------------------------------------------------------
# jax / lax / misc modules


def _mk_lax():
    lax = types.ModuleType("jax.lax")

    def fori_loop(lo, hi, body, init):
        v = init
        for i in range(int(lo), int(hi)):
            v = body(i, v)
        return v

    def while_loop(cond, body, init):
        v = init
        while bool(cond(v)):
            v = body(v)
        return v

    def cond(pred, tf, ff, *ops, operand=None):
        args = ops if ops else (operand,)
        return tf(*args) if bool(pred) else ff(*args)

    def associative_scan(fn, x, axis=0):
        if fn is _JNP.maximum or getattr(fn, "__name__", "") == "g":
            return _wrap(np.maximum.accumulate(np.asarray(x), axis=axis))
        raise NotImplementedError

    def clz(x):
        x = np.asarray(x)
        bits = x.dtype.itemsize * 8
        out = np.empty(x.shape, np.int64)
        flat = x.reshape(-1)
        o = out.reshape(-1)
        for k, v in enumerate(flat.tolist()):
            o[k] = bits - int(v).bit_length()
        return _wrap(out.astype(x.dtype))

    def scan(f, init, xs, length=None, unroll=1):
        carry = init
        ys = []
        n = length if length is not None else len(xs)
        for i in range(n):
            carry, y = f(carry, None if xs is None or xs == () else xs[i])
            ys.append(y)
        return carry, ys

    def dynamic_index_in_dim(operand, index, axis=0, keepdims=True):
        # JAX clamps a dynamic index into range
        a = np.asarray(operand)
        i = int(min(max(int(np.asarray(index)), 0), a.shape[axis] - 1))
        out = np.take(a, [i] if keepdims else i, axis=axis)
        return _wrap(out)

    lax.dynamic_index_in_dim = dynamic_index_in_dim
    lax.fori_loop = fori_loop
    lax.while_loop = while_loop
    lax.cond = cond
    lax.associative_scan = associative_scan
    lax.clz = clz
    lax.scan = scan
    lax.stop_gradient = lambda x: x
    lax.div = lambda a, b: _wrap(np.asarray(a) // np.asarray(b))
    return lax


class _Tracer:  # nothing is ever traced here
    pass


def _vmap(f, in_axes=0, out_axes=0, **kw):
    def g(*args):
        n = None
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        for a, ax in zip(args, axes):
            if ax is not None:
                n = np.asarray(a).shape[ax]
                break
        outs = []
        for i in range(n):
            call = []
            for a, ax in zip(args, axes):
                call.append(_wrap(np.take(np.asarray(a), i, axis=ax)) if ax is not None else a)
            outs.append(f(*call))
        if isinstance(outs[0], tuple):
            return tuple(_wrap(np.stack([np.asarray(o[k]) for o in outs]))
                         for k in range(len(outs[0])))
        return _wrap(np.stack([np.asarray(o) for o in outs]))
    return g


def _jit(fun=None, **kw):
    if fun is None:
        return lambda f: f
    return fun


def _segment_sum(data, segment_ids, num_segments=None, **kw):
    d = np.asarray(data)
    ids = np.asarray(segment_ids).astype(np.int64)
    out = np.zeros((num_segments,) + d.shape[1:], d.dtype)
    keep = (ids >= 0) & (ids < num_segments)
    np.add.at(out, ids[keep], d[keep])
    return _wrap(out)


_JNP = None


def install():
    """Register the stand-in modules in sys.modules."""
    global _JNP
    if "jax" in sys.modules and getattr(sys.modules["jax"], "__ygx_shim__", False):
        return
    jax = types.ModuleType("jax")
    jax.__ygx_shim__ = True
    _JNP = _mk_jnp()
    lax = _mk_lax()
    core = types.ModuleType("jax.core")
    core.Tracer = _Tracer
    typing_ = types.ModuleType("jax.typing")
    typing_.ArrayLike = object
    typing_.DTypeLike = object
    tree_util = types.ModuleType("jax.tree_util")
    tree_util.register_pytree_node = lambda *a, **k: None
    tree_util.register_pytree_node_class = lambda c: c
    tree_util.tree_map = lambda f, *t: f(*t)
    ops = types.ModuleType("jax.ops")
    ops.segment_sum = _segment_sum
    config = types.SimpleNamespace(update=lambda *a, **k: None)
    dlpack = types.ModuleType("jax.dlpack")
    debug = types.SimpleNamespace(callback=lambda f, *a, **k: f(*a), print=lambda *a, **k: None)
    jax.numpy = _JNP
    jax.lax = lax
    jax.core = core
    jax.typing = typing_
    jax.tree_util = tree_util
    jax.ops = ops
    jax.config = config
    jax.dlpack = dlpack
    jax.debug = debug
    jax.jit = _jit
    jax.vmap = _vmap
    jax.device_get = lambda x: x
    jax.device_put = lambda x, *a, **k: x
    jax.block_until_ready = lambda x: x
    jax.Array = np.ndarray
    jax.ShapeDtypeStruct = object
    jax.default_backend = lambda: "cpu"
    jax.devices = lambda *a: ["cpu"]
    sys.modules.update({
        "jax": jax, "jax.numpy": _JNP, "jax.numpy.linalg": _JNP.linalg, "jax.lax": lax,
        "jax.core": core, "jax.typing": typing_, "jax.tree_util": tree_util, "jax.ops": ops,
        "jax.dlpack": dlpack,
    })
    # typing decorators used at import time
    jt = types.ModuleType("jaxtyping")
    jt.jaxtyped = lambda *a, **k: (lambda f: f) if not a or not callable(a[0]) else a[0]

    class _AnyType:
        def __class_getitem__(cls, item):
            return object

    for name in ["Array", "Float", "Int", "Bool", "UInt", "Shaped", "Num", "Integer"]:
        setattr(jt, name, _AnyType)
    bt = types.ModuleType("beartype")
    bt.beartype = lambda f=None, **k: f if f is not None else (lambda g: g)
    btt = types.ModuleType("beartype.typing")
    import typing as _typing
    for name in dir(_typing):
        setattr(btt, name, getattr(_typing, name))
    sys.modules.update({"jaxtyping": jt, "beartype": bt, "beartype.typing": btt})


def load_reference(root: str):
    """Import the reference's modules (without its package __init__)."""
    install()
    import importlib

    pkg = types.ModuleType("yggdrax")
    pkg.__path__ = [root]
    sys.modules["yggdrax"] = pkg
    mods = {}
    for name in ["dtypes", "bounds", "morton", "_tree_impl", "octree", "kdtree", "tree",
                 "_geometry_impl", "geometry", "grouped_interactions", "_interactions_impl"]:
        mods[name] = importlib.import_module(f"yggdrax.{name}")
    return mods
