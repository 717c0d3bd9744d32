"""A numpy stand-in for the part of JAX the reference's island solver uses,
so that its own code can run in this container (which has no JAX) to make
golden vectors.  Test infrastructure only: ``make_golden_solver.py``
installs it under the module names ``jax``, ``jax.numpy``, ``jax.lax``,
``jax.scipy.signal`` before importing the reference.

Semantics, chosen so that the reference's programs compute what they do
under JAX, in float64:

* every float32 / complex64 dtype maps to float64 / complex128 (the run is
  the reference algorithm in double precision, comparable with the oracle's
  float64 mode);
* arrays are a numpy subclass carrying JAX's functional ``x.at[i].set/add``
  update;
* ``jit`` is the identity, ``vmap`` / ``lax.map`` / ``lax.scan`` are Python
  loops over the mapped axis with pytree (dict / tuple / list) arguments and
  results;
* ``linearize`` returns central differences with a step of 1e-7 of the
  coordinate's scale (``STAND_IN_H_REL`` overrides it), which in float64
  agree with the exact derivative to about 1e-9 or better;
* ``linalg.solve`` takes a batched right-hand side of one dimension less
  than the matrix as a batch of vectors, as JAX does;
* ``lax.dynamic_slice`` clamps its start indices into range, as JAX does.
"""

from __future__ import annotations

import sys
import types

import numpy as np

# ---------------------------------------------------------------- arrays ----


class JArr(np.ndarray):
    """numpy array with JAX's ``.at[...]`` functional update."""

    @property
    def at(self):
        return _At(self)

    def block_until_ready(self):
        return self


class _AtIdx:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def _copy(self):
        return np.array(self.arr, copy=True).view(JArr)

    def set(self, v, **_):
        out = self._copy()
        out[self.idx] = v
        return out

    def add(self, v, **_):
        out = self._copy()
        np.add.at(out, self.idx, v)
        return out

    def multiply(self, v, **_):
        out = self._copy()
        np.multiply.at(out, self.idx, v)
        return out

    def min(self, v, **_):
        out = self._copy()
        np.minimum.at(out, self.idx, v)
        return out

    def max(self, v, **_):
        out = self._copy()
        np.maximum.at(out, self.idx, v)
        return out

    def get(self, **_):
        return _wrap(np.asarray(self.arr)[self.idx])


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self.arr, idx)


_F64 = {np.dtype(np.float32): np.float64, np.dtype(np.float16): np.float64,
        np.dtype(np.complex64): np.complex128}


def _wide(dt):
    if dt is None:
        return None
    d = np.dtype(dt)
    return np.dtype(_F64.get(d, d))


def _wrap(x):
    """Promote float32 results to float64 and view arrays as JArr."""
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    if isinstance(x, np.ndarray):
        if x.dtype in _F64:
            x = x.astype(_F64[x.dtype])
        return x.view(JArr)
    if isinstance(x, (np.floating, np.complexfloating)) and x.dtype in _F64:
        return np.asarray(x, _F64[x.dtype]).view(JArr)
    if isinstance(x, np.generic):
        return np.asarray(x).view(JArr)
    return x


_DROP = ("precision", "preferred_element_type")


def _fn(f):
    def g(*a, **k):
        for key in _DROP:
            k.pop(key, None)
        if "dtype" in k:
            k["dtype"] = _wide(k["dtype"])
        return _wrap(f(*a, **k))
    g.__name__ = getattr(f, "__name__", "fn")
    return g


# ------------------------------------------------------------- jax.numpy ----

jnp = types.ModuleType("jax.numpy")


def _asarray(a, dtype=None, copy=None):
    if isinstance(a, (list, tuple)):
        a = np.array([np.asarray(v) for v in a]) if a and any(
            isinstance(v, np.ndarray) for v in a) else np.asarray(a)
    out = np.array(a, dtype=_wide(dtype), copy=True)
    return _wrap(out)


class _DT:
    """A dtype object that also converts like ``jnp.float32(x)``."""

    def __init__(self, base):
        self.base = np.dtype(base)
        self.dtype = self.base

    def __call__(self, x=0):
        return _wrap(np.asarray(x, self.base))

    def __eq__(self, o):
        try:
            return np.dtype(o) == self.base
        except TypeError:
            return False

    def __hash__(self):
        return hash(self.base)

    def __repr__(self):
        return f"jnp.{self.base.name}"

    @property
    def type(self):
        return self.base.type


# numpy resolves dtype= arguments through np.dtype(obj), which accepts an
# object with a ``dtype`` attribute, as _DT has
for _name, _base in (("float32", np.float64), ("float64", np.float64),
                     ("float16", np.float64), ("bfloat16", np.float64),
                     ("complex64", np.complex128), ("complex128", np.complex128),
                     ("int8", np.int8), ("int16", np.int16), ("int32", np.int32),
                     ("int64", np.int64), ("uint8", np.uint8), ("uint32", np.uint32),
                     ("bool_", np.bool_)):
    setattr(jnp, _name, _DT(_base))
jnp.bool = jnp.bool_
jnp.ndarray = np.ndarray
jnp.pi = np.pi
jnp.inf = np.inf
jnp.nan = np.nan
jnp.newaxis = None
jnp.asarray = _asarray
jnp.array = _asarray


def _result_type(*a):
    return _wide(np.result_type(*[np.asarray(x) if not isinstance(x, _DT) else x.base
                                  for x in a]))


jnp.result_type = _result_type


def _finfo(dt):
    return np.finfo(_wide(dt.base if isinstance(dt, _DT) else dt))


jnp.finfo = _finfo
jnp.iinfo = np.iinfo

for _n in ("where", "zeros", "ones", "full", "zeros_like", "ones_like", "full_like",
           "empty", "arange", "linspace", "sum", "prod", "mean", "max", "min", "maximum",
           "minimum", "abs", "sqrt", "exp", "log", "log10", "log1p", "expm1", "sin", "cos",
           "tan", "arctan2", "arctan", "arcsin", "arccos", "hypot", "square", "sign",
           "floor", "ceil", "round", "rint", "clip", "diag", "diagonal", "eye", "dot",
           "matmul", "einsum", "tensordot", "outer", "stack", "concatenate", "reshape",
           "transpose", "swapaxes", "moveaxis", "expand_dims", "squeeze", "tile",
           "repeat", "broadcast_to", "all", "any", "isfinite", "isnan", "isinf",
           "logical_and", "logical_or", "logical_not", "argmax", "argmin", "argsort",
           "sort", "cumsum", "searchsorted", "take", "take_along_axis", "pad", "real",
           "imag", "conj", "conjugate", "triu", "tril", "meshgrid", "nonzero",
           "count_nonzero", "minimum", "power", "mod", "floor_divide", "trace",
           "nan_to_num", "isclose", "allclose", "array_equal", "flip", "roll", "split",
           "unique", "cos", "cosh", "sinh", "tanh", "fmax", "fmin", "nanmax", "nanmin",
           "nansum", "median", "percentile", "var", "std", "ravel", "atleast_1d",
           "atleast_2d", "bincount", "cross", "sinc", "vstack", "hstack", "column_stack",
           "arctanh", "exp2", "log2", "copysign", "signbit", "heaviside", "interp",
           "equal", "not_equal", "less", "greater", "less_equal", "greater_equal",
           "add", "subtract", "multiply", "divide", "true_divide", "negative",
           "reciprocal", "float_power", "cbrt", "logaddexp", "select", "vdot",
           "inner", "kron", "indices", "diag_indices", "triu_indices", "tril_indices",
           "broadcast_arrays", "shape", "ndim", "size", "isscalar",
           "amax", "amin", "ptp", "average", "histogram", "digitize",
           "argwhere", "flatnonzero", "lexsort", "partition", "trapezoid"):
    if hasattr(np, _n):
        setattr(jnp, _n, _fn(getattr(np, _n)))

jnp.fft = types.ModuleType("jax.numpy.fft")
for _n in ("fft", "ifft", "fft2", "ifft2", "rfft", "irfft", "rfft2", "irfft2", "fftn",
           "ifftn", "rfftn", "irfftn", "fftfreq", "rfftfreq", "fftshift", "ifftshift"):
    setattr(jnp.fft, _n, _fn(getattr(np.fft, _n)))

jnp.linalg = types.ModuleType("jax.numpy.linalg")


def _solve(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if b.ndim == a.ndim - 1:
        return _wrap(np.linalg.solve(a, b[..., None])[..., 0])
    return _wrap(np.linalg.solve(a, b))


jnp.linalg.solve = _solve
for _n in ("inv", "norm", "cholesky", "eigh", "eigvalsh", "det", "slogdet", "qr", "svd",
           "pinv", "lstsq", "cond", "matrix_rank"):
    setattr(jnp.linalg, _n, _fn(getattr(np.linalg, _n)))

# ------------------------------------------------------------------- pytrees --


def _is_leaf(x):
    return not isinstance(x, (dict, tuple, list, types.SimpleNamespace))


def _tree_map(f, *trees):
    t0 = trees[0]
    if isinstance(t0, dict):
        return {k: _tree_map(f, *[t[k] for t in trees]) for k in t0}
    if isinstance(t0, types.SimpleNamespace):
        return types.SimpleNamespace(**{k: _tree_map(f, *[getattr(t, k) for t in trees])
                                        for k in vars(t0)})
    if isinstance(t0, (tuple, list)):
        out = [_tree_map(f, *[t[i] for t in trees]) for i in range(len(t0))]
        return type(t0)(out) if not hasattr(t0, "_fields") else type(t0)(*out)
    return f(*trees)


def _leaves(t, out=None):
    out = [] if out is None else out
    if isinstance(t, dict):
        for k in t:
            _leaves(t[k], out)
    elif isinstance(t, types.SimpleNamespace):
        for k in vars(t):
            _leaves(getattr(t, k), out)
    elif isinstance(t, (tuple, list)):
        for v in t:
            _leaves(v, out)
    elif t is not None:
        out.append(t)
    return out


def _stack_trees(items):
    if not items:
        raise ValueError("empty map")
    return _tree_map(lambda *xs: _wrap(np.stack([np.asarray(x) for x in xs])), *items)


def _slice_tree(arg, axes, i):
    """Index ``arg`` at ``i`` along ``axes`` (a pytree prefix of ints /
    None)."""
    if axes is None:
        return arg
    if isinstance(axes, int):
        return _tree_map(lambda x: _wrap(np.take(np.asarray(x), i, axis=axes)), arg)
    if isinstance(axes, dict):
        return {k: _slice_tree(arg[k], axes.get(k, 0) if k in axes else None, i)
                for k in arg}
    if isinstance(axes, (tuple, list)):
        return type(arg)(_slice_tree(a, ax, i) for a, ax in zip(arg, axes))
    raise TypeError(f"in_axes {axes!r}")


def _axis_size(arg, axes):
    if axes is None:
        return None
    if isinstance(axes, int):
        ls = _leaves(arg)
        return np.asarray(ls[0]).shape[axes] if ls else None
    if isinstance(axes, dict):
        for k, ax in axes.items():
            s = _axis_size(arg[k], ax)
            if s is not None:
                return s
        return None
    for a, ax in zip(arg, axes):
        s = _axis_size(a, ax)
        if s is not None:
            return s
    return None


def vmap(f, in_axes=0, out_axes=0, **_):
    def g(*args):
        axes = in_axes
        if isinstance(axes, int) or axes is None:
            axes = (axes,) * len(args)
        axes = tuple(axes)
        n = _axis_size(args, axes)
        outs = [f(*_slice_tree(args, axes, i)) for i in range(n)]
        res = _stack_trees(outs)
        if out_axes not in (0, None):
            res = _tree_map(lambda x: _wrap(np.moveaxis(np.asarray(x), 0, out_axes)), res)
        return res
    return g


def jit(f=None, **_):
    if f is None:
        return lambda h: h
    return f


H_REL = float(__import__('os').environ.get('STAND_IN_H_REL', '1e-7'))


def linearize(f, x):
    x = np.asarray(x, np.float64)
    y0 = f(_wrap(x))

    def lin(t):
        # central difference along t with a step of H_REL times the
        # coordinates' scale (1 for parameters below 1 in magnitude)
        t = np.asarray(t, np.float64)
        nt = float(np.max(np.abs(t))) if t.size else 0.0
        if nt == 0.0:
            return _tree_map(lambda v: _wrap(np.zeros_like(np.asarray(v))), y0)
        scale = max(1.0, float(np.max(np.abs(x[t != 0]))))
        h = H_REL * scale / nt
        yp = f(_wrap(x + h * t))
        ym = f(_wrap(x - h * t))
        return _tree_map(lambda a, b: _wrap((np.asarray(a) - np.asarray(b)) / (2 * h)),
                         yp, ym)
    return y0, lin


def jacrev(f, argnums=0, **_):
    def g(*args):
        x = np.asarray(args[argnums], np.float64)
        y0 = np.asarray(f(*args))
        J = np.zeros(y0.shape + x.shape)
        flat = x.reshape(-1)
        for j in range(flat.size):
            e = np.zeros_like(flat)
            h = 1e-6 * max(1.0, abs(flat[j]))
            e[j] = h
            ap, am = list(args), list(args)
            ap[argnums] = _wrap((flat + e).reshape(x.shape))
            am[argnums] = _wrap((flat - e).reshape(x.shape))
            d = (np.asarray(f(*ap)) - np.asarray(f(*am))) / (2 * h)
            J.reshape(y0.shape + (-1,))[..., j] = d
        return _wrap(J)
    return g


# ------------------------------------------------------------------ jax.lax --

lax = types.ModuleType("jax.lax")


def scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    n = length if xs is None else np.asarray(_leaves(xs)[0]).shape[0]
    carry = init
    ys = []
    order = range(n - 1, -1, -1) if reverse else range(n)
    for i in order:
        x = None if xs is None else _slice_tree(xs, 0, i)
        carry, y = f(carry, x)
        ys.append(y)
    if reverse:
        ys = ys[::-1]
    if not ys or all(y is None for y in ys):
        return carry, None
    return carry, _stack_trees(ys)


def lax_map(f, xs, batch_size=None):
    n = np.asarray(_leaves(xs)[0]).shape[0]
    return _stack_trees([f(_slice_tree(xs, 0, i)) for i in range(n)])


def dynamic_slice(x, starts, sizes):
    x = np.asarray(x)
    idx = []
    for s, sz, dim in zip(starts, sizes, x.shape):
        s = int(np.clip(int(np.asarray(s)), 0, dim - sz))
        idx.append(slice(s, s + sz))
    return _wrap(x[tuple(idx)])


def dynamic_update_slice(x, upd, starts):
    x = np.array(x, copy=True)
    upd = np.asarray(upd)
    idx = []
    for s, sz, dim in zip(starts, upd.shape, x.shape):
        s = int(np.clip(int(np.asarray(s)), 0, dim - sz))
        idx.append(slice(s, s + sz))
    x[tuple(idx)] = upd
    return _wrap(x)


def cond(pred, tf, ff, *ops):
    return tf(*ops) if bool(np.asarray(pred)) else ff(*ops)


def select(c, a, b):
    return _wrap(np.where(c, a, b))


def while_loop(cf, bf, init):
    v = init
    while bool(np.asarray(cf(v))):
        v = bf(v)
    return v


def fori_loop(lo, hi, bf, init):
    v = init
    for i in range(int(lo), int(hi)):
        v = bf(i, v)
    return v


def stop_gradient(x):
    return x


class Precision:
    HIGHEST = "highest"
    HIGH = "high"
    DEFAULT = "default"


lax.scan = scan
lax.map = lax_map
lax.dynamic_slice = dynamic_slice
lax.dynamic_update_slice = dynamic_update_slice
lax.cond = cond
lax.select = select
lax.while_loop = while_loop
lax.fori_loop = fori_loop
lax.stop_gradient = stop_gradient
lax.Precision = Precision

# --------------------------------------------------------------- jax.scipy --

jscipy = types.ModuleType("jax.scipy")
jsignal = types.ModuleType("jax.scipy.signal")


def _convolve(a, b, mode="full", method="auto", precision=None):
    from scipy import signal
    return _wrap(signal.convolve(np.asarray(a, np.float64), np.asarray(b, np.float64),
                                 mode=mode, method="direct"))


jsignal.convolve = _convolve
jscipy.signal = jsignal

# --------------------------------------------------------------------- jax --

jax = types.ModuleType("jax")
jax.numpy = jnp
jax.lax = lax
jax.scipy = jscipy
jax.vmap = vmap
jax.jit = jit
jax.linearize = linearize
jax.jacrev = jacrev
jax.Array = np.ndarray


class _Config:
    jax_enable_x64 = True

    def update(self, *_a, **_k):
        return None

    def read(self, *_a):
        return True


jax.config = _Config()


class _Device:
    platform = "cpu"
    device_kind = "numpy stand-in"
    id = 0

    def memory_stats(self):
        return None


jax.devices = lambda *a, **k: [_Device()]
jax.local_devices = lambda *a, **k: [_Device()]
jax.device_put = lambda x, *a, **k: _tree_map(
    lambda v: _asarray(v) if isinstance(v, (np.ndarray, np.generic)) else v, x)
jax.device_get = lambda x: x
jax.block_until_ready = lambda x: x
jax.tree_util = types.ModuleType("jax.tree_util")
jax.tree_util.tree_map = _tree_map
jax.tree_util.tree_leaves = _leaves
jax.tree_map = _tree_map


def install():
    """Register the stand-in under the ``jax`` module names."""
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.numpy.fft"] = jnp.fft
    sys.modules["jax.numpy.linalg"] = jnp.linalg
    sys.modules["jax.lax"] = lax
    sys.modules["jax.scipy"] = jscipy
    sys.modules["jax.scipy.signal"] = jsignal
    sys.modules["jax.tree_util"] = jax.tree_util
