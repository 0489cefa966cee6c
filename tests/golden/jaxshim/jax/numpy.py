"""``jax.numpy`` surface used by the reference, on numpy with JAX dtype rules."""
import types

import numpy as _np

from ._core import canon, JArray, config

ndarray = JArray
float32 = _np.float32
float64 = _np.float64
int8 = _np.int8
int32 = _np.int32
int64 = _np.int64
uint32 = _np.uint32
bool_ = _np.bool_
inf = _np.inf
pi = _np.pi
newaxis = None


def _fdt():
    return _np.float64 if config.x64 else _np.float32


def _raw(x):
    if isinstance(x, JArray):
        return _np.asarray(x)
    if isinstance(x, (list, tuple)):
        return type(x)(_raw(v) for v in x)
    return x


def _w(fn):
    def f(*a, **k):
        return canon(fn(*_raw(a), **{kk: _raw(v) for kk, v in k.items()}))
    f.__name__ = getattr(fn, '__name__', 'f')
    return f


def asarray(x, dtype=None):
    if isinstance(x, (list, tuple)):
        vals = [_np.asarray(_raw(v)) for v in x]
        if dtype is None:
            if all(isinstance(v, (int, float, bool)) for v in x):
                if any(isinstance(v, float) for v in x):
                    return canon(_np.asarray(x, dtype=_fdt()))
            x = _np.asarray(vals) if vals else _np.asarray(x)
    return canon(_raw(x), dtype)


array = asarray


def zeros(shape, dtype=None):
    return canon(_np.zeros(shape, dtype=dtype or _fdt()))


def ones(shape, dtype=None):
    return canon(_np.ones(shape, dtype=dtype or _fdt()))


def zeros_like(x, dtype=None):
    return canon(_np.zeros_like(_raw(x), dtype=dtype))


def full(shape, fill_value, dtype=None):
    fv = _raw(fill_value)
    if dtype is None:
        if isinstance(fv, float):
            dtype = _fdt()
        elif isinstance(fv, bool):
            dtype = bool
        elif isinstance(fv, int):
            dtype = _np.int64 if config.x64 else _np.int32
        else:
            dtype = _np.asarray(fv).dtype
    return canon(_np.full(shape, fv, dtype=dtype))


def arange(*args, dtype=None):
    a = _np.arange(*[_raw(v) for v in args])
    if dtype is not None:
        a = a.astype(dtype)
    return canon(a)


def eye(n, dtype=None):
    return canon(_np.eye(n, dtype=dtype or _fdt()))


def linspace(start, stop, num=50, endpoint=True, dtype=None):
    dt = _np.dtype(dtype or _fdt())
    lo = _np.asarray(start, dtype=dt)
    hi = _np.asarray(stop, dtype=dt)
    div = (num - 1) if endpoint else num
    t = (_np.arange(div, dtype=dt) / _np.asarray(div, dtype=dt)).astype(dt)
    out = (lo * (dt.type(1) - t) + hi * t).astype(dt)
    if endpoint:
        out = _np.concatenate([out, hi[None]])
    return canon(out.astype(dt))


def power(a, b):
    return canon(_np.power(_raw(a), _raw(b)))


def size(x):
    return _np.size(_raw(x))


def cumsum(x, axis=None):
    from .lax import associative_scan
    x = canon(_raw(x))
    if axis is None:
        x = x.reshape(-1)
        axis = 0
    return associative_scan(lambda a, b: a + b, x, axis=axis)


def digitize(x, bins, right=False):
    return canon(_np.digitize(_raw(x), _raw(bins), right=right).astype(_np.int64 if config.x64 else _np.int32))


def argmax(x, axis=None):
    return canon(_np.argmax(_raw(x), axis=axis))


def argmin(x, axis=None):
    return canon(_np.argmin(_raw(x), axis=axis))


def einsum(spec, *ops, **k):
    return canon(_np.einsum(spec, *[_raw(o) for o in ops]))


def std(x, axis=None):
    return canon(_np.std(_raw(x), axis=axis))


def dot(a, b):
    return canon(_np.dot(_raw(a), _raw(b)))


def take_along_axis(a, idx, axis):
    return canon(_np.take_along_axis(_raw(a), _raw(idx), axis))


def take(a, idx, axis=None):
    return canon(_np.take(_raw(a), _raw(idx), axis=axis))


def meshgrid(*xs, indexing='xy'):
    return [canon(m) for m in _np.meshgrid(*[_raw(x) for x in xs], indexing=indexing)]


def split(x, n, axis=0):
    return [canon(p) for p in _np.split(_raw(x), n, axis=axis)]


for _name in ['where', 'stack', 'sum', 'concatenate', 'mean', 'exp', 'minimum', 'clip', 'broadcast_to',
              'sqrt', 'max', 'maximum', 'log', 'isnan', 'diff', 'repeat', 'abs', 'min', 'arctan2',
              'tile', 'isfinite', 'ceil', 'allclose', 'log2', 'reshape', 'any', 'all', 'floor',
              'sin', 'cos', 'sign', 'square', 'round', 'prod', 'bitwise_and', 'bitwise_or', 'ravel',
              'expand_dims', 'squeeze', 'transpose', 'cbrt', 'abs', 'negative', 'logical_and',
              'logical_or', 'logical_not', 'nan_to_num', 'outer', 'cos', 'full_like', 'ones_like',
              'count_nonzero', 'searchsorted', 'sort', 'argsort', 'flip', 'cumprod', 'var']:
    if hasattr(_np, _name):
        globals()[_name] = _w(getattr(_np, _name))


def _solve(a, b):
    a = _raw(a)
    b = _raw(b)
    return canon(_np.linalg.solve(a, b).astype(_np.result_type(a.dtype, b.dtype)))


linalg = types.SimpleNamespace(solve=_solve, norm=_w(_np.linalg.norm))


def finfo(dt):
    return _np.finfo(dt)


def iinfo(dt):
    return _np.iinfo(dt)
