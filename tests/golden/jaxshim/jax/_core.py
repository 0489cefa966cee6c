"""Array type, dtype canonicalisation, pytrees, vmap and finite-difference AD."""
import numpy as np


class _Config:
    def __init__(self):
        self.x64 = False

    def update(self, name, value):
        if name == 'jax_enable_x64':
            self.x64 = bool(value)

    @property
    def jax_enable_x64(self):
        return self.x64


config = _Config()


def _canon_dtype(dt):
    dt = np.dtype(dt)
    if not config.x64:
        if dt == np.float64:
            return np.dtype(np.float32)
        if dt == np.int64:
            return np.dtype(np.int32)
        if dt == np.uint64:
            return np.dtype(np.uint32)
        if dt == np.complex128:
            return np.dtype(np.complex64)
    return dt


def canon(x, dtype=None):
    """numpy value -> JArray with JAX's default dtypes."""
    if isinstance(x, (bool, np.bool_)) and dtype is None:
        a = np.asarray(x, dtype=bool)
    elif isinstance(x, int) and not isinstance(x, bool) and dtype is None:
        a = np.asarray(x, dtype=np.int64 if config.x64 else np.int32)
    elif isinstance(x, float) and dtype is None:
        a = np.asarray(x, dtype=np.float64 if config.x64 else np.float32)
    else:
        a = np.asarray(x) if dtype is None else np.asarray(x, dtype=dtype)
    cd = _canon_dtype(a.dtype) if dtype is None else _canon_dtype(np.dtype(dtype))
    if a.dtype != cd:
        a = a.astype(cd)
    return a.view(JArray)


class _AtIndexer:
    def __init__(self, arr, idx):
        self.arr = arr
        self.idx = idx

    def _index_arrays(self):
        idx = self.idx if isinstance(self.idx, tuple) else (self.idx,)
        return idx

    def set(self, values):
        out = np.array(self.arr, copy=True)
        idx = self._index_arrays()
        vals = np.asarray(values)
        if len(idx) == 1 and isinstance(idx[0], np.ndarray) and idx[0].dtype != bool and idx[0].ndim == 1:
            # duplicate indices: apply in order, last writer wins (XLA CPU scatter)
            ii = np.asarray(idx[0]).astype(np.int64)
            vb = np.broadcast_to(vals, ii.shape + out.shape[1:])
            for k in range(ii.shape[0]):
                out[ii[k]] = vb[k]
        else:
            out[self.idx] = vals
        return canon(out, out.dtype)

    def add(self, values):
        out = np.array(self.arr, copy=True)
        np.add.at(out, self.idx, np.asarray(values))
        return canon(out, out.dtype)

    def get(self):
        return canon(np.asarray(self.arr)[self.idx])


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        if isinstance(idx, JArray):
            idx = np.asarray(idx)
        if isinstance(idx, tuple):
            idx = tuple(np.asarray(i) if isinstance(i, JArray) else i for i in idx)
        return _AtIndexer(self.arr, idx)


class JArray(np.ndarray):
    """numpy array that canonicalises dtypes like JAX and supports ``.at``."""

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        ins = [np.asarray(i) if isinstance(i, JArray) else i for i in inputs]
        if 'out' in kwargs:
            kwargs['out'] = tuple(np.asarray(o) if isinstance(o, JArray) else o for o in kwargs['out'])
        res = getattr(ufunc, method)(*ins, **kwargs)
        if isinstance(res, tuple):
            return tuple(canon(r) for r in res)
        if res is None:
            return None
        return canon(res)

    def __array_function__(self, func, types, args, kwargs):
        def strip(v):
            if isinstance(v, JArray):
                return np.asarray(v)
            if isinstance(v, (list, tuple)):
                return type(v)(strip(x) for x in v)
            return v
        res = func(*strip(args), **{k: strip(v) for k, v in kwargs.items()})
        if isinstance(res, np.ndarray):
            return canon(res)
        if isinstance(res, (np.generic,)):
            return canon(res)
        if isinstance(res, (list, tuple)):
            return type(res)(canon(r) if isinstance(r, np.ndarray) else r for r in res)
        return res

    @property
    def at(self):
        return _At(self)

    def astype(self, dtype, *a, **k):
        return canon(np.asarray(self).astype(dtype), np.dtype(dtype) if dtype is not None else None)

    def __getitem__(self, idx):
        if isinstance(idx, JArray):
            idx = np.asarray(idx)
        elif isinstance(idx, tuple):
            idx = tuple(np.asarray(i) if isinstance(i, JArray) else i for i in idx)
        r = np.asarray(self)[idx]
        return canon(r)

    def __float__(self):
        return float(np.asarray(self))

    def __int__(self):
        return int(np.asarray(self))

    def __bool__(self):
        return bool(np.asarray(self))

    def __hash__(self):
        return id(self)

    def tolist(self):
        return np.asarray(self).tolist()

    def block_until_ready(self):
        return self


# ---------------------------------------------------------------------------
# pytrees
# ---------------------------------------------------------------------------

class _TreeUtil:
    def __init__(self):
        self.registry = {}

    def register_pytree_node_class(self, cls):
        self.registry[cls] = (lambda x: x.tree_flatten(), lambda aux, ch: cls.tree_unflatten(aux, ch))
        return cls

    def register_pytree_node(self, cls, flatten, unflatten):
        self.registry[cls] = (flatten, unflatten)

    def _is_leaf(self, x):
        return not (x is None or isinstance(x, (tuple, list, dict)) or type(x) in self.registry)

    def tree_flatten(self, tree):
        leaves = []

        def rec(x):
            if x is None:
                return ('none',)
            t = type(x)
            if t in self.registry:
                ch, aux = self.registry[t][0](x)
                return ('reg', t, aux, [rec(c) for c in ch])
            if isinstance(x, tuple) and hasattr(x, '_fields'):
                return ('nt', t, [rec(c) for c in x])
            if isinstance(x, tuple):
                return ('tuple', [rec(c) for c in x])
            if isinstance(x, list):
                return ('list', [rec(c) for c in x])
            if isinstance(x, dict):
                keys = sorted(x.keys())
                return ('dict', t, keys, [rec(x[k]) for k in keys])
            leaves.append(x)
            return ('leaf',)
        spec = rec(tree)
        return leaves, spec

    def tree_unflatten(self, spec, leaves):
        it = iter(leaves)

        def rec(s):
            kind = s[0]
            if kind == 'none':
                return None
            if kind == 'leaf':
                return next(it)
            if kind == 'reg':
                _, t, aux, ch = s
                return self.registry[t][1](aux, [rec(c) for c in ch])
            if kind == 'nt':
                return s[1](*[rec(c) for c in s[2]])
            if kind == 'tuple':
                return tuple(rec(c) for c in s[1])
            if kind == 'list':
                return [rec(c) for c in s[1]]
            if kind == 'dict':
                _, t, keys, ch = s
                vals = [rec(c) for c in ch]
                d = dict(zip(keys, vals))
                return t(d) if t is not dict else d
            raise ValueError(kind)
        return rec(spec)

    def tree_map(self, f, tree, *rest):
        leaves, spec = self.tree_flatten(tree)
        others = [self.tree_flatten(r)[0] for r in rest]
        return self.tree_unflatten(spec, [f(*xs) for xs in zip(leaves, *others)])

    def tree_leaves(self, tree):
        return self.tree_flatten(tree)[0]


tree_util = _TreeUtil()


# ---------------------------------------------------------------------------
# vmap
# ---------------------------------------------------------------------------

def _stack_leaves(outs):
    return canon(np.stack([np.asarray(o) for o in outs]))


def vmap(fun, in_axes=0, out_axes=0):
    def wrapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is None:
                continue
            for leaf in tree_util.tree_leaves(a):
                n = np.shape(leaf)[0]
                break
            if n is not None:
                break
        outs = []
        for i in range(n):
            call = []
            for a, ax in zip(args, axes):
                if ax is None:
                    call.append(a)
                else:
                    call.append(tree_util.tree_map(lambda x: canon(np.asarray(x)[i]) if np.ndim(x) else x, a))
            outs.append(fun(*call))
        leaves0, spec = tree_util.tree_flatten(outs[0])
        all_leaves = [tree_util.tree_flatten(o)[0] for o in outs]
        stacked = [_stack_leaves([ls[j] for ls in all_leaves]) for j in range(len(leaves0))]
        return tree_util.tree_unflatten(spec, stacked)
    return wrapped


# ---------------------------------------------------------------------------
# finite-difference forward/reverse derivatives
# ---------------------------------------------------------------------------

def _to64(tree):
    return tree_util.tree_map(
        lambda x: np.asarray(x, dtype=np.float64).view(JArray)
        if np.issubdtype(np.asarray(x).dtype, np.floating) else x, tree)


def _eval64(fun, *args):
    prev = config.x64
    config.x64 = True
    try:
        return fun(*args)
    finally:
        config.x64 = prev


def jvp(fun, primals, tangents):
    (x,), (v,) = primals, tangents
    f0 = fun(x)
    x64 = np.asarray(x, dtype=np.float64)
    v64 = np.asarray(v, dtype=np.float64)
    vmax = np.max(np.abs(v64))
    if vmax == 0 or not np.isfinite(vmax):
        return f0, canon(np.zeros_like(np.asarray(f0)), np.asarray(f0).dtype)
    scale = max(1.0, float(np.max(np.abs(x64))))
    h = 1e-7 * scale / vmax
    fp = np.asarray(_eval64(fun, (x64 + h * v64).view(JArray)), dtype=np.float64)
    fm = np.asarray(_eval64(fun, (x64 - h * v64).view(JArray)), dtype=np.float64)
    t = (fp - fm) / (2 * h)
    return f0, canon(t.astype(np.asarray(f0).dtype), np.asarray(f0).dtype)


def grad(fun, argnums=0):
    def g(*args):
        x = float(np.asarray(args[argnums]))
        h = 1e-6 * max(1.0, abs(x))

        def at(val):
            a = list(args)
            a[argnums] = np.asarray(val, dtype=np.float64).view(JArray)
            return float(np.asarray(_eval64(fun, *a), dtype=np.float64))
        d = (at(x + h) - at(x - h)) / (2 * h)
        return canon(np.asarray(d, dtype=np.asarray(args[argnums]).dtype))
    return g
