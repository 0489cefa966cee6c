"""``jax.lax`` control flow on Python loops; JAX's associative_scan recursion."""
import numpy as _np

from ._core import canon, tree_util


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(_np.asarray(cond_fun(val))):
        val = body_fun(val)
    return val


def fori_loop(lower, upper, body_fun, init_val):
    val = init_val
    for i in range(int(lower), int(upper)):
        val = body_fun(i, val)
    return val


def scan(f, init, xs, length=None, unroll=1, reverse=False):
    leaves, spec = tree_util.tree_flatten(xs)
    n = _np.shape(leaves[0])[0] if leaves else length
    carry = init
    ys = []
    for i in range(n):
        x_i = tree_util.tree_unflatten(spec, [canon(_np.asarray(l)[i]) for l in leaves])
        carry, y = f(carry, x_i)
        ys.append(y)
    y_leaves0, y_spec = tree_util.tree_flatten(ys[0])
    ally = [tree_util.tree_flatten(y)[0] for y in ys]
    stacked = [canon(_np.stack([_np.asarray(a[j]) for a in ally])) for j in range(len(y_leaves0))]
    return carry, tree_util.tree_unflatten(y_spec, stacked)


def _slice(x, start, stop, step, axis):
    sl = [slice(None)] * _np.ndim(x)
    sl[axis] = slice(start, stop, step)
    return canon(_np.asarray(x)[tuple(sl)])


def _interleave(a, b, axis):
    a = _np.asarray(a)
    b = _np.asarray(b)
    n = a.shape[axis] + b.shape[axis]
    shape = list(a.shape)
    shape[axis] = n
    out = _np.empty(shape, dtype=_np.result_type(a.dtype, b.dtype))
    sl_a = [slice(None)] * a.ndim
    sl_b = [slice(None)] * a.ndim
    sl_a[axis] = slice(0, n, 2)
    sl_b[axis] = slice(1, n, 2)
    out[tuple(sl_a)] = a
    out[tuple(sl_b)] = b
    return canon(out)


def associative_scan(fn, elems, reverse=False, axis=0):
    """Prefix scan with JAX's odd/even recursive association order."""
    single = not isinstance(elems, (tuple, list))
    elems_l = [elems] if single else list(elems)
    if reverse:
        elems_l = [canon(_np.flip(_np.asarray(e), axis)) for e in elems_l]

    def combine(a, b):
        r = fn(a[0], b[0]) if single else fn(tuple(a), tuple(b))
        return [r] if single else list(r)

    def rec(es):
        n = _np.shape(es[0])[axis]
        if n < 2:
            return es
        reduced = combine([_slice(e, 0, -1, 2, axis) for e in es], [_slice(e, 1, None, 2, axis) for e in es])
        odd = rec(reduced)
        if n % 2 == 0:
            even = combine([_slice(e, 0, -1, None, axis) for e in odd], [_slice(e, 2, None, 2, axis) for e in es])
        else:
            even = combine(odd, [_slice(e, 2, None, 2, axis) for e in es])
        even = [canon(_np.concatenate([_np.asarray(_slice(e, 0, 1, None, axis)), _np.asarray(r)], axis=axis))
                for e, r in zip(es, even)]
        return [_interleave(e, o, axis) for e, o in zip(even, odd)]

    out = rec(elems_l)
    if reverse:
        out = [canon(_np.flip(_np.asarray(e), axis)) for e in out]
    return out[0] if single else tuple(out)
