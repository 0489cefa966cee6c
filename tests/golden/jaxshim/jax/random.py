"""``jax.random`` on the oracle's Threefry implementation."""
import numpy as _np

from ._core import canon, config


def _prng():
    import oracle.prng as p
    return p


def PRNGKey(seed):
    return canon(_prng().PRNGKey(int(seed)), _np.uint32)


def split(key, num=2):
    return canon(_prng().split(_np.asarray(key), int(num)), _np.uint32)


def uniform(key, shape=(), dtype=None, minval=0.0, maxval=1.0):
    n = int(_np.prod(shape)) if shape else 1
    dt = dtype or (_np.float64 if config.x64 else _np.float32)
    u = _prng().uniform(_np.asarray(key), n, dt).reshape(shape)
    return canon(u, dt)
