"""NumPy-backed stand-in for the small part of JAX the reference uses.

TEST INFRASTRUCTURE: used only by ``tests/golden/make_golden.py`` to execute the
reference's own Python source (``multifil_jax``) in an environment without
JAX, so that golden fixtures come from the reference code itself.  It is never
imported by the product package, the oracle or any test at run time.

Semantics kept from JAX (x64 disabled unless ``config.update('jax_enable_x64',
True)``): float64/int64 results are canonicalised to float32/int32, Python
scalars are weakly typed, ``.at[].set`` applies duplicate updates in index
order (last writer wins, as XLA on CPU does), ``.at[].add``/``segment_sum``
accumulate in index order, ``lax.associative_scan`` reassociates with JAX's
odd/even recursion, ``jnp.cumsum`` is that scan, ``jnp.linspace`` evaluates
``lo*(1-t)+hi*t`` in the working dtype.  ``jax.jvp``/``jax.grad`` are central
finite differences evaluated in float64 and rounded to the primal dtype --
the one place where this stand-in is only an approximation of JAX.
"""
import functools
import sys
import types

import numpy as _np

from ._core import JArray, canon, config  # noqa: F401
from . import tree_util  # noqa: F401
from . import numpy  # noqa: F401
from . import lax  # noqa: F401
from . import random  # noqa: F401
from . import ops  # noqa: F401
from . import scipy  # noqa: F401
from ._core import vmap, jvp, grad  # noqa: F401

Array = JArray


def jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def device_put(x, *a, **k):
    return x


def block_until_ready(x):
    return x
