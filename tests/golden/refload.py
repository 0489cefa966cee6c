"""Import the reference's Python source under the NumPy JAX stand-in.

TEST INFRASTRUCTURE for the fixture generators only: needs a checkout of the
reference project, named by the ``MULTIFIL_REF`` environment variable (the
directory that holds its ``multifil_jax`` package).  GPU machines have none;
the fixtures they test against are committed.  Package ``__init__`` files of the
reference are bypassed (they configure XLA), submodules are imported directly.
"""
import importlib
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def reference_root() -> str:
    ref = os.environ.get('MULTIFIL_REF')
    if not ref or not os.path.isdir(os.path.join(ref, 'multifil_jax')):
        raise RuntimeError('set MULTIFIL_REF to a checkout of the reference project (the directory '
                           'holding its multifil_jax package) to regenerate the fixtures')
    return ref


def load():
    REF = reference_root()
    shim = os.path.join(HERE, 'jaxshim')
    if shim not in sys.path:
        sys.path.insert(0, shim)
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    base = os.path.join(REF, 'multifil_jax')
    for name, path in [('multifil_jax', base), ('multifil_jax.core', os.path.join(base, 'core')),
                       ('multifil_jax.kernels', os.path.join(base, 'kernels')),
                       ('multifil_jax.utils', os.path.join(base, 'utils'))]:
        if name not in sys.modules:
            m = types.ModuleType(name)
            m.__path__ = [path]
            sys.modules[name] = m
    mods = {}
    for short, full in [('params', 'multifil_jax.core.params'), ('geo', 'multifil_jax.core.sarc_geometry'),
                        ('state', 'multifil_jax.core.state'), ('geometry', 'multifil_jax.kernels.geometry'),
                        ('rates', 'multifil_jax.kernels.rate_functions'),
                        ('trans', 'multifil_jax.kernels.transitions'), ('forces', 'multifil_jax.kernels.forces'),
                        ('solver', 'multifil_jax.kernels.solver'), ('timestep', 'multifil_jax.timestep'),
                        ('metrics', 'multifil_jax.metrics_fn'), ('sim', 'multifil_jax.simulation')]:
        mods[short] = importlib.import_module(full)
    return types.SimpleNamespace(**mods)
