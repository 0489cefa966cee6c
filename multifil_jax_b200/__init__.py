"""multifil_jax_b200 -- the multifil_jax half-sarcomere timestep on NVIDIA B200 (sm_100a).

Drop-in for the reference's public API (travistune3/multifil_jax):

    from multifil_jax_b200 import SarcTopology, run, get_skeletal_params
    static, dynamic = get_skeletal_params()
    topo = SarcTopology.create(nrows=2, ncols=2, static_params=static, dynamic_params=dynamic)
    result = run(topo, pCa=4.5, z_line=900.0, duration_ms=1000,
                 dynamic_params=dynamic, static_params=static)
    result.axial_force            # (replicates, time)

The time loop runs in hand-written CUDA kernels (``csrc/``) behind a C ABI
(``include/multifil_b200.h``) loaded through ctypes; there is no CPU fallback.
"""
__version__ = '0.1.0'

from .params import (StaticParams, DynamicParams, DYNAMIC_FIELDS, get_skeletal_params,  # noqa: F401
                     get_cardiac_params, get_lethocerus_params, get_drosophila_params)
from .topology import SarcTopology  # noqa: F401
from .simulation import run, run_conditions, SimulationResult, MetricsDict, METRIC_KEYS  # noqa: F401
from .subpopulation import Subpopulation  # noqa: F401
from . import timestep  # noqa: F401


def get_ca_concentration(pCa: float) -> float:
    """10**(-pCa) (reference core/state.py:319-328)."""
    return 10.0 ** (-pCa)


__all__ = ['run', 'run_conditions', 'SimulationResult', 'SarcTopology', 'Subpopulation', 'timestep', 'StaticParams', 'DynamicParams', 'DYNAMIC_FIELDS',
           'get_skeletal_params', 'get_cardiac_params', 'get_lethocerus_params', 'get_drosophila_params', 'get_ca_concentration', 'MetricsDict',
           'METRIC_KEYS']
