"""Per-condition status bits on the device, caused without any GPU fault.

* A NaN in one condition's parameter row makes its residual non-finite: the
  condition reports MF_STATUS_NONFINITE (the reference zeroes non-finite
  Newton updates, kernels/solver.py:415, and its while-loop test is false on
  NaN), and the other conditions of the same launch are untouched.
* A Newton cap of one iteration with a tight residual tolerance leaves
  residuals above the tolerance: MF_STATUS_NOT_CONVERGED, and run() raises
  the reference's residual warning (simulation.py:1119-1127).
"""
import warnings

import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, StaticParams, get_skeletal_params, run
from multifil_jax_b200.engine import MF_FLAG_PRECISE, MF_STATUS_NONFINITE, MF_STATUS_NOT_CONVERGED
from multifil_jax_b200.params import DYNAMIC_FIELDS
from oracle import prng
from tests.gpu_helpers import run_engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('flags', [0, MF_FLAG_PRECISE])
def test_nan_parameter_row_sets_nonfinite_only_there(engine, flags):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    B, T = 3, 12
    P = np.tile(d.param_row(), (B, 1))
    P[1, DYNAMIC_FIELDS.index('titin_a')] = np.nan
    keys = prng.split(prng.PRNGKey(9), B)
    Z, PC, L = np.full((B, T), 900.0), np.full((B, T), 4.5), np.full((B, T), 14.0)
    res = run_engine(engine, topo, P, Z, PC, L, keys, flags=flags)
    assert res['status'][1] & MF_STATUS_NONFINITE
    # max|F| is NaN, so the Newton loop stops at once and reports it
    assert np.all(np.isnan(res['metrics'][1, 1])) and np.all(res['metrics'][1, 51] == 0)
    assert res['status'][0] == 0 and res['status'][2] == 0
    clean = run_engine(engine, topo, P[[0, 2]], Z[:2], PC[:2], L[:2], keys[[0, 2]], flags=flags)
    assert np.array_equal(clean['metrics'], res['metrics'][[0, 2]])
    assert np.array_equal(clean['status'], res['status'][[0, 2]])


def test_nan_parameter_warns_through_run():
    s, d = get_skeletal_params()
    topo = SarcTopology.create(1, 1, s, d)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter('always')
        r = run(topo, duration_ms=5, dynamic_params={'titin_a': [float('nan'), float(d.titin_a)]})
    assert any('non-finite' in str(x.message) for x in w)
    assert np.all(np.isfinite(r.axial_force[1]))


@pytest.mark.parametrize('precision', ['float32', 'mixed'])
def test_starved_newton_sets_not_converged(engine, precision):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    B, T = 2, 15
    keys = prng.split(prng.PRNGKey(2), B)
    args = (topo, np.tile(d.param_row(), (B, 1)), np.full((B, T), 900.0), np.full((B, T), 4.5),
            np.full((B, T), 14.0), keys)
    flags = MF_FLAG_PRECISE if precision == 'mixed' else 0
    loose = run_engine(engine, *args, flags=flags)
    assert np.all(loose['status'] == 0)
    # one Newton iteration and a 1e-4 pN tolerance: float32 cannot go below
    # its ~0.75 pN floor, and mixed precision stops near 1e-3 pN
    import torch
    from tests.gpu_helpers import tt, keys_tensor
    res = engine.run_batch(topo, tt(args[1], torch.float32), tt(args[2], torch.float32), tt(args[3], torch.float32),
                           tt(args[4], torch.float32), tt(np.full(B, T, np.int32)), keys_tensor(keys),
                           K_lat=tt(np.zeros(B), torch.float32), nu=tt(np.zeros(B), torch.float32),
                           dt=tt(np.ones(B), torch.float32), n_newton=1, flags=flags, residual_warn=1e-4)
    torch.cuda.synchronize()
    st = res['status'].cpu().numpy()
    m = res['metrics'].cpu().numpy()
    assert np.all(st & MF_STATUS_NOT_CONVERGED) and not np.any(st & MF_STATUS_NONFINITE)
    assert m[:, 1].max() > 1e-4 and m[:, 51].max() <= 1
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter('always')
        run(topo, duration_ms=T, z_line=900.0, static_params=StaticParams().replace(
            n_newton_steps=1, solver_residual_tol=1e-4), precision=precision)
    assert any('exceeds threshold' in str(x.message) for x in w)
