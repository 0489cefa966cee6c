"""Ensemble statistics against the reference: 64 seeds of the 2x2 isometric run.

``tests/golden/ensemble.npz`` holds the axial-force traces of the reference's
own ``run(topo, duration_ms=100, pCa=4.5, z_line=900, replicates=64,
rng_seed=0)`` (generated by ``tests/golden/make_ensemble.py``).  The engine
runs the same call (same per-replicate keys) in both precision modes; the
ensemble mean of the per-seed mean force over the last 50 ms must lie inside
the reference ensemble's 95 % interval for its mean, mean +- 1.96 sd / sqrt(64).
"""
import os

import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params, run

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
WINDOW = 50


@pytest.mark.parametrize('precision', ['float32', 'mixed'])
def test_ensemble_mean_force_within_reference_interval(precision):
    fx = np.load(os.path.join(HERE, 'golden', 'ensemble.npz'))
    ref = fx['axial_force']
    n_seeds = ref.shape[0]
    per_seed_ref = ref[:, -WINDOW:].mean(axis=1)
    mu, sd = per_seed_ref.mean(), per_seed_ref.std(ddof=1)
    half = 1.96 * sd / np.sqrt(n_seeds)
    s, d = get_skeletal_params()
    topo = SarcTopology.create(int(fx['nrows']), int(fx['ncols']), s, d)
    r = run(topo, duration_ms=float(fx['duration_ms']), pCa=float(fx['pCa']), z_line=float(fx['z_line']),
            replicates=n_seeds, rng_seed=int(fx['rng_seed']), dynamic_params=d, static_params=s,
            precision=precision)
    per_seed = r.axial_force.reshape(n_seeds, -1)[:, -WINDOW:].mean(axis=1)
    m = per_seed.mean()
    print(f"\n  {precision}: ensemble mean force {m:.3f} pN, reference {mu:.3f} +- {half:.3f} pN (95 %)")
    assert abs(m - mu) <= half, (m, mu, half)
