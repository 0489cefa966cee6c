"""Subpopulations: host resolution and the oracle against the reference's own runs.

Fixtures: tests/golden/make_subpop.py (the reference's ``run(...,
subpopulation=...)`` and mask generators under the NumPy JAX stand-in).
"""
import os
import sys

import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params, get_cardiac_params
from multifil_jax_b200.subpopulation import Subpopulation, generate_random_masks_batch, c_zone_masks
from multifil_jax_b200.simulation import plan_batch, METRIC_KEYS
from tests.oracle_helpers import oracle_plan, first_divergence, compare_metrics

sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
from make_subpop import CASES  # noqa: E402

KEYS = list(METRIC_KEYS)
SUBPOP = os.path.join(os.path.dirname(__file__), 'golden', 'subpop.npz')


@pytest.fixture(scope='module')
def fx():
    return dict(np.load(SUBPOP))


def _sub(topo, spec):
    ctor, args, kw = spec
    if ctor == 'c_zone':
        return Subpopulation.c_zone(topo, *args, **kw)
    return getattr(Subpopulation, ctor)(*args, **kw)


def subpop_case(name):
    """(topology, BatchPlan, static, dynamic) of one fixture case through the product's plan_batch."""
    nr, nc, preset, spec, kw = CASES[name]
    s, d = get_cardiac_params() if preset == 'cardiac' else get_skeletal_params()
    topo = SarcTopology.create(nr, nc, s, d)
    sub = [_sub(topo, x) for x in spec] if isinstance(spec, list) else _sub(topo, spec)
    plan = plan_batch(topo, dynamic_params=d, static_params=s, rng_seed=0, subpopulation=sub, **kw)
    return topo, plan, s, d, sub, kw


def test_random_masks_match_reference(fx):
    s, d = get_skeletal_params()
    t = SarcTopology.create(2, 2, s, d)
    xb, tm = generate_random_masks_batch(3, np.asarray([0.3, 0.6], np.float32), t, 2)
    assert np.array_equal(xb, fx['masks_random__xb'])
    assert np.array_equal(tm, fx['masks_random__tm'])


def test_czone_masks_match_reference(fx):
    s, d = get_skeletal_params()
    t = SarcTopology.create(2, 2, s, d)
    cz = Subpopulation.c_zone(t, tm_k_01=2.0, xb_r01_coeff=2.0)
    assert np.array_equal(cz.xb_mask, fx['masks_czone__xb'])
    assert np.array_equal(cz.tm_mask, fx['masks_czone__tm'])
    assert np.array_equal(cz.fractions, fx['masks_czone__fractions'])
    xb, tm = c_zone_masks(t, 350.0, 650.0, {'xb_r01_coeff': 2.0})
    assert not tm.any() and np.array_equal(xb, cz.xb_mask)


def test_subpopulation_errors():
    s, d = get_skeletal_params()
    t = SarcTopology.create(1, 1, s, d)
    with pytest.raises(ValueError, match='Unknown subpopulation scale'):
        Subpopulation.mean_field(0.5, not_a_field=2.0)
    with pytest.raises(ValueError, match='xb_\\* or tm_\\*'):
        plan_batch(t, duration_ms=3, subpopulation=Subpopulation.mean_field(0.5, thick_k=2.0))
    with pytest.raises(ValueError, match='share one mode'):
        plan_batch(t, duration_ms=3, subpopulation=[Subpopulation.mean_field(0.5, xb_r01_coeff=2.0),
                                                   Subpopulation.random(0.5, xb_r01_coeff=2.0)])
    with pytest.raises(ValueError, match='share one seed'):
        plan_batch(t, duration_ms=3, subpopulation=[Subpopulation.random(0.5, seed=1, xb_r01_coeff=2.0),
                                                   Subpopulation.random(0.5, seed=2, xb_r01_coeff=2.0)])
    with pytest.raises(ValueError, match='list is empty'):
        plan_batch(t, duration_ms=3, subpopulation=[])
    with pytest.raises(ValueError, match='candidate-style'):
        plan_batch(t, duration_ms=3, dynamic_params=[d, d], subpopulation=[Subpopulation.mean_field(0.5, xb_r01_coeff=2.0)])


def test_sweep_axis_and_rows():
    """A list of subpopulations is the last sweep axis; population rows scale only
    the named fields, in float32."""
    s, d = get_skeletal_params()
    t = SarcTopology.create(1, 1, s, d)
    subs = [Subpopulation.mean_field(f, xb_r34_coeff=3.0, tm_k_01=0.5) for f in (0.0, 0.25, 1.0)]
    plan = plan_batch(t, duration_ms=4, pCa=[4.5, 6.0], subpopulation=subs, replicates=2)
    assert plan.axis_names == ['pCa', 'subpopulation', 'replicates', 'time']
    assert plan.grid_shape == (2, 3)
    sp = plan.subpop
    assert sp.K == 2 and not sp.explicit and sp.xb and sp.tm
    from multifil_jax_b200.params import DYNAMIC_FIELDS
    c34, c01 = DYNAMIC_FIELDS.index('xb_r34_coeff'), DYNAMIC_FIELDS.index('tm_k_01')
    assert np.array_equal(sp.rows[:, 0], plan.params)
    assert np.all(sp.rows[:, 1, c34] == plan.params[:, c34] * np.float32(3.0))
    assert np.all(sp.rows[:, 1, c01] == plan.params[:, c01] * np.float32(0.5))
    others = [i for i in range(44) if i not in (c34, c01)]
    assert np.array_equal(sp.rows[:, 1, others], plan.params[:, others])
    assert np.allclose(sp.fractions[:, 1], np.tile(np.repeat([0.0, 0.25, 1.0], 2), 2))


@pytest.mark.parametrize('name', list(CASES))
def test_oracle_subpop_run_matches_reference(fx, name):
    topo, plan, s, d, _, _ = subpop_case(name)
    assert np.array_equal(plan.rng_key, fx[f'run_{name}__rng_key'])
    ref = np.stack([fx[f'run_{name}__{k}'].reshape(plan.total, plan.n_steps) for k in KEYS], axis=1)
    mine, _ = oracle_plan(topo, plan, s)
    div = first_divergence(mine, ref, KEYS)
    upto = div if div is not None else plan.n_steps
    assert upto == plan.n_steps, f"states or solver path diverged at step {div}"
    bad = compare_metrics(mine, ref, KEYS, rtol=1e-4, upto=upto)
    assert not bad, bad


def test_oracle_fraction_edges_are_exact():
    """fraction 0 reproduces the wild type and fraction 1 a global scale, bit for
    bit, in the mean-field and random modes (core/subpopulation.py:53-58)."""
    s, d = get_skeletal_params()
    t = SarcTopology.create(1, 1, s, d)
    kw = dict(duration_ms=10, pCa=4.5)
    wt, _ = oracle_plan(t, plan_batch(t, dynamic_params=d, **kw), s)
    scaled = d.copy(xb_r01_coeff=np.float32(d.xb_r01_coeff) * np.float32(3.0))
    glob, _ = oracle_plan(t, plan_batch(t, dynamic_params=scaled, **kw), s)
    assert not np.array_equal(wt, glob)
    for ctor in (Subpopulation.mean_field, Subpopulation.random):
        f0, _ = oracle_plan(t, plan_batch(t, dynamic_params=d, subpopulation=ctor(0.0, xb_r01_coeff=3.0), **kw), s)
        f1, _ = oracle_plan(t, plan_batch(t, dynamic_params=d, subpopulation=ctor(1.0, xb_r01_coeff=3.0), **kw), s)
        assert np.array_equal(f0, wt), ctor
        assert np.array_equal(f1, glob), ctor
