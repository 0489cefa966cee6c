"""Invertebrate (insect flight muscle), superlattice and legacy-face lattices:
the topology builder and the oracle against the reference's own outputs.

Fixtures: tests/golden/make_invertebrate.py (the reference's
SarcTopology.create and run() under the NumPy JAX stand-in).
"""
import os
import sys

import numpy as np
import pytest

from multifil_jax_b200 import (SarcTopology, get_skeletal_params, get_lethocerus_params, get_drosophila_params,
                               StaticParams)
from multifil_jax_b200.simulation import plan_batch, METRIC_KEYS
from tests.oracle_helpers import oracle_plan, first_divergence, compare_metrics

sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
from make_invertebrate import LATTICES, RUNS  # noqa: E402
from make_golden import TOPO_FIELDS  # noqa: E402

KEYS = list(METRIC_KEYS)
FIXTURE = os.path.join(os.path.dirname(__file__), 'golden', 'invertebrate.npz')
PRESETS = {'lethocerus': get_lethocerus_params, 'drosophila': get_drosophila_params,
           'skeletal': get_skeletal_params}


@pytest.fixture(scope='module')
def inv():
    return dict(np.load(FIXTURE))


def lattice(name):
    nr, nc, preset, ov = LATTICES[name]
    s, d = PRESETS[preset]()
    if ov:
        s = s.replace(**ov)
    return SarcTopology.create(nr, nc, s, d), s, d


@pytest.mark.parametrize('name', list(LATTICES))
def test_topology_matches_reference(inv, name):
    t, _, _ = lattice(name)
    ints = [t.n_thick, t.n_crowns, t.n_thin, t.n_sites, t.n_titin, t.n_xb_per_crown, t.n_faces_per_thin,
            t.max_sites_per_face, t.total_xbs, t.n_xb_bins]
    assert ints == list(inv[f'topo_{name}__ints'])
    for f in TOPO_FIELDS:
        a, b = np.asarray(getattr(t, f)), inv[f'topo_{name}__{f}']
        assert a.shape == b.shape and a.dtype == b.dtype, (f, a.shape, b.shape, a.dtype, b.dtype)
        assert np.array_equal(a, b), f


def test_preset_values():
    s, d = get_lethocerus_params()
    assert (s.actin_geometry, s.n_xb_per_crown, s.n_crowns, s.mono_per_poly) == ('invertebrate', 4, 100, 28)
    assert float(d.titin_rest) == 50.0
    s2, _ = get_drosophila_params()
    assert s2.n_superlattice_classes == 3 and s2.replace(n_superlattice_classes=1) == s


def test_lattice_errors():
    s, d = get_drosophila_params()
    with pytest.raises(ValueError, match='superlattice'):
        SarcTopology.create(2, 2, s, d)
    s, d = get_lethocerus_params()
    with pytest.raises(ValueError, match='even nrows'):
        SarcTopology.create(3, 2, s, d)
    with pytest.raises(ValueError):
        StaticParams(legacy_crown_geometry=True, n_xb_per_crown=4)


@pytest.mark.parametrize('name', list(RUNS))
def test_oracle_run_matches_reference(inv, name):
    lat, kw = RUNS[name]
    t, s, d = lattice(lat)
    plan = plan_batch(t, dynamic_params=d, static_params=s, rng_seed=0, **kw)
    assert np.array_equal(plan.rng_key, inv[f'run_{name}__rng_key'])
    ref = np.stack([inv[f'run_{name}__{k}'].reshape(plan.total, plan.n_steps) for k in KEYS], axis=1)
    mine, _ = oracle_plan(t, plan, s)
    assert first_divergence(mine, ref, KEYS, solver=False) is None
    div = first_divergence(mine, ref, KEYS)
    upto = plan.n_steps if div is None else div
    assert upto >= min(plan.n_steps, 5)
    bad = compare_metrics(mine, ref, KEYS, rtol=1e-4, upto=upto)
    assert not bad, bad
