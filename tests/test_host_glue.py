"""run()'s host side: sweep expansion, parameter tables, result container (CPU only)."""
import warnings

import numpy as np
import pytest

from multifil_jax_b200 import (SarcTopology, DynamicParams, StaticParams, get_skeletal_params,
                               get_cardiac_params, DYNAMIC_FIELDS)
from multifil_jax_b200.simulation import plan_batch, assemble_result, SimulationResult, METRIC_KEYS, MetricsDict
from oracle import prng


@pytest.fixture(scope='module')
def topo():
    return SarcTopology.create(2, 2)


def test_scalar_run_shape_and_keys(topo):
    p = plan_batch(topo, duration_ms=10)
    assert p.total == 1 and p.n_steps == 10 and p.grid_shape == () and p.axis_names == ['replicates', 'time']
    assert np.array_equal(p.keys[0], prng.split(prng.PRNGKey(0), 1)[0])
    assert p.params.shape == (1, 44) and p.params.dtype == np.float32
    assert np.all(p.z == 900.0) and np.all(p.pCa == 4.5) and np.all(p.ls == 14.0)


def test_fixed_axis_order_and_cartesian_product(topo):
    # axes come out z_line, pCa, lattice_spacing, K_lat, nu, params -- not call order
    p = plan_batch(topo, duration_ms=5, pCa=[4.0, 5.0, 6.0], z_line=[900.0, 950.0], replicates=2,
                   dynamic_params={'xb_r01_coeff': [300.0, 310.0]})
    assert p.axis_names == ['z_line', 'pCa', 'xb_r01_coeff', 'replicates', 'time']
    assert p.grid_shape == (2, 3, 2) and p.total == 24
    # replicates innermost: rows 0,1 share every sweep value
    assert p.pCa[0, 0] == p.pCa[1, 0] and p.z[0, 0] == 900.0 and p.z[-1, 0] == 950.0
    i = DYNAMIC_FIELDS.index('xb_r01_coeff')
    assert p.params[0, i] == np.float32(300.0) and p.params[2, i] == np.float32(310.0)
    assert np.array_equal(p.keys, prng.split(prng.PRNGKey(0), 24))


def test_candidate_list_and_dict_overrides(topo):
    _, card = get_cardiac_params()
    _, skel = get_skeletal_params()
    p = plan_batch(topo, duration_ms=3, dynamic_params=[skel, card])
    assert p.axis_names[0] == 'candidates' and p.total == 2
    j = DYNAMIC_FIELDS.index('xb_r05')
    assert p.params[0, j] == np.float32(0.007) and p.params[1, j] == np.float32(0.2)
    p = plan_batch(topo, duration_ms=3, dynamic_params={'thick_k': 8000.0})
    assert p.params[0, 0] == 8000.0 and p.total == 1


def test_traces_and_trace_sweeps(topo):
    tr = 900 + np.arange(6.0)
    p = plan_batch(topo, duration_ms=6, z_line=tr)
    assert np.array_equal(p.z[0], tr.astype(np.float32))
    p = plan_batch(topo, duration_ms=6, z_line=[tr, tr + 1])
    assert p.grid_shape == (2,) and isinstance(p.coords['z_line'][0], np.ndarray)
    with pytest.raises(ValueError):
        plan_batch(topo, duration_ms=6, z_line=np.arange(5.0))


def test_poisson_and_dynamic_lattice_spacing(topo):
    tr = 900 + np.arange(4.0)
    p = plan_batch(topo, duration_ms=4, z_line=tr, nu=0.5)
    expect = (np.float32(14.0) * (np.float32(900.0) / tr.astype(np.float32)) ** np.float32(0.5)).astype(np.float32)
    assert np.allclose(p.ls[0], expect, rtol=1e-7)
    p = plan_batch(topo, duration_ms=4, K_lat=5.0, nu=0.5)
    assert p.dynamic_ls and p.K_lat[0] == np.float32(5.0 * topo.n_thick)
    assert p.topology_config['K_lat_eff'] == 5.0 * topo.n_thick


def test_errors(topo):
    with pytest.raises(ValueError):
        plan_batch(topo, duration_ms=3, pCa=[])
    with pytest.raises(ValueError):
        plan_batch(topo, duration_ms=3, dynamic_params={'nope': 1.0})
    with pytest.raises(ValueError):
        plan_batch(topo, duration_ms=3, dynamic_params=[])
    with pytest.raises(ValueError):
        plan_batch(topo, duration_ms=3, dynamic_params=42)
    with pytest.raises(TypeError):
        plan_batch(topo, duration_ms=3, subpopulation=object())


def test_padding_key_is_last_of_bucket(topo):
    # 3 conditions pad to 4: the returned key is split(PRNGKey(seed+1), 1)[-1]
    p = plan_batch(topo, duration_ms=2, pCa=[4.0, 5.0, 6.0], rng_seed=5)
    assert np.array_equal(p.rng_key, prng.split(prng.PRNGKey(6), 1)[-1])
    p = plan_batch(topo, duration_ms=2, pCa=[4.0, 5.0], rng_seed=5)
    assert np.array_equal(p.rng_key, p.keys[-1])


def _fake_result(topo, **kw):
    p = plan_batch(topo, **kw)
    m = np.random.default_rng(0).random((p.total, 52, p.n_steps)).astype(np.float32)
    m[:, METRIC_KEYS.index('solver_residual')] = 0.1
    return p, assemble_result(p, m, StaticParams(), 0)


def test_result_cube_sel_mean_std_stack(topo):
    p, r = _fake_result(topo, duration_ms=5, pCa=[4.0, 5.0, 6.0], replicates=4)
    assert r.axial_force.shape == (3, 4, 5) and r.n_steps == 5 and r.metrics['newton_iters'].dtype == np.int32
    assert isinstance(r.metrics, MetricsDict) and r.metrics.axial_force is r.metrics['axial_force']
    s = r.sel(pCa=5.0)
    assert s.axial_force.shape == (4, 5) and 'pCa' not in s.coords
    m = r.mean()
    assert m.axial_force.shape == (3, 5) and np.allclose(m.axial_force, r.axial_force.mean(axis=-2))
    sd = r.std()
    assert np.allclose(sd.axial_force, r.axial_force.std(axis=-2))
    st = SimulationResult.stack([r, r], axis_name='size', axis_values=[2, 3])
    assert st.axial_force.shape == (2, 3, 4, 5) and st._axis_names[0] == 'size'
    sub = r[1:]
    assert sub.coords['pCa'] == [5.0, 6.0]
    assert 'Mean force' in r.summary() and np.isclose(r.time[-1], 4.0)
    with pytest.raises(ValueError):
        r.sel(pCa=9.9)
    with pytest.raises(ValueError):
        r.sel(thick_k=1.0)


def test_result_axis_bookkeeping(topo):
    """Integers drop their axis, slices cut coordinates, other keys keep the
    bookkeeping; reductions average the drivers; trace-sweep coordinates
    select by value."""
    p, r = _fake_result(topo, duration_ms=4, pCa=[4.0, 5.0], z_line=[900.0, 950.0, 1000.0], replicates=2)
    assert r._axis_names == ['z_line', 'pCa', 'replicates', 'time']
    a = r[1]
    assert a._axis_names == ['pCa', 'replicates', 'time'] and 'z_line' not in a.coords
    assert a.axial_force.shape == (2, 2, 4) and np.array_equal(a.z_line, r.z_line[1])
    b = r[:, 0]
    assert b._axis_names == ['z_line', 'replicates', 'time'] and b.coords['z_line'] == [900.0, 950.0, 1000.0]
    c = r[np.array([0, 2])]
    assert c._axis_names == r._axis_names and c.coords == r.coords and c.axial_force.shape[0] == 2
    d = r[::2]
    assert d.coords['z_line'] == [900.0, 1000.0]
    sd = r.std()
    assert sd.name == 'run_std' and sd._axis_names == ['z_line', 'pCa', 'time']
    assert np.array_equal(sd.pCa, r.pCa.mean(axis=-2)) and 'replicates' not in sd.coords
    one = SimulationResult.stack([r.mean()], axis_name='size')
    assert one.coords['size'] == [0] and one.name == 'run_mean_stacked'
    tr = np.linspace(900.0, 905.0, 4)
    _, t = _fake_result(topo, duration_ms=4, z_line=[tr, tr + 1.0])
    picked = t.sel(z_line=t.coords['z_line'][1])
    assert np.array_equal(picked.z_line[0], (tr + 1.0).astype(np.float32))
    with pytest.raises(ValueError):
        r.mean().mean()


def test_residual_warning(topo):
    p = plan_batch(topo, duration_ms=2)
    m = np.zeros((1, 52, 2), np.float32)
    m[:, 1] = 3.0
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter('always')
        assemble_result(p, m, StaticParams(), 0)
    assert any('exceeds threshold' in str(x.message) for x in w)


def test_params_api():
    s, d = get_skeletal_params()
    d2 = d.copy(xb_r01_coeff=350.0)
    assert float(d2.xb_r01_coeff) == np.float32(350.0) and float(d.xb_r01_coeff) == np.float32(305.99)
    with pytest.raises(ValueError):
        d.copy(bogus=1.0)
    assert len(DYNAMIC_FIELDS) == 44 and d.param_row().shape == (44,)
    assert s.replace(n_cg_steps=3).n_cg_steps == 3
    with pytest.raises(ValueError):
        StaticParams(n_superlattice_classes=2)


def test_choose_batch_sizes_keeps_the_faster_set(monkeypatch):
    """The batch-level check of the autotuner: per-lattice sizes against the
    largest of them for every lattice, timed by run_short, faster set kept
    and left set in the engine (host logic only, with a stand-in engine)."""
    from types import SimpleNamespace
    from multifil_jax_b200 import autotune

    class FakeEngine:
        def __init__(self):
            self.sizes = {}

        def tune_threads(self, topo, threads, precision=None):
            if threads == 1024 and topo.nrows == 4:
                raise RuntimeError('does not fit')
            self.sizes[(topo.nrows, topo.ncols)] = threads

    eng = FakeEngine()
    monkeypatch.setattr(autotune, 'get_engine', lambda device=None: eng)
    tops = [SimpleNamespace(nrows=1, ncols=1), SimpleNamespace(nrows=2, ncols=2), SimpleNamespace(nrows=4, ncols=4)]
    picks = {(1, 1): 256, (2, 2): 384, (4, 4): 512}

    def timer(uniform_faster):
        def run_short():
            uniform = len(set(eng.sizes.values())) == 1
            return 1.0 if uniform == uniform_faster else 2.0
        return run_short

    kept = autotune.choose_batch_sizes(tops, picks, timer(True), precision='mixed')
    assert kept == {(1, 1): 512, (2, 2): 512, (4, 4): 512} and eng.sizes == kept
    eng.sizes = dict(picks)
    kept = autotune.choose_batch_sizes(tops, picks, timer(False), precision='mixed')
    assert kept == picks and eng.sizes == picks
    # one size already: nothing to compare
    assert autotune.choose_batch_sizes(tops[:1], {(1, 1): 256}, timer(True)) == {(1, 1): 256}


def test_scalar_sweep_matches_constant_trace_sweep(topo):
    """plan_batch broadcasts a sweep of scalars; the driver arrays equal those
    of the same sweep given as constant traces.  Scalars stay one value per
    condition (time stride 0, uploaded as [B] with MF_FLAG_CONST_DRIVERS);
    traces are materialised."""
    pcas = [4.0, 5.25, 6.5]
    a = plan_batch(topo, duration_ms=7, pCa=pcas, z_line=[900.0, 950.0])
    b = plan_batch(topo, duration_ms=7, pCa=[np.full(7, v) for v in pcas],
                   z_line=[np.full(7, 900.0), np.full(7, 950.0)])
    for name in ('pCa', 'z', 'ls', 'params', 'keys'):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert a.pCa.dtype == np.float32 and a.pCa.shape == (6, 7)
    assert a.const_drivers and a.pCa.strides[1] == 0
    assert not b.const_drivers and b.pCa.flags['C_CONTIGUOUS']


def test_const_drivers_only_when_every_driver_is_held(topo):
    """BatchPlan.const_drivers (the [B] upload with MF_FLAG_CONST_DRIVERS) holds
    exactly when z, pCa and the spacing are each one value per condition."""
    T = 6
    ramp = np.linspace(900.0, 905.0, T)
    cases = [
        (dict(pCa=4.5, z_line=900.0), True),
        (dict(pCa=[4.5, 5.5], z_line=[900.0, 950.0], lattice_spacing=[13.5, 14.0]), True),
        (dict(pCa=4.5, z_line=ramp), False),                      # a z trace
        (dict(pCa=[np.full(T, 4.5), np.full(T, 5.0)]), False),    # a sweep of traces
        (dict(pCa=4.5, z_line=ramp, nu=0.5), False),              # Poisson spacing from the z trace
        (dict(pCa=4.5, z_line=900.0, K_lat=5.0, nu=0.5), True),   # spacing solved: drivers still held
    ]
    for kw, expect in cases:
        p = plan_batch(topo, duration_ms=T, **kw)
        assert p.const_drivers is expect, kw
        for a in (p.z, p.pCa, p.ls):
            assert a.shape == (p.total, T) and a.dtype == np.float32
        if expect:
            for a in (p.z, p.pCa, p.ls):
                assert np.array_equal(a, np.repeat(a[:, :1], T, axis=1))
    assert not plan_batch(topo, duration_ms=0.5, pCa=4.5).const_drivers  # no steps
