"""The oracle against fixtures produced by running the reference source itself.

Fixtures: tests/golden/make_golden.py (reference run() / timestep() / expm
under the NumPy JAX stand-in).  The run cases go through the product's own
host glue (``plan_batch``), so sweep expansion, key split, Poisson spacing and
parameter tables are checked here too.
"""
import numpy as np
import pytest
import scipy.linalg

from multifil_jax_b200 import SarcTopology, StaticParams, DynamicParams, get_skeletal_params, get_cardiac_params
from multifil_jax_b200.simulation import plan_batch, METRIC_KEYS
from oracle import physics as ph, step as OS, prng
from tests.oracle_helpers import oracle_plan, first_divergence, compare_metrics

import sys, os
sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
from make_golden import RUNS, _trace  # noqa: E402


@pytest.mark.parametrize('tag', ['4.5_14.0', '6.0_12.5'])
def test_expm_tables_match_reference(golden, tag):
    s, d = get_skeletal_params()
    pCa, dd = map(float, tag.split('_'))
    t = SarcTopology.create(2, 2, s, d)
    p = ph.param_dict(d.param_row(), np.float32)
    Q = ph.xb_Q_bins(t, p, np.float32(pCa), np.float32(dd), np.float32)
    assert np.allclose(Q, golden[f'expm__Q_{tag}'], rtol=2e-6, atol=1e-6)
    Qg = golden[f'expm__Q_{tag}']
    truth = np.stack([scipy.linalg.expm(q.astype(np.float64)) for q in Qg])
    P, sq = ph.expm_pade6(Qg.astype(np.float32), with_s=True)
    R = golden[f'expm__P_{tag}']
    # float32 scaling-and-squaring is only good to ~6e-3 after 12+ squarings
    # (both the reference and the oracle); ~2e-4 below that.
    for X in (P, R):
        err = np.abs(X - truth) / (1e-6 + np.abs(truth))
        assert err[sq < 12].max() < 5e-4 and err[sq >= 12].max() < 1e-2
    err = np.abs(P - R) / (1e-6 + np.abs(R))
    assert err[sq < 12].max() < 5e-4 and err[sq >= 12].max() < 1e-2
    # the float64 path of the same algorithm is the truth to Pade accuracy
    assert np.allclose(ph.expm_pade6(Qg.astype(np.float64)), truth, rtol=1e-5, atol=1e-9)
    Pa, sa = ph.expm_pade6(ph.absorbing(Qg).astype(np.float32), with_s=True)
    err = np.abs(Pa - golden[f'expm__Pabs_{tag}']) / (1e-6 + np.abs(golden[f'expm__Pabs_{tag}']))
    assert err[sa < 12].max() < 5e-4 and err[sa >= 12].max() < 1e-2
    Qt = ph.tm_Q27(p, np.float32(pCa), np.float32)
    assert np.allclose(Qt, golden[f'expm__Qtm_{tag}'], rtol=2e-6, atol=1e-9)
    Pt = ph.expm_pade6(golden[f'expm__Qtm_{tag}'].astype(np.float32))
    assert np.allclose(Pt, golden[f'expm__Ptm_{tag}'], rtol=1e-4, atol=2e-6)


def _case(name):
    nr, nc, preset, kw = RUNS[name]
    s, d = get_cardiac_params() if preset == 'cardiac' else get_skeletal_params()
    kw = dict(kw)
    n = int(kw['duration_ms'])
    if isinstance(kw.get('z_line'), str):
        kw['z_line'] = _trace(kw['z_line'], n)
    topo = SarcTopology.create(nr, nc, s, d)
    plan = plan_batch(topo, dynamic_params=d, static_params=s, rng_seed=0, **kw)
    return topo, plan, s, d


def _golden_metrics(golden, name, plan):
    ref = np.stack([golden[f'run_{name}__{k}'].reshape(plan.total, plan.n_steps) for k in METRIC_KEYS], axis=1)
    return ref


@pytest.mark.parametrize('name', [n for n in RUNS if not n.startswith('x64')])
def test_oracle_run_matches_reference(golden, name):
    topo, plan, s, d = _case(name)
    assert np.allclose(plan.ls.reshape(-1), golden[f'run_{name}__lattice_spacing_trace'].reshape(-1)) or plan.dynamic_ls
    assert np.array_equal(plan.rng_key, golden[f'run_{name}__rng_key'])
    ref = _golden_metrics(golden, name, plan)
    mine, _ = oracle_plan(topo, plan, s)
    div = first_divergence(mine, ref, list(METRIC_KEYS))
    upto = div if div is not None else plan.n_steps
    # isometric cases agree over the whole run; z traces may hit a residual-floor
    # Newton decision earlier (poisson_1x1 does at step 5)
    assert upto >= min(plan.n_steps, 5), f"states or solver path diverged at step {div}"
    if 'z_line' not in RUNS[name][3] or not isinstance(RUNS[name][3]['z_line'], str):
        assert div is None, f"isometric case diverged at step {div}"
    bad = compare_metrics(mine, ref, list(METRIC_KEYS), rtol=1e-4, upto=upto)
    assert not bad, bad


def test_oracle_x64_matches_reference_fp64(golden):
    name = 'x64_2x2'
    topo, plan, s, d = _case(name)
    # FP64 reference: python-float parameters, float64 uniforms (64-bit draws)
    from multifil_jax_b200.params import _DEFAULTS
    row64 = np.array(list(_DEFAULTS.values()), dtype=np.float64)
    ref = _golden_metrics(golden, name, plan)
    mine, _ = oracle_plan(topo, plan, s, dtype=np.float64, udtype=np.float64, params=row64[None])
    div = first_divergence(mine, ref, list(METRIC_KEYS))
    upto = div if div is not None else plan.n_steps
    assert upto >= 10
    bad = compare_metrics(mine, ref, list(METRIC_KEYS), rtol=1e-6, upto=upto)
    bad.pop('solver_residual', None)
    assert not bad, bad


def test_oracle_steps_match_reference_states(golden):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    p = ph.param_dict(d.param_row(), np.float32)
    pre = ph.Preconditioner(topo, p, np.float32)
    c = OS.initial_condition(topo, p, 900.0, 4, 6, np.float32, pre)
    assert np.allclose(c.thick_x, golden['steps_2x2__init_thick_axial'], rtol=0, atol=2e-4)
    assert np.allclose(c.thin_x, golden['steps_2x2__init_thin_axial'], rtol=0, atol=2e-4)
    key = golden['steps_2x2__key0']
    tab = OS.tables(topo, p, 4.5, 14.0, 1.0, np.float32)
    cum = OS.thin_rest_cumsum(topo, np.float32)
    for t in range(golden['steps_2x2__xb_states'].shape[0]):
        ut, ux, key = prng.step_uniforms(key, topo.n_sites_total, topo.total_xbs)
        c, _, ex = OS.timestep(topo, p, c, 900.0, 4.5, 14.0, 0.0, ut, ux, tab, 4, 6, np.float32, pre, 1.0,
                               want_metrics=False, thin_rest_cum=cum)
        assert np.array_equal(c.xb_state, golden['steps_2x2__xb_states'][t]), t
        assert np.array_equal(c.xb_bound, golden['steps_2x2__xb_bound_to'][t]), t
        assert np.array_equal(c.tm.reshape(-1), golden['steps_2x2__tm_states'][t].reshape(-1)), t
        assert np.array_equal(c.thin_bound, golden['steps_2x2__thin_bound_to'][t]), t
        assert np.allclose(c.thick_x, golden['steps_2x2__thick_axial'][t], rtol=1e-6, atol=1e-4), t
        assert np.allclose(c.thin_x, golden['steps_2x2__thin_axial'][t], rtol=1e-6, atol=1e-4), t
        assert ex['iters'] == golden['steps_2x2__iters'][t] or abs(ex['residual'] - 0.75) < 0.3


def test_jvp_matches_finite_difference():
    s, d = get_skeletal_params()
    topo = SarcTopology.create(1, 1, s, d)
    p = ph.param_dict(d.param_row(), np.float64)
    rng = np.random.default_rng(0)
    st = rng.integers(0, 6, topo.total_xbs).astype(np.int8)
    bound = np.where((st >= 1) & (st <= 3), rng.integers(30, 80, topo.total_xbs), -1).astype(np.int32)
    fm = ph.ForceModel(topo, p, st, bound, 900.0, np.float64)
    x = np.concatenate([topo.crown_offsets.reshape(-1), (900.0 - topo.binding_offsets).reshape(-1)]).astype(np.float64)
    x = x + rng.normal(0, 0.5, x.shape)
    v = rng.normal(0, 1, x.shape)
    d0, vd, K, dref = 14.0, 0.3, 20.0, 14.2
    h = 1e-4
    fd = (fm.residual(x + h * v, d0 + h * vd) - fm.residual(x - h * v, d0 - h * vd)) / (2 * h)
    an, rad = fm.jvp(x, d0, v, vd, K)
    assert np.allclose(an, fd, rtol=1e-6, atol=1e-3)
    fdr = (fm.radial(x + h * v, d0 + h * vd, K, dref) - fm.radial(x - h * v, d0 - h * vd, K, dref)) / (2 * h)
    assert np.isclose(rad, fdr, rtol=1e-6, atol=1e-3)
