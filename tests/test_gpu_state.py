"""The public timestep split on caller-owned states (needs a B200).

``multifil_jax_b200.timestep`` (kinetics_step / solve_equilibrium / timestep /
create_and_equilibrate over ``mf_step_states``) against the reference's own
``timestep()`` states (golden fixture), against the fused kernel and against
the oracle.
"""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params
from multifil_jax_b200 import timestep as TS
from multifil_jax_b200.subpopulation import Subpopulation
from multifil_jax_b200.simulation import plan_batch
from oracle import prng, step as OS, physics as ph
from tests.gpu_helpers import run_engine

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _topo(nr=2, nc=2):
    s, d = get_skeletal_params()
    return SarcTopology.create(nr, nc, s, d), s, d


def test_state_steps_match_reference_timestep(golden):
    """20 calls of timestep() from create_and_equilibrate reproduce the states
    the reference's own timestep() produced (same key, same drivers)."""
    topo, s, d = _topo()
    st = TS.create_and_equilibrate(topo, d, 900.0, 4.5, 14.0)
    assert np.allclose(_np(st.thick.axial), golden['steps_2x2__init_thick_axial'], rtol=0, atol=2e-4)
    assert np.allclose(_np(st.thin.axial), golden['steps_2x2__init_thin_axial'], rtol=0, atol=2e-4)
    key = golden['steps_2x2__key0']
    drv = TS.Drivers(pCa=4.5, z_line=900.0, lattice_spacing=14.0)
    for t in range(golden['steps_2x2__xb_states'].shape[0]):
        st, key, res, ls, it = TS.timestep(st, d, drv, topo, key, dt=1.0, n_cg_steps=6, n_newton_steps=4)
        assert np.array_equal(_np(st.thick.xb_states).reshape(-1), golden['steps_2x2__xb_states'][t]), t
        assert np.array_equal(_np(st.thick.xb_bound_to).reshape(-1), golden['steps_2x2__xb_bound_to'][t]), t
        assert np.array_equal(_np(st.thin.tm_states).reshape(-1), golden['steps_2x2__tm_states'][t].reshape(-1)), t
        assert np.array_equal(_np(st.thin.bound_to), golden['steps_2x2__thin_bound_to'][t]), t
        assert np.allclose(_np(st.thick.axial), golden['steps_2x2__thick_axial'][t], rtol=1e-6, atol=1e-4), t
        assert np.allclose(_np(st.thin.axial), golden['steps_2x2__thin_axial'][t], rtol=1e-6, atol=1e-4), t
        assert int(it) == golden['steps_2x2__iters'][t] or abs(float(res) - 0.75) < 0.3
        assert float(ls) == 14.0


def test_kinetics_then_solve_equals_timestep():
    topo, s, d = _topo()
    st0 = TS.create_and_equilibrate(topo, d, 900.0, 4.5, 14.0)
    key = prng.split(prng.PRNGKey(5), 1)[0]
    drv = TS.Drivers(pCa=5.0, z_line=901.0, lattice_spacing=13.5)
    a, ka, ra, la, ia = TS.timestep(st0, d, drv, topo, key, dt=1.0, n_newton_steps=4)
    k1, kk, rc = TS.kinetics_step(st0, d, drv, topo, key, dt=1.0)
    assert np.array_equal(_np(k1.thick.axial), _np(st0.thick.axial))  # kinetics leaves positions
    assert float(rc.pCa) == 5.0 and float(rc.z_line) == 901.0 and float(rc.lattice_spacing) == 13.5
    b, rb, lb, ib = TS.solve_equilibrium(k1, rc, topo, n_newton_steps=4)
    assert np.array_equal(ka, kk)
    for x, y in zip(a.thick + a.thin, b.thick + b.thin):
        assert np.array_equal(_np(x), _np(y))
    assert float(ra) == float(rb) and int(ia) == int(ib)
    # the inputs were not modified
    assert np.array_equal(_np(st0.thick.xb_states), np.zeros_like(_np(st0.thick.xb_states)))


def test_state_api_equals_fused_run():
    """B states stepped one call per step equal the fused kernel's per-step
    states and positions, bit for bit (same phase code, same keys)."""
    topo, s, d = _topo()
    B, T = 3, 25
    pcas = np.array([4.5, 5.5, 6.5], np.float32)
    keys = prng.split(prng.PRNGKey(0), B)
    from multifil_jax_b200.engine import get_engine
    res = run_engine(get_engine(0), topo, np.tile(d.param_row(), (B, 1)), np.full((B, T), 900.0), np.repeat(pcas[:, None], T, 1),
                     np.full((B, T), 14.0), keys, traces=True)
    st = TS.create_and_equilibrate(topo, d, 900.0, 4.5, 14.0, batch=B)
    key = keys.copy()
    X, S = topo.total_xbs, topo.n_sites_total
    drv = TS.Drivers(pCa=pcas, z_line=900.0, lattice_spacing=14.0)
    for t in range(T):
        st, key, r, l, it = TS.timestep(st, d, drv, topo, key, dt=1.0, n_newton_steps=4)
        assert np.array_equal(_np(st.thick.xb_states).reshape(B, X), res['state_trace'][:, t, :X]), t
        assert np.array_equal(_np(st.thin.tm_states).reshape(B, S), res['state_trace'][:, t, X:X + S]), t
        assert np.array_equal(_np(st.thick.xb_bound_to).reshape(B, X), res['bound_trace'][:, t, :X]), t
        assert np.array_equal(_np(st.thin.bound_to).reshape(B, S), res['bound_trace'][:, t, X:X + S]), t
        x = np.concatenate([_np(st.thick.axial).reshape(B, -1), _np(st.thin.axial).reshape(B, -1)], axis=1)
        assert np.array_equal(x, res['x_trace'][:, t, :topo.n_dof]), t
        assert np.array_equal(_np(it), res['metrics'][:, 51, t].astype(np.int32)), t


def test_state_api_dynamic_spacing_matches_oracle():
    """timestep() with the spacing as an unknown against the oracle's
    augmented Newton (same uniforms): states identical, positions and spacing
    within 1e-5."""
    topo, s, d = _topo(1, 1)
    p = ph.param_dict(d.param_row(), np.float32)
    pre = ph.Preconditioner(topo, p, np.float32)
    c = OS.initial_condition(topo, p, 900.0, 4, 6, np.float32, pre)
    st = TS.create_and_equilibrate(topo, d, 900.0, 4.5, 14.0)
    K = 5.0 * topo.n_thick
    key = prng.split(prng.PRNGKey(3), 1)[0]
    cur = np.float32(14.0)
    tab_cache = {}
    for t in range(10):
        ut, ux, key_o = prng.step_uniforms(key, topo.n_sites_total, topo.total_xbs)
        k = float(cur)
        if k not in tab_cache:
            tab_cache.clear()
            tab_cache[k] = OS.tables(topo, p, 4.5, cur, 1.0, np.float32)
        c, _, ex = OS.timestep(topo, p, c, 900.0, 4.5, cur, 0.0, ut, ux, tab_cache[k], 4, 6, np.float32, pre, 1.0,
                               K_lat=K, d_ref=np.float32(14.0), want_metrics=False)
        st, key, r, ls, it = TS.timestep(st, d, TS.Drivers(4.5, 900.0, float(cur)), topo, key, dt=1.0, K_lat=K,
                                         d_ref=14.0, n_newton_steps=4, uniforms=(ut, ux))
        assert np.array_equal(_np(st.thick.xb_states).reshape(-1), c.xb_state), t
        assert np.array_equal(_np(st.thin.tm_states).reshape(-1), c.tm.reshape(-1)), t
        assert abs(float(ls) - float(ex['ls'])) <= 1e-5 * float(ex['ls']), t
        xo = np.concatenate([c.thick_x.reshape(-1), c.thin_x.reshape(-1)])
        xg = np.concatenate([_np(st.thick.axial).reshape(-1), _np(st.thin.axial).reshape(-1)])
        assert np.max(np.abs(xg - xo) / np.maximum(np.abs(xo), 10.0)) < 1e-5, t
        cur = np.float32(ex['ls'])
        key = key_o


def test_kinetics_step_with_subpopulations_equals_fused():
    """kinetics_step / timestep with the reference's (mode, constants_k, labels)
    tuples follow the same populations as run(subpopulation=...)."""
    topo, s, d = _topo()
    T = 12
    sub = Subpopulation.random(0.4, seed=1, xb_r01_coeff=3.0, tm_k_01=0.5)
    plan = plan_batch(topo, duration_ms=T, pCa=4.8, dynamic_params=d, static_params=s, rng_seed=3, subpopulation=sub)
    from tests.test_gpu_subpop import _run_plan_engine
    from multifil_jax_b200.engine import get_engine
    res = _run_plan_engine(get_engine(0), topo, plan)
    sp = plan.subpop
    ck = sub.apply_scales(d)
    xs = ('explicit', ck, sp.xb_label[0].astype(np.int32))
    tsub = ('explicit', ck, sp.tm_label[0].astype(np.int32))
    st = TS.create_and_equilibrate(topo, d, 900.0, 4.5, 14.0)
    key = plan.keys[0]
    X, S = topo.total_xbs, topo.n_sites_total
    for t in range(T):
        st, key, r, l, it = TS.timestep(st, d, TS.Drivers(4.8, 900.0, 14.0), topo, key, dt=1.0, n_newton_steps=4,
                                        xb_subpop=xs, tm_subpop=tsub)
        assert np.array_equal(_np(st.thick.xb_states).reshape(-1), res['state_trace'][0, t, :X]), t
        assert np.array_equal(_np(st.thin.tm_states).reshape(-1), res['state_trace'][0, t, X:X + S]), t


def test_state_api_errors():
    topo, s, d = _topo(1, 1)
    st = TS.realize_state(topo, d, 900.0, 4.5, 14.0)
    with pytest.raises(ValueError, match='d_ref'):
        TS.solve_equilibrium(st, d, topo, K_lat=5.0)
    other, _, _ = _topo(2, 2)
    with pytest.raises(ValueError, match='does not match'):
        TS.update_nearest_neighbors(st, d, other)
    with pytest.raises(ValueError, match='rng_key'):
        TS.kinetics_step(st, d, TS.Drivers(), topo, np.zeros(3, np.uint32), dt=1.0)
