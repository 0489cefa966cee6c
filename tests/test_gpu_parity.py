"""CUDA engine vs the oracle and vs the reference's own outputs (needs a B200)."""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params, get_cardiac_params, run
from multifil_jax_b200.engine import MF_FLAG_DYNAMIC_LS, MF_FLAG_PRECISE, MF_FLAG_PLAIN, MF_FLAG_ORIGINAL_PRNG
from multifil_jax_b200.simulation import plan_batch, METRIC_KEYS
from oracle import prng, step as OS
from tests.gpu_helpers import (run_engine, oracle_with_states, state_divergence, oracle_positions,
                               divergence_cause, float32_force_floor)
from tests.oracle_helpers import first_divergence, compare_metrics

pytestmark = pytest.mark.gpu
KEYS = list(METRIC_KEYS)


@pytest.mark.parametrize('nr,nc,T,pCa,z', [(1, 1, 30, 4.5, 900.0), (2, 2, 40, 4.5, 900.0),
                                           (2, 2, 25, 6.0, 950.0), (3, 3, 12, 5.0, 1000.0),
                                           (5, 5, 12, 4.5, 900.0), (6, 6, 10, 5.5, 950.0)])
def test_kernel_matches_oracle_per_step(engine, nr, nc, T, pCa, z):
    """Injected identical uniforms: integer states bit-identical, positions/forces within 1e-5."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(nr, nc, s, d)
    key = prng.split(prng.PRNGKey(11), 1)[0]
    zt, pt, lt = np.full(T, z), np.full(T, pCa), np.full(T, 14.0)
    m_o, info = oracle_with_states(topo, d.param_row(), zt, pt, lt, key)
    ut = np.stack([u[0] for u in info['uniforms']])[None]
    ux = np.stack([u[1] for u in info['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], pt[None], lt[None], key[None],
                     u_thin=ut, u_xb=ux, traces=True)
    div = state_divergence(res, 0, info, topo, T)
    mdiv = first_divergence(res['metrics'], m_o[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    if win < T:  # only a near tie that float32 rounding can split
        cause, margin = divergence_cause(topo, d.param_row(), pCa, 14.0, np.float32, info, res, 0, win)
        assert cause in ('newton', 'bin') or margin < 1e-3, (win, cause, margin)
    xo = oracle_positions(info, topo)[:win]
    xg = res['x_trace'][0, :win, :topo.n_dof]
    # relative to the coordinate scale: a node near the M-line inherits the
    # float32 spacing of positions ~1000 nm away through the coupled solve
    assert np.max(np.abs(xg - xo) / np.maximum(np.abs(xo), 10.0)) < 1e-5
    # the force reads float32 absolute positions: within two roundings of
    # every M-line node (the float32 floor), bit-identical in most steps
    f_o, f_g = m_o[0, :win], res['metrics'][0, 0, :win]
    assert np.max(np.abs(f_g - f_o)) <= float32_force_floor(topo, d)
    bad = compare_metrics(res['metrics'], m_o[None], KEYS, rtol=1e-4, upto=win)
    assert not bad, bad


def test_device_threefry_matches_jax_layout(engine):
    """No injection: the kernel's own Threefry stream draws exactly the
    oracle's uniforms (jax.random layout), in both counter layouts, so the
    run equals the one with the oracle's draws injected, at every step."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    T = 60
    for part, flags in ((None, 0), (False, MF_FLAG_ORIGINAL_PRNG)):
        key = prng.split(prng.PRNGKey(3), 1, partitionable=part)[0]
        m_o, info = OS.run_condition(topo, d.param_row(), np.full(T, 900.0), np.full(T, 4.5), np.full(T, 14.0),
                                     key, record_states=True, partitionable=part)
        args = (engine, topo, d.param_row()[None], np.full((1, T), 900.0), np.full((1, T), 4.5),
                np.full((1, T), 14.0), key[None])
        own = run_engine(*args, traces=True, flags=flags)
        inj = run_engine(*args, traces=True, flags=flags,
                         u_thin=np.stack([u[0] for u in info['uniforms']])[None],
                         u_xb=np.stack([u[1] for u in info['uniforms']])[None])
        for k in ('state_trace', 'bound_trace', 'metrics', 'x_trace'):
            assert np.array_equal(own[k], inj[k]), (part, k)


def _golden_case(name):
    import os, sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_golden import RUNS, _trace
    nr, nc, preset, kw = RUNS[name]
    s, d = get_cardiac_params() if preset == 'cardiac' else get_skeletal_params()
    kw = dict(kw)
    if isinstance(kw.get('z_line'), str):
        kw['z_line'] = _trace(kw['z_line'], int(kw['duration_ms']))
    return SarcTopology.create(nr, nc, s, d), s, d, kw


@pytest.mark.parametrize('name', ['skel_1x1', 'skel_2x2', 'card_2x2_z950', 'sweep_2x2', 'dynls_1x1',
                                  'dynls_2x2', 'sine_2x2', 'poisson_1x1'])
def test_run_api_matches_reference_fixture(golden, name):
    """run() on the GPU against the reference's own run() output for the same inputs."""
    topo, s, d, kw = _golden_case(name)
    r = run(topo, dynamic_params=d, static_params=s, rng_seed=0, **kw)
    assert np.array_equal(r.rng_key, golden[f'run_{name}__rng_key'])
    B = int(np.prod(r.axial_force.shape[:-1]))
    T = r.n_steps
    mine = np.stack([r.metrics[k].reshape(B, T).astype(np.float64) for k in KEYS], axis=1)
    ref = np.stack([golden[f'run_{name}__{k}'].reshape(B, T) for k in KEYS], axis=1)
    div = first_divergence(mine, ref, KEYS)
    upto = div if div is not None else T
    print(f'\n{name}: window {upto} of {T}')
    assert upto >= min(T, 5), div
    bad = compare_metrics(mine, ref, KEYS, rtol=1e-4, upto=upto)
    assert not bad, bad


def test_plain_chunked_and_batched_are_identical(engine):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    B, T = 3, 24
    keys = prng.split(prng.PRNGKey(0), B)
    P = np.tile(d.param_row(), (B, 1))
    Z, PC, L = np.full((B, T), 900.0), np.repeat(np.array([4.5, 5.5, 6.5])[:, None], T, 1), np.full((B, T), 14.0)
    a = run_engine(engine, topo, P, Z, PC, L, keys)
    b = run_engine(engine, topo, P, Z, PC, L, keys, flags=MF_FLAG_PLAIN)
    c = run_engine(engine, topo, P, Z, PC, L, keys, chunk_steps=5)
    assert np.array_equal(a['metrics'], b['metrics'])
    assert np.array_equal(a['metrics'], c['metrics'])
    # a second chunked batch of the same shape replays the cached graph with
    # the new descriptor table: other inputs, the same results as unchunked
    PC2 = PC[::-1].copy()
    a2 = run_engine(engine, topo, P, Z, PC2, L, keys[::-1].copy())
    c2 = run_engine(engine, topo, P, Z, PC2, L, keys[::-1].copy(), chunk_steps=5)
    assert np.array_equal(a2['metrics'], c2['metrics'])
    assert not np.array_equal(a2['metrics'], a['metrics'])


def test_condition_alone_equals_in_mixed_batch(engine):
    """Uneven lattices and durations in one launch; each row equals its solo run."""
    s, d = get_skeletal_params()
    sizes = [(1, 1), (2, 2), (3, 2), (2, 2)]
    topos = [SarcTopology.create(r, c, s, d) for r, c in sizes]
    T = 20
    n_steps = [20, 7, 13, 20]
    keys = prng.split(prng.PRNGKey(5), 4)
    pcas = [4.5, 5.0, 6.0, 7.0]
    P = np.tile(d.param_row(), (4, 1))
    Z, PC, L = np.full((4, T), 920.0), np.repeat(np.array(pcas)[:, None], T, 1), np.full((4, T), 13.5)
    mix = run_engine(engine, topos, P, Z, PC, L, keys, n_steps=n_steps)
    for i in range(4):
        solo = run_engine(engine, topos[i], P[i:i + 1], Z[i:i + 1], PC[i:i + 1], L[i:i + 1], keys[i:i + 1],
                          n_steps=[n_steps[i]])
        assert np.array_equal(solo['metrics'][0, :, :n_steps[i]], mix['metrics'][i, :, :n_steps[i]])


@pytest.mark.parametrize('nr,nc', [(1, 1), (2, 2)])
def test_dynamic_lattice_spacing_matches_oracle(engine, nr, nc):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(nr, nc, s, d)
    T = 15
    key = prng.split(prng.PRNGKey(2), 1)[0]
    K = 5.0 * topo.n_thick
    zt = 900.0 + 0.5 * np.arange(T)
    m_o, info = oracle_with_states(topo, d.param_row(), zt, np.full(T, 4.5), np.full(T, 14.0), key, K_lat=K, nu=0.5)
    ut = np.stack([u[0] for u in info['uniforms']])[None]
    ux = np.stack([u[1] for u in info['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], np.full((1, T), 4.5), np.full((1, T), 14.0),
                     key[None], K_lat=[K], nu=[0.5], flags=MF_FLAG_DYNAMIC_LS, u_thin=ut, u_xb=ux, traces=True)
    div = state_divergence(res, 0, info, topo, T)
    mdiv = first_divergence(res['metrics'], m_o[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    print(f'\ndynamic spacing {nr}x{nc}: window {win} of {T}')
    assert win >= 5
    ls_o, ls_g = m_o[4, :win], res['metrics'][0, 4, :win]
    assert np.max(np.abs(ls_g - ls_o) / ls_o) < 1e-5
    bad = compare_metrics(res['metrics'], m_o[None], KEYS, rtol=1e-4, upto=win)
    assert not bad, bad


@pytest.mark.parametrize('nr,nc,pCa,T', [(2, 2, 4.5, 200), (2, 2, 5.5, 200), (2, 2, 6.5, 200),
                                         (5, 5, 5.0, 30), (6, 6, 4.5, 30)])
def test_mixed_precision_force_error_vs_fp64_oracle(engine, nr, nc, pCa, T):
    """'mixed' precision: <= 1e-5 relative force error against the FP64 oracle
    (same uniforms) over 200 steps at 2x2, and over 30 steps on the lattices
    whose solver vectors live in the workspace (5x5, 6x6); the states follow
    the oracle's throughout unless a draw falls within 1e-5 of a table
    threshold."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(nr, nc, s, d)
    key = prng.split(prng.PRNGKey(0), 1)[0]
    zt, pt, lt = np.full(T, 900.0), np.full(T, pCa), np.full(T, 14.0)
    m32, info32 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key)
    m64, info64 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, dt=np.float64,
                                   uniforms=info32['uniforms'], record_states=True)
    ut = np.stack([u[0] for u in info32['uniforms']])[None]
    ux = np.stack([u[1] for u in info32['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], pt[None], lt[None], key[None],
                     flags=MF_FLAG_PRECISE, u_thin=ut, u_xb=ux, traces=True)
    div = state_divergence(res, 0, info64, topo, T)
    mdiv = first_divergence(res['metrics'], m64[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    if win < T:
        cause, margin = divergence_cause(topo, d.param_row(), pCa, 14.0, np.float64, info64, res, 0, win)
        assert cause == 'bin' or (cause == 'draw' and margin < 1e-5), (win, cause, margin)
    f64, fg = m64[0, :win], res['metrics'][0, 0, :win]
    err_mixed = np.max(np.abs(fg - f64) / np.abs(f64))
    assert err_mixed <= 1e-5, err_mixed


@pytest.mark.parametrize('nr,nc,pCa', [(2, 2, 4.5), (3, 2, 5.5)])
def test_mixed_precision_dynamic_ls_vs_fp64_oracle(engine, nr, nc, pCa):
    """'mixed' precision with the lattice spacing solved as an unknown: force and
    spacing within 1e-5 relative of the FP64 oracle (same uniforms)."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(nr, nc, s, d)
    T = 25
    key = prng.split(prng.PRNGKey(4), 1)[0]
    K = 5.0 * topo.n_thick
    zt, pt, lt = 900.0 + 0.5 * np.arange(T), np.full(T, pCa), np.full(T, 14.0)
    m32, info32 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, K_lat=K, nu=0.5)
    m64, info64 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, dt=np.float64, K_lat=K, nu=0.5,
                                   uniforms=info32['uniforms'], record_states=True)
    ut = np.stack([u[0] for u in info32['uniforms']])[None]
    ux = np.stack([u[1] for u in info32['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], pt[None], lt[None], key[None], K_lat=[K],
                     nu=[0.5], flags=MF_FLAG_PRECISE | MF_FLAG_DYNAMIC_LS, u_thin=ut, u_xb=ux, traces=True)
    div = state_divergence(res, 0, info64, topo, T)
    mdiv = first_divergence(res['metrics'], m64[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    print(f'\nmixed dynamic spacing {nr}x{nc} pCa {pCa}: window {win} of {T}')
    assert win >= 3
    for row in (0, 4):  # axial_force, lattice_spacing
        ref, got = m64[row, :win], res['metrics'][0, row, :win]
        err = np.max(np.abs(got - ref) / np.abs(ref))
        assert err <= 1e-5, (METRIC_KEYS[row], err)


def test_bad_arguments_raise(engine):
    import torch
    from multifil_jax_b200.engine import EngineError
    s, d = get_skeletal_params()
    topo = SarcTopology.create(1, 1, s, d)
    with pytest.raises(EngineError):
        run_engine(engine, topo, d.param_row()[None], np.full((1, 4), 900.0), np.full((1, 4), 4.5),
                   np.full((1, 4), 14.0), prng.split(prng.PRNGKey(0), 1), n_steps=[9])


def test_run_conditions_matches_run_per_condition():
    """Mixed lattices, durations, dt and spacing modes in one launch equal one run() each."""
    from multifil_jax_b200 import run_conditions
    from multifil_jax_b200.engine import prng_split, prng_key
    s, d = get_skeletal_params()
    _, c = get_cardiac_params()
    t22, t11, t32 = (SarcTopology.create(r, k, s, d) for r, k in ((2, 2), (1, 1), (3, 2)))
    conds = [dict(topology=t22, duration_ms=20, pCa=5.0, z_line=910.0, key=prng_split(prng_key(3), 1)[0]),
             dict(topology=t11, duration_ms=6, dt=0.5, pCa=4.5, dynamic_params=c, key=prng_split(prng_key(4), 1)[0]),
             dict(topology=t32, duration_ms=9, pCa=6.0, lattice_spacing=13.5, key=prng_split(prng_key(5), 1)[0])]
    got = run_conditions(conds, precision='mixed')
    for cond, seed, g in zip(conds, (3, 4, 5), got):
        ref = run(cond['topology'], duration_ms=cond['duration_ms'], dt=cond.get('dt', 1.0), pCa=cond['pCa'],
                  z_line=cond.get('z_line', 900.0), lattice_spacing=cond.get('lattice_spacing', 14.0),
                  dynamic_params=cond.get('dynamic_params'), rng_seed=seed, precision='mixed')
        for k in METRIC_KEYS:
            assert np.array_equal(np.asarray(ref.metrics[k]).reshape(-1), g[k]), k
    dyn = run_conditions([dict(topology=t22, duration_ms=8, K_lat=5.0, nu=0.5),
                          dict(topology=t11, duration_ms=5, K_lat=5.0, nu=0.5)])
    ref = run(t22, duration_ms=8, K_lat=5.0, nu=0.5, rng_seed=0)
    assert np.array_equal(ref.metrics['lattice_spacing'].reshape(-1), dyn[0]['lattice_spacing'])
    with pytest.raises(ValueError):
        run_conditions([dict(topology=t22, duration_ms=5, K_lat=5.0), dict(topology=t11, duration_ms=5)])


def test_run_conditions_autotune():
    """run_conditions(autotune=True): per-lattice sizes checked on the batch itself;
    the results agree with the default sizes' (same draws; reduction orders differ)."""
    from multifil_jax_b200 import run_conditions
    from multifil_jax_b200.engine import get_engine
    s, d = get_skeletal_params()
    tops = [SarcTopology.create(r, k, s, d) for r, k in ((1, 1), (2, 1), (2, 2))]
    conds = [dict(topology=t, duration_ms=12, pCa=4.5 + 0.5 * i, K_lat=5.0, nu=0.5)
             for i, t in enumerate(tops * 3)]
    ref = run_conditions(conds, precision='mixed')
    try:
        got = run_conditions(conds, precision='mixed', autotune=True)
    finally:
        eng = get_engine()
        for t in tops:
            eng.tune_threads(t, 0, 'mixed')
    for r, g in zip(ref, got):
        assert np.all(np.isfinite(g['axial_force']))
        np.testing.assert_allclose(g['axial_force'], r['axial_force'], rtol=1e-2, atol=5.0)
        np.testing.assert_allclose(g['lattice_spacing'], r['lattice_spacing'], rtol=1e-3)


def test_identical_conditions_identical_results():
    """Copies of one condition in one launch give bit-identical metrics.  Sites
    holding two heads sum them in head order: their slots come from an atomic
    counter, and a contracted multiply-add is not symmetric in its terms (a
    4x4 mixed run split into two result classes at step 19 before)."""
    from multifil_jax_b200.engine import get_engine
    from tests.gpu_helpers import run_engine
    s, d = get_skeletal_params()
    topo = SarcTopology.create(4, 4, s, d)
    eng = get_engine()
    # the condition that showed it: pCa 4.0045, z 996.02 nm, key split(PRNGKey(1004), 1)[0]
    B, T = 48, 57
    key = prng.split(prng.PRNGKey(1004), 1)[0]
    for nt in (0, 1024):
        eng.tune_threads(topo, nt, 'mixed')
        try:
            m = run_engine(eng, topo, np.repeat(d.param_row()[None], B, 0), np.full((B, T), 996.0190412149619),
                           np.full((B, T), 4.004470250526508), np.full((B, T), 14.0), np.repeat(key[None], B, 0),
                           flags=MF_FLAG_PRECISE)['metrics']
        finally:
            eng.tune_threads(topo, 0, 'mixed')
        for b in range(1, B):
            assert np.array_equal(m[b], m[0]), (nt, b)


@pytest.mark.parametrize('flags', [0, MF_FLAG_PRECISE, MF_FLAG_PLAIN, MF_FLAG_PRECISE | MF_FLAG_DYNAMIC_LS])
def test_constant_drivers_equal_traces(engine, flags):
    """[B] drivers held for every step (MF_FLAG_CONST_DRIVERS, what run() sends
    for scalar sweeps) give exactly the results of the same values as [B, T]
    traces, in one launch, in CUDA-graph chunks and on the plain path."""
    import torch
    from tests.gpu_helpers import tt, keys_tensor
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    B, T = 5, 18
    zc, pc, lc = np.linspace(880.0, 960.0, B), np.linspace(4.2, 6.8, B), np.full(B, 14.0)
    P = np.tile(d.param_row(), (B, 1))
    keys = prng.split(prng.PRNGKey(9), B)
    dyn = bool(flags & MF_FLAG_DYNAMIC_LS)
    kl = np.full(B, 5.0 * topo.n_thick) if dyn else np.zeros(B)
    nu = np.full(B, 0.5) if dyn else np.zeros(B)
    common = dict(K_lat=tt(kl, torch.float32), nu=tt(nu, torch.float32), dt=tt(np.ones(B), torch.float32),
                  flags=flags)
    for chunk in (0, 7):
        if chunk and flags & MF_FLAG_PLAIN:
            continue
        ref = engine.run_batch(topo, tt(P, torch.float32), tt(np.repeat(zc[:, None], T, 1), torch.float32),
                               tt(np.repeat(pc[:, None], T, 1), torch.float32),
                               tt(np.repeat(lc[:, None], T, 1), torch.float32), tt(np.full(B, T, np.int32)),
                               keys_tensor(keys), chunk_steps=chunk, **common)
        got = engine.run_batch(topo, tt(P, torch.float32), tt(zc, torch.float32), tt(pc, torch.float32),
                               tt(lc, torch.float32), tt(np.full(B, T, np.int32)), keys_tensor(keys),
                               chunk_steps=chunk, n_time=T, **common)
        torch.cuda.synchronize()
        assert np.array_equal(got['metrics'].cpu().numpy(), ref['metrics'].cpu().numpy()), chunk
        assert np.array_equal(got['status'].cpu().numpy(), ref['status'].cpu().numpy())
