"""Insect flight muscle, superlattice and legacy-face lattices on the CUDA
engine (needs a B200): 160-site thin filaments with two faces, four heads per
crown of which about half have no partner, 100 crowns per thick filament."""
import numpy as np
import pytest

from multifil_jax_b200 import run
from multifil_jax_b200.engine import MF_FLAG_PRECISE
from multifil_jax_b200.simulation import plan_batch, METRIC_KEYS
from oracle import prng, step as OS
from tests.gpu_helpers import run_engine, state_divergence, oracle_positions, float32_force_floor
from tests.oracle_helpers import first_divergence, compare_metrics
from tests.test_invertebrate_oracle import lattice, inv, RUNS  # noqa: F401

pytestmark = pytest.mark.gpu
KEYS = list(METRIC_KEYS)


@pytest.mark.parametrize('name,z,T', [('leth_2x2', 1550.0, 20), ('dros_2x3', 1525.0, 12), ('vert4_2x2', 900.0, 20),
                                      ('legacy_2x2', 900.0, 20)])
def test_kernel_matches_oracle_per_step(engine, name, z, T):
    """Injected identical uniforms: integer states bit-identical over the run,
    positions within 1e-5 of the coordinate scale, metrics within 1e-4."""
    topo, s, d = lattice(name)
    key = prng.split(prng.PRNGKey(12), 1)[0]
    zt, pt, lt = np.full(T, z), np.full(T, 4.5), np.full(T, 14.0)
    m_o, info = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, record_states=True)
    ut = np.stack([u[0] for u in info['uniforms']])[None]
    ux = np.stack([u[1] for u in info['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], pt[None], lt[None], key[None],
                     u_thin=ut, u_xb=ux, traces=True)
    assert state_divergence(res, 0, info, topo, T) is None
    assert first_divergence(res['metrics'], m_o[None], KEYS, solver=False) is None
    div = first_divergence(res['metrics'], m_o[None], KEYS)
    win = T if div is None else div
    print(f'\n{name}: states identical over {T} steps, Newton path over {win}')
    assert win >= 5
    xo = oracle_positions(info, topo)[:win]
    xg = res['x_trace'][0, :win, :topo.n_dof]
    assert np.max(np.abs(xg - xo) / np.maximum(np.abs(xo), 10.0)) < 1e-5
    assert np.max(np.abs(res['metrics'][0, 0, :win] - m_o[0, :win])) <= 4 * float32_force_floor(topo, d)
    rest = [k for k in KEYS if k not in ('axial_force', 'thick_energy_first_avg')]
    idx = [KEYS.index(k) for k in rest]
    bad = compare_metrics(res['metrics'][:, idx], m_o[None][:, idx], rest, rtol=1e-4, upto=win)
    assert not bad, bad


@pytest.mark.parametrize('name', list(RUNS))
def test_run_matches_reference_fixture(inv, name):
    lat, kw = RUNS[name]
    topo, s, d = lattice(lat)
    r = run(topo, dynamic_params=d, static_params=s, rng_seed=0, **kw)
    assert np.array_equal(r.rng_key, inv[f'run_{name}__rng_key'])
    B = int(np.prod(r.axial_force.shape[:-1]))
    T = r.n_steps
    mine = np.stack([r.metrics[k].reshape(B, T).astype(np.float64) for k in KEYS], axis=1)
    ref = np.stack([inv[f'run_{name}__{k}'].reshape(B, T) for k in KEYS], axis=1)
    assert first_divergence(mine, ref, KEYS, solver=False) is None
    div = first_divergence(mine, ref, KEYS)
    upto = T if div is None else div
    print(f'\n{name}: state counts identical over {T} steps, Newton path over {upto}')
    assert upto >= min(T, 5)
    fi, ei = KEYS.index('axial_force'), KEYS.index('thick_energy_first_avg')
    assert np.max(np.abs(mine[:, fi, :upto] - ref[:, fi, :upto])) <= 4 * float32_force_floor(topo, d)
    rest = [k for k in KEYS if k not in ('axial_force', 'thick_energy_first_avg')]
    idx = [KEYS.index(k) for k in rest]
    bad = compare_metrics(mine[:, idx], ref[:, idx], rest, rtol=1e-4, upto=upto)
    assert not bad, bad


def test_ifm_mixed_precision_vs_fp64_oracle(engine):
    """'mixed' precision on the Lethocerus lattice: force within 1e-5 of the
    FP64 oracle (same uniforms) while the states agree."""
    topo, s, d = lattice('leth_2x2')
    T = 25
    key = prng.split(prng.PRNGKey(2), 1)[0]
    zt, pt, lt = np.full(T, 1550.0), np.full(T, 4.5), np.full(T, 14.0)
    _, info32 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key)
    m64, info64 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, dt=np.float64,
                                   uniforms=info32['uniforms'], record_states=True)
    ut = np.stack([u[0] for u in info32['uniforms']])[None]
    ux = np.stack([u[1] for u in info32['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], pt[None], lt[None], key[None],
                     flags=MF_FLAG_PRECISE, u_thin=ut, u_xb=ux, traces=True)
    div = state_divergence(res, 0, info64, topo, T)
    mdiv = first_divergence(res['metrics'], m64[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    print(f'\nIFM mixed: window {win} of {T}')
    assert win >= 10
    err = np.max(np.abs(res['metrics'][0, 0, :win] - m64[0, :win]) / np.abs(m64[0, :win]))
    assert err <= 1e-5, err


def test_ifm_dynamic_spacing_matches_oracle(engine):
    """Dynamic lattice spacing on the insect lattice (float32, injected
    uniforms): states identical to the oracle's, spacing and positions within
    1e-5, over the Newton path shared with the oracle."""
    from multifil_jax_b200.engine import MF_FLAG_DYNAMIC_LS
    topo, s, d = lattice('leth_2x2')
    T = 10
    key = prng.split(prng.PRNGKey(6), 1)[0]
    K = 5.0 * topo.n_thick
    zt = 1550.0 + 0.5 * np.arange(T)
    m_o, info = OS.run_condition(topo, d.param_row(), zt, np.full(T, 4.5), np.full(T, 14.0), key, K_lat=K, nu=0.5,
                                 record_states=True)
    ut = np.stack([u[0] for u in info['uniforms']])[None]
    ux = np.stack([u[1] for u in info['uniforms']])[None]
    res = run_engine(engine, topo, d.param_row()[None], zt[None], np.full((1, T), 4.5), np.full((1, T), 14.0),
                     key[None], K_lat=[K], nu=[0.5], flags=MF_FLAG_DYNAMIC_LS, u_thin=ut, u_xb=ux, traces=True)
    sdiv = state_divergence(res, 0, info, topo, T)
    div = first_divergence(res['metrics'], m_o[None], KEYS)
    win = min(v for v in (sdiv, div, T) if v is not None)
    print(f'\nIFM dynamic spacing: window {win} of {T}')
    assert win >= 5
    ls_o, ls_g = m_o[4, :win], res['metrics'][0, 4, :win]
    assert np.max(np.abs(ls_g - ls_o) / ls_o) < 1e-5
    xo = oracle_positions(info, topo)[:win]
    xg = res['x_trace'][0, :win, :topo.n_dof]
    assert np.max(np.abs(xg - xo) / np.maximum(np.abs(xo), 10.0)) < 1e-5
