"""Subpopulations on the CUDA engine: against the oracle step by step and
against the reference's own run() output (needs a B200)."""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params, run
from multifil_jax_b200.engine import device_pops
from multifil_jax_b200.simulation import plan_batch, METRIC_KEYS
from multifil_jax_b200.subpopulation import Subpopulation
from oracle import prng, step as OS
from tests.gpu_helpers import run_engine, state_divergence, oracle_positions, float32_force_floor
from tests.oracle_helpers import first_divergence, compare_metrics, plan_subpop
from tests.test_subpop_oracle import CASES, subpop_case, fx  # noqa: F401

pytestmark = pytest.mark.gpu
KEYS = list(METRIC_KEYS)


def _run_plan_engine(engine, topo, plan, uniforms=None, flags=0):
    """The plan's conditions through Engine.run_batch with traces (and injected uniforms)."""
    import torch
    pops = device_pops(plan.subpop, torch.device('cuda', 0)) if plan.subpop is not None else None
    ut = ux = None
    if uniforms is not None:
        ut = np.stack([np.stack([u[0] for u in us]) for us in uniforms])
        ux = np.stack([np.stack([u[1] for u in us]) for us in uniforms])
    K = plan.K_lat if plan.dynamic_ls else None
    from tests.gpu_helpers import tt, keys_tensor
    B, T = plan.total, plan.n_steps
    res = engine.run_batch(topo, tt(plan.params, torch.float32), tt(plan.z, torch.float32), tt(plan.pCa, torch.float32),
                           tt(plan.ls, torch.float32), tt(np.full(B, T, np.int32)), keys_tensor(plan.keys),
                           K_lat=tt(np.zeros(B) if K is None else K, torch.float32), nu=tt(plan.nu, torch.float32),
                           dt=tt(np.full(B, plan.dt), torch.float32), flags=flags | (1 if plan.dynamic_ls else 0),
                           u_thin=None if ut is None else tt(ut, torch.float32),
                           u_xb=None if ux is None else tt(ux, torch.float32),
                           want_x_trace=True, want_state_trace=True, pops=pops)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in res.items()}


@pytest.mark.parametrize('kind', ['mean_field', 'random', 'c_zone', 'random_dyn'])
def test_kernel_matches_oracle_with_subpopulations(engine, kind):
    """Injected identical uniforms: integer states bit-identical over the whole
    run, positions within 1e-5 of the coordinate scale, force within the float32
    floor, metrics within 1e-4."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    T = 30
    kw = dict(duration_ms=T, pCa=4.8, z_line=900.0, dynamic_params=d, static_params=s, rng_seed=5)
    if kind == 'mean_field':
        sub = Subpopulation.mean_field(0.4, xb_r01_coeff=2.5, xb_r34_coeff=0.5, tm_k_01=2.0)
    elif kind == 'c_zone':
        sub = Subpopulation.c_zone(topo, xb_r23_coeff=0.5, tm_k_12=1.5)
    else:
        sub = Subpopulation.random(0.35, seed=9, xb_r01_coeff=3.0, tm_J_C=2.0)
    if kind == 'random_dyn':
        kw.update(K_lat=5.0, nu=0.5, duration_ms=15)
        T = 15
    plan = plan_batch(topo, subpopulation=sub, **kw)
    m_o, info = OS.run_condition(topo, plan.params[0], plan.z[0], plan.pCa[0], plan.ls[0], plan.keys[0],
                                 K_lat=float(plan.K_lat[0]) if plan.dynamic_ls else None, nu=float(plan.nu[0]),
                                 record_states=True, subpop=plan_subpop(plan, 0))
    res = _run_plan_engine(engine, topo, plan, uniforms=[info['uniforms']])
    sdiv = state_divergence(res, 0, info, topo, T)
    mdiv = first_divergence(res['metrics'], m_o[None], KEYS, solver=False)
    assert sdiv is None and mdiv is None, (sdiv, mdiv)
    # the Newton iteration count may split where the float32 residual sits at
    # its floor (an accept-or-iterate decision within rounding); compare the
    # continuous values up to the first such step
    ndiv = first_divergence(res['metrics'], m_o[None], KEYS)
    win = T if ndiv is None else ndiv
    print(f'\n{kind}: states identical over {T} steps, Newton path over {win}')
    assert win >= 5
    xo = oracle_positions(info, topo)[:win]
    xg = res['x_trace'][0, :win, :topo.n_dof]
    assert np.max(np.abs(xg - xo) / np.maximum(np.abs(xo), 10.0)) < 1e-5
    assert np.max(np.abs(res['metrics'][0, 0, :win] - m_o[0, :win])) <= float32_force_floor(topo, d)
    bad = compare_metrics(res['metrics'], m_o[None], KEYS, rtol=1e-4, upto=win)
    assert not bad, bad
    # the device's own Threefry draws the oracle's uniforms: same run without injection
    own = _run_plan_engine(engine, topo, plan)
    assert np.array_equal(own['state_trace'], res['state_trace'])


@pytest.mark.parametrize('name', list(CASES))
def test_run_subpop_matches_reference_fixture(fx, name):
    """run(subpopulation=...) on the GPU against the reference's own run()."""
    topo, plan, s, d, sub, kw = subpop_case(name)
    r = run(topo, dynamic_params=d, static_params=s, rng_seed=0, subpopulation=sub, **kw)
    assert np.array_equal(r.rng_key, fx[f'run_{name}__rng_key'])
    B = int(np.prod(r.axial_force.shape[:-1]))
    T = r.n_steps
    mine = np.stack([r.metrics[k].reshape(B, T).astype(np.float64) for k in KEYS], axis=1)
    ref = np.stack([fx[f'run_{name}__{k}'].reshape(B, T) for k in KEYS], axis=1)
    assert first_divergence(mine, ref, KEYS, solver=False) is None, name
    div = first_divergence(mine, ref, KEYS)
    upto = T if div is None else div
    print(f'\n{name}: state counts identical over {T} steps, Newton path over {upto}')
    assert upto >= min(T, 5)
    # the force (and the first-crown energy) read float32 absolute positions of
    # the M-line nodes: within two roundings of each of them (the float32 floor)
    fi, ei = KEYS.index('axial_force'), KEYS.index('thick_energy_first_avg')
    assert np.max(np.abs(mine[:, fi, :upto] - ref[:, fi, :upto])) <= float32_force_floor(topo, d)
    assert np.max(np.abs(mine[:, ei, :upto] - ref[:, ei, :upto]) / np.abs(ref[:, ei, :upto])) < 1e-3
    rest = np.ones(len(KEYS), bool)
    rest[[fi, ei]] = False
    bad = compare_metrics(mine[:, rest], ref[:, rest], [k for k, r in zip(KEYS, rest) if r], rtol=1e-4, upto=upto)
    assert not bad, bad


@pytest.mark.parametrize('ctor', ['mean_field', 'random'])
def test_fraction_edges_are_exact_on_gpu(ctor):
    """fraction 0 is the wild type and fraction 1 a global scale, bit for bit."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    kw = dict(duration_ms=20, pCa=[4.5, 5.5], static_params=s, rng_seed=2)
    wt = run(topo, dynamic_params=d, **kw)
    scaled = d.copy(xb_r01_coeff=np.float32(d.xb_r01_coeff) * np.float32(3.0), tm_k_01=np.float32(d.tm_k_01) * np.float32(0.5))
    glob = run(topo, dynamic_params=scaled, **kw)
    f = getattr(Subpopulation, ctor)
    f0 = run(topo, dynamic_params=d, subpopulation=f(0.0, xb_r01_coeff=3.0, tm_k_01=0.5), **kw)
    f1 = run(topo, dynamic_params=d, subpopulation=f(1.0, xb_r01_coeff=3.0, tm_k_01=0.5), **kw)
    for k in KEYS:
        assert np.array_equal(f0.metrics[k], wt.metrics[k]), k
        assert np.array_equal(f1.metrics[k], glob.metrics[k]), k
    assert not np.array_equal(wt.axial_force, glob.axial_force)


@pytest.mark.parametrize('kind', ['mean_field', 'random'])
def test_subpop_mixed_precision_vs_fp64_oracle(engine, kind):
    """'mixed' precision with populations: force within 1e-5 relative of the
    FP64 oracle (same uniforms, same populations) while the states agree."""
    from multifil_jax_b200.engine import MF_FLAG_PRECISE
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    T = 60
    f = getattr(Subpopulation, kind)
    plan = plan_batch(topo, duration_ms=T, pCa=5.0, dynamic_params=d, static_params=s, rng_seed=8,
                      subpopulation=f(0.4, xb_r01_coeff=2.0, xb_r34_coeff=1.5, tm_k_01=0.5))
    sp = plan_subpop(plan, 0)
    args = (topo, plan.params[0], plan.z[0], plan.pCa[0], plan.ls[0], plan.keys[0])
    _, info32 = OS.run_condition(*args, subpop=sp)
    m64, info64 = OS.run_condition(*args, dt=np.float64, uniforms=info32['uniforms'], record_states=True, subpop=sp)
    res = _run_plan_engine(engine, topo, plan, uniforms=[info32['uniforms']], flags=MF_FLAG_PRECISE)
    div = state_divergence(res, 0, info64, topo, T)
    mdiv = first_divergence(res['metrics'], m64[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    print(f'\nmixed {kind}: window {win} of {T}')
    assert win >= 20
    err = np.max(np.abs(res['metrics'][0, 0, :win] - m64[0, :win]) / np.abs(m64[0, :win]))
    assert err <= 1e-5, err


def test_subpop_sweep_axis_layout():
    """A list of subpopulations is a sweep axis of the result."""
    s, d = get_skeletal_params()
    topo = SarcTopology.create(1, 1, s, d)
    subs = [Subpopulation.random(f, seed=4, xb_r01_coeff=2.0, tm_k_01=0.5) for f in (0.2, 0.8)]
    a = run(topo, duration_ms=20, pCa=[4.5, 6.0], dynamic_params=d, static_params=s, subpopulation=subs, replicates=2)
    assert a.axial_force.shape == (2, 2, 2, 20)
    assert a._axis_names == ['pCa', 'subpopulation', 'replicates', 'time']
    assert np.all(np.isfinite(a.axial_force))
