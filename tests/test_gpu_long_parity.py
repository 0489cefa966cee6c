"""Long runs of the benchmark workloads against the oracle, with injected draws.

* The single-condition workload: 2x2 skeletal lattice, pCa 4.5, z_line 900 nm,
  1000 steps of 1 ms, key split(PRNGKey(0), 1)[0].
* 16 of the 256 conditions of the pCa sweep (pCa = linspace(4, 7, 256),
  every 17th condition, keys split(PRNGKey(0), 256)[i]), 500 steps each.

Every condition runs on the oracle in float32 (its own draws) and in float64
(the float32 run's draws injected), and on the GPU in both precision modes
with the same draws injected:

* mixed mode vs the float64 oracle: integer state arrays bit-identical,
  positions and the force within 1e-5 relative, step by step, until the first
  divergence; a divergence is accepted only when its cause is a near tie that
  the two sides' rounding can split (a draw within 1e-5 of a cumulative-table
  threshold, an axial offset within 1e-4 nm of a bin edge).
* float32 mode vs the float32 oracle: the same, with the float32 floor.  The
  force sums thick_k * (x - x_rest) over positions stored as absolute float32
  (~58 nm at the M-line), so one rounding of a node position moves it by
  thick_k * ulp(58 nm) ~ 0.03 pN per filament: the bound is two ulps per
  thick filament.  The float32 residual sits at the reference's own floor
  (thick_k * 1e-4 ~ 0.75 pN, kernels/solver.py:91-104), right at the Newton
  tolerance, so whether a step takes one more Newton iteration follows
  rounding: that decision, or a draw within 1e-3 of a threshold, is the only
  accepted cause of a divergence.
* The GPU's own Threefry stream (no injection) gives the injected run's states
  at every step of the 1000-step run.

Set MF_PARITY_REPORT=<path> to write the per-run windows and errors as JSON.
"""
import json
import multiprocessing as mp
import os

import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params
from multifil_jax_b200.engine import MF_FLAG_PRECISE
from multifil_jax_b200.simulation import METRIC_KEYS
from oracle import prng
from tests.gpu_helpers import (run_engine, state_divergence, oracle_positions, divergence_cause,
                               float32_force_floor)
from tests.oracle_helpers import first_divergence

pytestmark = pytest.mark.gpu
KEYS = list(METRIC_KEYS)
SWEEP_IDX = list(range(0, 256, 17))  # 16 conditions
TIE = {np.float32: 1e-3, np.float64: 1e-5}


def _runs():
    pcas = np.linspace(4.0, 7.0, 256)
    keys = prng.split(prng.PRNGKey(0), 256)
    runs = [dict(name='single_2x2_pCa4.5_1000', pCa=4.5, T=1000, key=prng.split(prng.PRNGKey(0), 1)[0])]
    runs += [dict(name=f'sweep_{i}_pCa{pcas[i]:.4f}_500', pCa=float(pcas[i]), T=500, key=keys[i]) for i in SWEEP_IDX]
    return runs


def _oracle_job(job):
    """Both oracle runs of one condition (module-level: runs in a spawned worker)."""
    import numpy as np
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from oracle import step as OS
    pCa, T, key = job
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    zt, pt, lt = np.full(T, 900.0), np.full(T, pCa), np.full(T, 14.0)
    m32, i32 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, record_states=True)
    m64, i64 = OS.run_condition(topo, d.param_row(), zt, pt, lt, key, dt=np.float64, uniforms=i32['uniforms'],
                                record_states=True)
    return m32, i32, m64, i64


@pytest.fixture(scope='module')
def oracle_runs():
    jobs = [(r['pCa'], r['T'], r['key']) for r in _runs()]
    n = max(1, min(len(jobs), len(os.sched_getaffinity(0))))
    with mp.get_context('spawn').Pool(n) as pool:
        return pool.map(_oracle_job, jobs)


@pytest.fixture(scope='module')
def gpu_runs(engine, oracle_runs):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    runs = _runs()
    out = {}
    for mode, flags in (('float32', 0), ('mixed', MF_FLAG_PRECISE)):
        res = []
        for group in ([0], list(range(1, len(runs)))):
            T = runs[group[0]]['T']
            B = len(group)
            ut = np.stack([np.stack([u[0] for u in oracle_runs[g][1]['uniforms']]) for g in group])
            ux = np.stack([np.stack([u[1] for u in oracle_runs[g][1]['uniforms']]) for g in group])
            P = np.tile(d.param_row(), (B, 1))
            Z, L = np.full((B, T), 900.0), np.full((B, T), 14.0)
            PC = np.repeat(np.array([runs[g]['pCa'] for g in group])[:, None], T, 1)
            K = np.stack([runs[g]['key'] for g in group])
            r = run_engine(engine, topo, P, Z, PC, L, K, flags=flags, u_thin=ut, u_xb=ux, traces=True)
            res.append((group, r))
        out[mode] = res
    return topo, d, out


def _compare(topo, d, run, oracle, r, b, dtype):
    T = run['T']
    m_o, info = oracle
    div = state_divergence(r, b, info, topo, T)
    mdiv = first_divergence(r['metrics'][b:b + 1], m_o[None], KEYS)
    win = min(v for v in (div, mdiv, T) if v is not None)
    f_o, f_g = m_o[0, :win], r['metrics'][b, 0, :win]
    ferr = float(np.max(np.abs(f_g - f_o) / np.abs(f_o))) if win else 0.0
    fabs = float(np.max(np.abs(f_g - f_o))) if win else 0.0
    xo = oracle_positions(info, topo)[:win]
    xg = r['x_trace'][b, :win, :topo.n_dof]
    xerr = float(np.max(np.abs(xg - xo) / np.maximum(np.abs(xo), 10.0))) if win else 0.0
    cause = None
    if win < T:
        cause = divergence_cause(topo, d.param_row(), run['pCa'], 14.0, dtype, info, r, b, win)
    return dict(window=win, steps=T, force_rel_err=ferr, force_abs_err=fabs, pos_rel_err=xerr,
                cause=None if cause is None else cause[0], margin=None if cause is None else cause[1])


def _check_mode(gpu_runs, oracle_runs, mode):
    topo, d, out = gpu_runs
    runs = _runs()
    dtype = np.float32 if mode == 'float32' else np.float64
    which = 0 if mode == 'float32' else 2
    report = {}
    for group, r in out[mode]:
        for b, g in enumerate(group):
            oracle = (oracle_runs[g][which], oracle_runs[g][which + 1])
            report[runs[g]['name']] = _compare(topo, d, runs[g], oracle, r, b, dtype)
    path = os.environ.get('MF_PARITY_REPORT')
    if path:
        old = json.load(open(path)) if os.path.exists(path) else {}
        old[mode] = report
        json.dump(old, open(path, 'w'), indent=1)
    floor = float32_force_floor(topo, d)
    for name, rep in report.items():
        if mode == 'mixed':
            assert rep['force_rel_err'] <= 1e-5, (name, rep)
        else:
            assert rep['force_abs_err'] <= floor, (name, rep, floor)
        assert rep['pos_rel_err'] <= 1e-5, (name, rep)
        if rep['window'] < rep['steps']:
            ok = (rep['cause'] == 'draw' and rep['margin'] < TIE[dtype]) or \
                 (rep['cause'] == 'bin') or (rep['cause'] == 'newton' and mode == 'float32')
            assert ok, (name, rep)
    return report


def test_float32_mode_vs_float32_oracle(gpu_runs, oracle_runs):
    _check_mode(gpu_runs, oracle_runs, 'float32')


def test_mixed_mode_vs_float64_oracle(gpu_runs, oracle_runs):
    rep = _check_mode(gpu_runs, oracle_runs, 'mixed')
    full = sum(r['window'] == r['steps'] for r in rep.values())
    assert full >= len(rep) - 2, rep


def test_device_threefry_over_1000_steps(engine, gpu_runs):
    """No injection: the kernel draws the same uniforms itself (jax.random
    layout), so every state of the 1000-step run equals the injected run's."""
    topo, d, out = gpu_runs
    run = _runs()[0]
    T = run['T']
    r = run_engine(engine, topo, d.param_row()[None], np.full((1, T), 900.0), np.full((1, T), 4.5),
                   np.full((1, T), 14.0), run['key'][None], traces=True)
    inj = out['float32'][0][1]
    assert np.array_equal(r['state_trace'], inj['state_trace'])
    assert np.array_equal(r['bound_trace'], inj['bound_trace'])
    assert np.array_equal(r['metrics'], inj['metrics'])
