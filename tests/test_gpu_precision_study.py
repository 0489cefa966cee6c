"""Sinusoidal length perturbation: complex stiffness, float32 and mixed vs the FP64 oracle.

2x2 skeletal lattice at pCa 4.5, z(t) = 900 + 2 sin(2 pi f t) nm, for four
frequencies of the grid f = logspace(0, 2.7, 64) Hz (indices 31, 36, 41, 46:
21-94 Hz, the range where the FP64 oracle finishes in seconds).  dt =
min(1, 1000 / (20 f)) ms, duration max(5 cycles, 200 ms); the complex
stiffness Y = DFT(F) / DFT(z) at the stimulus frequency over the whole
cycles after one settling cycle (the method of the reference's
``examples/sinusoidal_analysis.py``).  Every run consumes the same uniforms
(drawn once from the condition's key), so the GPU and the FP64 oracle
sample against the same numbers; a trajectory may still leave the FP64 one
where a transition probability sits within rounding of a uniform.

Asserted: mixed precision's force stays within 1e-5 of the FP64 oracle up to
the first step where an integer state count or the Newton iteration count
differs, and that window covers the settling cycle.  The stiffness errors
are printed per frequency (``-s`` shows them).
"""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params
from multifil_jax_b200.engine import MF_FLAG_PRECISE
from multifil_jax_b200.simulation import METRIC_KEYS
from oracle import prng, step as OS
from tests.gpu_helpers import run_engine
from tests.oracle_helpers import first_divergence

pytestmark = pytest.mark.gpu
FREQ_INDEX = (31, 36, 41, 46)


def sinusoid(k):
    f = 10.0 ** (2.7 * k / 63.0)
    dt = min(1.0, 1000.0 / (20.0 * f))
    n = int(max(5000.0 / f, 200.0) / dt)
    t_ms = np.arange(n) * dt
    return f, dt, n, (900.0 + 2.0 * np.sin(2.0 * np.pi * f * t_ms / 1000.0)).astype(np.float32)


def complex_stiffness(force, z, f, dt):
    period = 1000.0 / f / dt
    n0 = int(round(period))
    cycles = int((len(force) - n0) // period)
    n1 = n0 + int(round(cycles * period))
    t = np.arange(n0, n1) * dt / 1000.0
    ph = np.exp(-2j * np.pi * f * t)
    F = np.asarray(force[n0:n1], np.float64)
    Z = np.asarray(z[n0:n1], np.float64)
    return np.sum((F - F.mean()) * ph) / np.sum((Z - Z.mean()) * ph)


def uniforms_for(key, topo, n):
    out = []
    for _ in range(n):
        ut, ux, key = prng.step_uniforms(key, topo.n_sites_total, topo.total_xbs, np.float32)
        out.append((ut, ux))
    return out


def test_sinusoid_complex_stiffness_vs_fp64_oracle(engine):
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    key = prng.split(prng.PRNGKey(0), 1)[0]
    rows = []
    for k in FREQ_INDEX:
        f, dt, n, z = sinusoid(k)
        pCa, ls = np.full(n, 4.5), np.full(n, 14.0)
        uni = uniforms_for(key, topo, n)
        m64, _ = OS.run_condition(topo, d.param_row(), z, pCa, ls, key, dt_ms=dt, dt=np.float64, uniforms=uni)
        ut = np.stack([u[0] for u in uni])[None]
        ux = np.stack([u[1] for u in uni])[None]
        y64 = complex_stiffness(m64[0], z, f, dt)
        res = {}
        for name, flags in (('float32', 0), ('mixed', MF_FLAG_PRECISE)):
            g = run_engine(engine, topo, d.param_row()[None], z[None], pCa[None], ls[None], key[None],
                           flags=flags, u_thin=ut, u_xb=ux, dt=[dt])['metrics']
            res[name] = (g, first_divergence(g, m64[None], list(METRIC_KEYS)))
        gm, dm = res['mixed']
        win = dm if dm is not None else n
        period = int(round(1000.0 / f / dt))
        assert win >= period, (f, win, period)
        ferr = np.max(np.abs(gm[0, 0, :win] - m64[0, :win]) / np.maximum(np.abs(m64[0, :win]), 1.0))
        assert ferr <= 1e-5, (f, ferr)
        for name in ('float32', 'mixed'):
            g, div = res[name]
            y = complex_stiffness(g[0, 0], z, f, dt)
            rows.append((f, name, abs(y - y64) / abs(y64), np.angle(y / y64), div, n))
    print('\n  f (Hz)  mode     |dY|/|Y|   dphase (rad)  first divergence / steps')
    for f, name, ry, dph, div, n in rows:
        print(f'  {f:6.1f}  {name:7s}  {ry:9.2e}  {dph:+10.2e}    {div if div is not None else "none"} / {n}')
        assert np.isfinite(ry) and np.isfinite(dph)
