"""The kernel's transition tables against the reference's and the float64 truth.

The tables are what sampling reads: cumulative rows of expm(Q dt) on the
crossbridge bin grid and for the 27 tropomyosin configurations, and the three
absorbing-chain entries the metrics read (kernels/transitions.py:99-190,
434-513, 807-922, 1029-1078).  The device builds them with the step kernel's
own table builder (mf_transition_tables).

* float32 mode: against the reference's own expm_pade6_batch output (the
  golden fixtures), within the bounds float32 scaling-and-squaring itself
  meets against the truth (it amplifies a rounding difference by 2^s).
* mixed mode (float64 squaring of the renormalised Pade result): against
  scipy's float64 expm of the same generators, <= 1e-5 relative on every
  entry, which is the per-step transition-probability bar.
"""
import numpy as np
import pytest
import scipy.linalg

from multifil_jax_b200 import SarcTopology, get_skeletal_params
from oracle import physics as ph

pytestmark = pytest.mark.gpu
TAGS = ['4.5_14.0', '6.0_12.5']


def _rel(a, b):
    return np.abs(a - b) / (np.abs(b) + 1e-6)


def _squarings(Q):
    return ph.expm_pade6(Q.astype(np.float32), with_s=True)[1]


def _setup(tag):
    s, d = get_skeletal_params()
    pCa, dd = map(float, tag.split('_'))
    return SarcTopology.create(2, 2, s, d), d, pCa, dd


@pytest.mark.parametrize('tag', TAGS)
def test_float32_tables_match_reference(engine, golden, tag):
    topo, d, pCa, dd = _setup(tag)
    cum_tm, cum_xb, pabs = engine.transition_tables(topo, d.param_row(), pCa, dd, 1.0, 'float32')
    Q = golden[f'expm__Q_{tag}']
    sq = _squarings(Q).reshape(2, -1)
    ref = np.cumsum(golden[f'expm__P_{tag}'].astype(np.float64), axis=-1).reshape(cum_xb.shape)
    err = _rel(cum_xb, ref).max(axis=(2, 3))
    lo, hi = err[sq < 8].max(), err[sq >= 8].max()
    print(f'\n{tag} float32 cum rows vs reference: s<8 {lo:.2e}, s>=8 {hi:.2e}')
    assert lo < 1e-4 and hi < 1e-2, (lo, hi)
    Pa = golden[f'expm__Pabs_{tag}'].reshape(2, -1, 6, 6)
    ref_abs = np.stack([Pa[..., 3, 4], Pa[..., 2, 0], Pa[..., 3, 0]], axis=-1)
    sa = _squarings(ph.absorbing(Q)).reshape(2, -1)
    ea = np.abs(pabs - ref_abs).max(axis=-1)  # absolute: the metrics sum these probabilities
    assert ea[sa < 8].max() < 1e-5 and ea.max() < 1e-3, (ea[sa < 8].max(), ea.max())
    ref_tm = np.cumsum(golden[f'expm__Ptm_{tag}'].astype(np.float64), axis=-1)
    assert _rel(cum_tm, ref_tm).max() < 1e-4


@pytest.mark.parametrize('tag', TAGS)
def test_mixed_tables_match_float64_truth(engine, golden, tag):
    """Transition probabilities of the mixed mode within 1e-5 of float64 expm."""
    topo, d, pCa, dd = _setup(tag)
    cum_tm, cum_xb, pabs = engine.transition_tables(topo, d.param_row(), pCa, dd, 1.0, 'mixed')
    Q = golden[f'expm__Q_{tag}'].astype(np.float64)
    truth = np.stack([scipy.linalg.expm(q) for q in Q])
    err = _rel(cum_xb, np.cumsum(truth, axis=-1).reshape(cum_xb.shape))
    print(f'\n{tag} mixed cum rows vs float64 expm: max rel {err.max():.2e}')
    assert err.max() <= 1e-5, err.max()
    Ta = np.stack([scipy.linalg.expm(q) for q in ph.absorbing(Q)]).reshape(2, -1, 6, 6)
    ref_abs = np.stack([Ta[..., 3, 4], Ta[..., 2, 0], Ta[..., 3, 0]], axis=-1)
    ea = _rel(pabs, ref_abs)
    print(f'{tag} mixed absorbing entries vs float64 expm: max rel {ea.max():.2e}')
    assert ea.max() <= 1e-5, ea.max()
    Tt = np.stack([scipy.linalg.expm(q) for q in golden[f'expm__Qtm_{tag}'].astype(np.float64)])
    et = _rel(cum_tm, np.cumsum(Tt, axis=-1))
    assert et.max() <= 1e-5, et.max()


def test_tables_follow_dt(engine):
    """dt enters as Q dt: the table at dt = 0.5 ms is the square root step of dt = 1 ms."""
    topo, d, pCa, dd = _setup('4.5_14.0')
    _, c1, _ = engine.transition_tables(topo, d.param_row(), pCa, dd, 1.0, 'mixed')
    _, ch, _ = engine.transition_tables(topo, d.param_row(), pCa, dd, 0.5, 'mixed')
    P1 = np.diff(np.concatenate([np.zeros(c1.shape[:-1] + (1,)), c1], axis=-1), axis=-1)
    Ph = np.diff(np.concatenate([np.zeros(ch.shape[:-1] + (1,)), ch], axis=-1), axis=-1)
    assert np.abs(Ph @ Ph - P1).max() < 1e-5
