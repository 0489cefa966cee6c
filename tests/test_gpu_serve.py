"""Continuous batching: every served result equals the same condition run alone."""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params, get_cardiac_params
from multifil_jax_b200.serve import SimulationServer
from multifil_jax_b200.engine import EngineError, MF_FLAG_PRECISE
from multifil_jax_b200.simulation import METRIC_KEYS
from oracle import prng
from tests.gpu_helpers import run_engine

pytestmark = pytest.mark.gpu


def _requests(n, seed=1, lo=1, hi=3):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        r, c = rng.integers(lo, hi + 1, 2)
        preset = get_skeletal_params() if rng.random() < 0.5 else get_cardiac_params()
        out.append(dict(topo=SarcTopology.create(int(r), int(c), *preset), params=preset[1],
                        pCa=float(rng.uniform(4, 7)), z=float(rng.uniform(850, 1000)),
                        dur=float(rng.integers(10, 60)), key=prng.split(prng.PRNGKey(1000 + i), 1)[0]))
    return out


def _alone(engine, q, precision='mixed'):
    T = int(q['dur'])
    res = run_engine(engine, q['topo'], q['params'].param_row()[None], np.full((1, T), q['z']),
                     np.full((1, T), q['pCa']), np.full((1, T), 14.0), q['key'][None],
                     flags=MF_FLAG_PRECISE if precision == 'mixed' else 0)
    return res['metrics'][0]


@pytest.mark.parametrize('precision', ['mixed', 'float32'])
def test_served_equals_alone_with_late_arrivals(engine, precision):
    reqs = _requests(12)
    with SimulationServer(mem_budget=256 << 20, chunk_steps=7, precision=precision) as srv:
        ids = [srv.submit(q['topo'], q['params'], q['pCa'], q['z'], q['dur'], q['key']) for q in reqs[:6]]
        srv.step(2)  # the first six are on the GPU when the rest arrive
        ids += [srv.submit(q['topo'], q['params'], q['pCa'], q['z'], q['dur'], q['key']) for q in reqs[6:]]
        srv.drain()
        for rid, q in zip(ids, reqs):
            r = srv.poll(rid)
            assert r is not None and r.latency_s >= 0
            ref = _alone(engine, q, precision)
            got = np.stack([r.metrics[k].astype(np.float32) for k in METRIC_KEYS])
            assert np.array_equal(got, ref), q


def test_admission_by_memory_budget(engine):
    reqs = _requests(8, seed=3, lo=3, hi=4)
    # a 1 MB budget holds only a few 3x3..4x4 requests at a time; all complete
    with SimulationServer(mem_budget=1 << 20, chunk_steps=10) as srv:
        ids = [srv.submit(q['topo'], q['params'], q['pCa'], q['z'], q['dur'], q['key']) for q in reqs]
        a, q = srv.step(1)
        assert q > 0  # not everything fit at once
        srv.drain()
        for rid, qq in zip(ids, reqs):
            r = srv.poll(rid)
            assert np.array_equal(np.stack([r.metrics[k].astype(np.float32) for k in METRIC_KEYS]), _alone(engine, qq))
        # a request larger than the whole budget is refused up front
        big = SarcTopology.create(6, 6)
        with pytest.raises(EngineError):
            srv.submit(big, get_skeletal_params()[1], 4.5, 900.0, 20000.0, (0, 0))


def test_cancel_and_busy(engine):
    reqs = _requests(3, seed=4)
    with SimulationServer(mem_budget=64 << 20, chunk_steps=5) as srv:
        ids = [srv.submit(q['topo'], q['params'], q['pCa'], q['z'], 50.0, q['key']) for q in reqs]
        assert srv.poll(ids[0]) is None  # still queued
        srv.step(1)
        srv.cancel(ids[1])
        srv.drain()
        assert srv.poll(ids[0]) is not None and srv.poll(ids[2]) is not None


def test_served_insect_lattice_equals_alone(engine):
    """An insect flight muscle request (160-site thin filaments, four heads
    per crown, 512-thread CTAs) served beside vertebrate ones equals it alone."""
    from multifil_jax_b200 import get_lethocerus_params
    s, d = get_lethocerus_params()
    ifm = dict(topo=SarcTopology.create(2, 2, s, d), params=d, pCa=4.5, z=1550.0, dur=20.0,
               key=prng.split(prng.PRNGKey(77), 1)[0])
    reqs = _requests(3, seed=5) + [ifm]
    with SimulationServer(mem_budget=256 << 20, chunk_steps=6, precision='mixed') as srv:
        ids = [srv.submit(q['topo'], q['params'], q['pCa'], q['z'], q['dur'], q['key']) for q in reqs]
        srv.drain()
        for rid, q in zip(ids, reqs):
            r = srv.poll(rid)
            got = np.stack([r.metrics[k].astype(np.float32) for k in METRIC_KEYS])
            assert np.array_equal(got, _alone(engine, q)), q['topo']
