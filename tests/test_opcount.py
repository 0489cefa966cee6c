"""The op counter of the oracle, and the counts bench.py uses for its roofline."""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, get_skeletal_params
from oracle import opcount


def test_counter_counts_element_operations():
    counts = {}
    opcount._state['counts'] = counts = __import__('collections').defaultdict(
        lambda: __import__('collections').defaultdict(int))
    try:
        with opcount.phase('x'):
            a = opcount._wrap(np.ones(10, np.float32))
            b = a * 2.0 + a                      # 10 mul + 10 add
            np.sum(b)                            # 9 adds
            np.exp(a)                            # 10 sfu
            m = opcount._wrap(np.ones((3, 4), np.float32))
            m @ np.ones((4, 5), np.float32)      # 2 * 3 * 5 * 4
            out = np.zeros(4, np.float32)
            np.add.at(out, np.array([0, 1, 1]), a[:3])  # 3 adds
            (a > 0.5).sum()                      # integer work: not counted
    finally:
        opcount._state['counts'] = None
    assert counts['x']['flops'] == 10 + 10 + 9 + 120 + 3
    assert counts['x']['sfu'] == 10


def test_expm_flops_formula():
    # n = 6, s = 0: norm 71, scale 36, 4 products 1584, sums 288, LU 305, back 216, renorm 66
    assert opcount.expm_flops(6, [0]) == 2566
    assert opcount.expm_flops(6, [0, 3]) == 2 * 2566 + 3 * (2 * 216 - 36)


def test_bench_roofline_counts_are_current():
    """bench.py's 2x2 per-unit counts equal a fresh op-counting run."""
    import bench
    s, d = get_skeletal_params()
    u = opcount.unit_counts(SarcTopology.create(2, 2, s, d), d.param_row())
    for k, v in bench.OPCOUNT_2X2.items():
        assert u[k] == pytest.approx(v, rel=1e-9), k
