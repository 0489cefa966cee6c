"""SarcTopology restatement vs the reference builder's own output (golden fixtures)."""
import numpy as np
import pytest

from multifil_jax_b200 import SarcTopology, StaticParams, get_skeletal_params, get_cardiac_params
from multifil_jax_b200.topology import thin_rest_cumsum

SIZES = [(1, 1), (2, 2), (2, 3), (3, 1), (4, 4)]
INTS = ('n_thick', 'n_crowns', 'n_thin', 'n_sites', 'n_titin', 'n_xb_per_crown', 'n_faces_per_thin',
        'max_sites_per_face', 'total_xbs', 'n_xb_bins')


@pytest.mark.parametrize('nr,nc', SIZES)
def test_topology_bit_identical(golden, nr, nc):
    s, d = get_skeletal_params()
    t = SarcTopology.create(nr, nc, s, d)
    ints = golden[f'topo_{nr}x{nc}__ints']
    assert [getattr(t, k) for k in INTS] == list(ints)
    for key, ref in golden.items():
        if key.startswith(f'topo_{nr}x{nc}__') and not key.endswith('__ints'):
            f = key.split('__', 1)[1]
            mine = np.asarray(getattr(t, f))
            assert mine.dtype == ref.dtype, f
            assert mine.shape == ref.shape, f
            assert np.array_equal(mine, ref), f


def test_cardiac_geometry_equals_skeletal():
    a = SarcTopology.create(2, 2, *get_skeletal_params())
    b = SarcTopology.create(2, 2, *get_cardiac_params())
    for f in SarcTopology.ARRAY_FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f))


def test_known_sizes():
    # sizes of the lattices the benchmarks use (vertebrate, 52 crowns, 90 sites)
    expect = {(1, 1): (1, 4, 156), (2, 2): (4, 8, 624), (3, 3): (9, 24, 1404), (6, 6): (36, 72, 5616)}
    for (r, c), (nth, nthin, x) in expect.items():
        t = SarcTopology.create(r, c)
        assert (t.n_thick, t.n_thin, t.total_xbs) == (nth, nthin, x)
        assert t.n_sites == 90 and t.max_sites_per_face == 30


def test_bad_lattice_arguments_raise():
    with pytest.raises(ValueError):
        SarcTopology.create(2, 2, thick_starts=[1, 2])
    with pytest.raises(ValueError):
        SarcTopology.create(0, 2)


def test_thin_rest_cumsum_is_scan_order():
    t = SarcTopology.create(2, 2)
    c = thin_rest_cumsum(t)
    # same values as a running sum up to float32 reassociation, but not bitwise
    assert np.allclose(c, np.cumsum(t.binding_rests.astype(np.float64), axis=1), rtol=1e-6, atol=1e-3)
    assert c.dtype == np.float32
