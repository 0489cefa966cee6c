"""Threefry-2x32 (published Random123 answers) and the jax.random layering, host side."""
import numpy as np
import pytest

from oracle import prng

# Random123 known-answer vectors for threefry2x32_20: (key, counter) -> output
KAT = [((0x0, 0x0), (0x0, 0x0), (0x6b200159, 0x99ba4efe)),
       ((0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff), (0x1cb996fc, 0xbb002be7)),
       ((0x13198a2e, 0x03707344), (0x243f6a88, 0x85a308d3), (0xc4923a9c, 0x483df7a0))]


@pytest.mark.parametrize('key,ctr,out', KAT)
def test_oracle_threefry_kat(key, ctr, out):
    a, b = prng.threefry2x32(np.uint32(key[0]), np.uint32(key[1]), np.uint32(ctr[0]), np.uint32(ctr[1]))
    assert (int(a), int(b)) == out


def test_prngkey_layout():
    assert prng.PRNGKey(0).tolist() == [0, 0]
    assert prng.PRNGKey(42).tolist() == [0, 42]


@pytest.mark.parametrize('part', [True, False])
def test_library_host_prng_matches_oracle(part):
    from multifil_jax_b200.engine import load_library, prng_split, prng_key
    lib = load_library()
    for seed, n in [(0, 1), (0, 256), (7, 3), (1000, 513)]:
        got = prng_split(prng_key(seed), n, partitionable=part)
        ref = prng.split(prng.PRNGKey(seed), n, partitionable=part)
        assert np.array_equal(got, ref)
    for n in (1, 5, 624, 720):
        u = np.zeros(n, np.float32)
        lib.mf_prng_uniform(123, 456, n, 1 if part else 0, u.ctypes.data)
        assert np.array_equal(u, prng.uniform(np.array([123, 456], np.uint32), n, partitionable=part))


def test_uniform_range_and_layering():
    u = prng.uniform(prng.PRNGKey(0), 10000)
    assert u.dtype == np.float32 and u.min() >= 0 and u.max() < 1
    assert abs(u.mean() - 0.5) < 0.02
    # one step draws: four splits, site and head uniforms, carried key
    ut, ux, k = prng.step_uniforms(prng.PRNGKey(3), 720, 624)
    assert ut.shape == (720,) and ux.shape == (624,) and k.shape == (2,)
    k1, tk = prng.split(prng.PRNGKey(3))
    assert np.array_equal(ut, prng.uniform(prng.split(tk)[1], 720))
