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


# Outputs of jax.random itself for key 0, as JAX prints them (public JAX
# documentation and examples): split(PRNGKey(0)) and uniform(PRNGKey(0)) in
# the original counter layout (jax_threefry_partitionable=False, the default
# before JAX 0.5; the "Sharp Bits" notebook prints this split), and the same
# calls in the partitionable layout (the default from JAX 0.5 on).  The first
# partitionable pair is also H(key=(0,0), counter=(0,0)), the first Random123
# answer above, which is what the partitionable split hashes.
JAX_SPLIT0 = {False: [[4146024105, 967050713], [2718843009, 1272950319]],
              True: [[1797259609, 2579123966], [928981903, 3453687069]]}
JAX_UNIFORM0 = {False: 0.41845703, True: 0.947667}


@pytest.mark.parametrize('part', [False, True])
def test_jax_known_answers_oracle(part):
    assert prng.split(prng.PRNGKey(0), 2, partitionable=part).tolist() == JAX_SPLIT0[part]
    u = prng.uniform(prng.PRNGKey(0), 1, partitionable=part)
    assert u.dtype == np.float32 and abs(float(u[0]) - JAX_UNIFORM0[part]) < 5e-7


@pytest.mark.parametrize('part', [False, True])
def test_jax_known_answers_library(part):
    """The library's own jax.random layer (the code the kernel runs, compiled
    for the host) gives the same answers."""
    from multifil_jax_b200.engine import load_library, prng_split, prng_key
    lib = load_library()
    assert prng_split(prng_key(0), 2, partitionable=part).tolist() == JAX_SPLIT0[part]
    u = np.zeros(1, np.float32)
    assert lib.mf_prng_uniform(0, 0, 1, 1 if part else 0, u.ctypes.data) == 0
    assert abs(float(u[0]) - JAX_UNIFORM0[part]) < 5e-7
