"""Threefry-2x32 counter-based PRNG and the ``jax.random`` layering on top of it.

TEST INFRASTRUCTURE (oracle).  Third-party algorithm, not in the reference
tree: the reference draws all randomness through ``jax.random``
(``simulation.py:1032,1043``; ``timestep.py:120,125``;
``kernels/transitions.py:615-616,1160-1161``), pinned at ``jax>=0.4.25``
(``pyproject.toml:9-12``; docs test 0.9.x).

* Hash: Threefry-2x32 with 20 rounds (Salmon, Moraes, Dror, Shaw, "Parallel
  Random Numbers: As Easy as 1, 2, 3", SC'11), rotation constants
  (13,15,26,6)/(17,29,16,24), key-schedule parity 0x1BD11BDA, key injection
  every 4 rounds with the injection counter added to word 1.
* ``PRNGKey(seed)`` -> ``[seed >> 32, seed & 0xffffffff]`` as uint32.
* Partitionable layout (JAX >= 0.5 default): ``split(k, n)[i] = H(k, (0, i))``
  and ``random_bits(k, (n,))[i] = H(k, (0, i)).x0 ^ H(k, (0, i)).x1``.
* Original layout (older JAX): counters ``iota(2n)`` are cut in two halves
  ``x0 = c[:h], x1 = c[h:]``, hashed pairwise and concatenated.
* ``uniform`` float32: ``bitcast((bits >> 9) | 0x3f800000) - 1``; float64 uses
  64-bit draws ``(x0 << 32) | x1`` shifted by 12.
"""
from __future__ import annotations

import numpy as np

_ROT = ((13, 15, 26, 6), (17, 29, 16, 24))
_PARITY = np.uint32(0x1BD11BDA)

PARTITIONABLE = True  # JAX >= 0.5 default; set False for the original layout


def _rotl(v, r):
    return ((v << np.uint32(r)) | (v >> np.uint32(32 - r))).astype(np.uint32)


def threefry2x32(k0, k1, x0, x1):
    """Vectorised Threefry-2x32-20 hash of counters (x0, x1) under key (k0, k1)."""
    with np.errstate(over='ignore'):
        k0 = np.asarray(k0, dtype=np.uint32)
        k1 = np.asarray(k1, dtype=np.uint32)
        ks = (k0, k1, (k0 ^ k1 ^ _PARITY).astype(np.uint32))
        a = (np.asarray(x0, dtype=np.uint32) + ks[0]).astype(np.uint32)
        b = (np.asarray(x1, dtype=np.uint32) + ks[1]).astype(np.uint32)
        for g in range(5):
            for r in _ROT[g % 2]:
                a = (a + b).astype(np.uint32)
                b = _rotl(b, r)
                b = (b ^ a).astype(np.uint32)
            a = (a + ks[(g + 1) % 3]).astype(np.uint32)
            b = (b + ks[(g + 2) % 3] + np.uint32(g + 1)).astype(np.uint32)
    return a, b


def PRNGKey(seed: int) -> np.ndarray:
    s = int(seed)
    return np.array([(s >> 32) & 0xFFFFFFFF if s >= 0 else 0, s & 0xFFFFFFFF], dtype=np.uint32)


def _hash_halves(key, counts):
    """Original-layout helper: the reference ``threefry_2x32(key, count)``."""
    counts = np.asarray(counts, dtype=np.uint32).ravel()
    odd = counts.size % 2
    if odd:
        counts = np.concatenate([counts, np.zeros(1, np.uint32)])
    h = counts.size // 2
    y0, y1 = threefry2x32(key[0], key[1], counts[:h], counts[h:])
    out = np.concatenate([y0, y1])
    return out[:-1] if odd else out


def split(key, num: int = 2, partitionable: bool | None = None) -> np.ndarray:
    key = np.asarray(key, dtype=np.uint32)
    part = PARTITIONABLE if partitionable is None else partitionable
    if part:
        i = np.arange(num, dtype=np.uint32)
        y0, y1 = threefry2x32(key[0], key[1], np.zeros(num, np.uint32), i)
        return np.stack([y0, y1], axis=1)
    return _hash_halves(key, np.arange(2 * num, dtype=np.uint32)).reshape(num, 2)


def random_bits32(key, n: int, partitionable: bool | None = None) -> np.ndarray:
    key = np.asarray(key, dtype=np.uint32)
    part = PARTITIONABLE if partitionable is None else partitionable
    if part:
        y0, y1 = threefry2x32(key[0], key[1], np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32))
        return (y0 ^ y1).astype(np.uint32)
    return _hash_halves(key, np.arange(n, dtype=np.uint32))


def random_bits64(key, n: int, partitionable: bool | None = None) -> np.ndarray:
    key = np.asarray(key, dtype=np.uint32)
    part = PARTITIONABLE if partitionable is None else partitionable
    if part:
        y0, y1 = threefry2x32(key[0], key[1], np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32))
        return (y0.astype(np.uint64) << np.uint64(32)) | y1.astype(np.uint64)
    bits = _hash_halves(key, np.arange(2 * n, dtype=np.uint32))
    hi, lo = bits[:n], bits[n:]
    return (hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)


def uniform(key, n: int, dtype=np.float32, partitionable: bool | None = None) -> np.ndarray:
    if np.dtype(dtype) == np.float32:
        bits = random_bits32(key, n, partitionable)
        f = ((bits >> np.uint32(9)) | np.uint32(0x3F800000)).view(np.float32) - np.float32(1.0)
        return np.maximum(np.float32(0.0), f).astype(np.float32)
    bits = random_bits64(key, n, partitionable)
    f = ((bits >> np.uint64(12)) | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.0
    return np.maximum(0.0, f)


def step_uniforms(key, n_sites_total: int, n_xb_total: int, dtype=np.float32,
                  partitionable: bool | None = None):
    """The draws of one reference timestep and the carried key.

    ``timestep.py:120,125`` and ``transitions.py:615-616,1160-1161``:
    k, thin_k = split(k); _, sub = split(thin_k); u_thin = uniform(sub, sites)
    k, thick_k = split(k); _, sub = split(thick_k); u_xb = uniform(sub, xbs)
    """
    k1, thin_k = split(key, 2, partitionable)
    sub_t = split(thin_k, 2, partitionable)[1]
    u_thin = uniform(sub_t, n_sites_total, dtype, partitionable)
    k2, thick_k = split(k1, 2, partitionable)
    sub_x = split(thick_k, 2, partitionable)[1]
    u_xb = uniform(sub_x, n_xb_total, dtype, partitionable)
    return u_thin, u_xb, k2
