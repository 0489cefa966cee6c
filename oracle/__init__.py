"""CPU oracle for the multifil_jax per-timestep hot path -- TEST INFRASTRUCTURE ONLY.

A NumPy restatement of the reference algorithm (travistune3/multifil_jax), used
exclusively by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
``cpu_baseline`` / ``--impl reference`` legs, and only as the checker or the
timed CPU baseline.  The product package ``multifil_jax_b200`` never imports,
links or calls anything here; its CUDA path fails loudly when its extension
is missing.

Modules, each citing the reference file:line it follows:
  prng      -- Threefry-2x32 and the jax.random key/uniform layering
  physics   -- rate laws, rate matrices, Pade expm, nearest sites, forces, JVPs
  step      -- one timestep (kinetics + Newton-CG equilibrium) and the metrics
  run       -- the run() batch/scan driver

Pinning: the topology and the whole timestep are checked against fixtures
produced by running the reference's own Python source under a NumPy-backed
JAX stand-in (``tests/golden/make_golden.py``).  The Threefry hash is checked
against the published Random123 known-answer vectors, and the jax.random key
split / uniform layering against outputs of JAX itself for key 0 in both
counter layouts (``tests/test_prng.py``): the partitionable layout of
JAX >= 0.5 (the default here) and the original one.  What stays unpinned is
JAX's own arithmetic under the stand-in (``jvp``/``grad``, the reassociation
of ``associative_scan``): the fixtures were made without JAX.
"""
