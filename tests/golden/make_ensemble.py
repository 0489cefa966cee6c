"""Generate the 64-seed ensemble fixture by running the reference's own ``run()``.

TEST INFRASTRUCTURE.  Runs ``multifil_jax.simulation.run`` (the reference
checkout named by ``MULTIFIL_REF``) under the NumPy JAX stand-in in
``jaxshim/`` for the 2x2 skeletal lattice at pCa 4.5, z_line 900 nm, 100 ms,
``replicates=64``, ``rng_seed=0`` (keys ``split(PRNGKey(0), 64)``), and writes
``ensemble.npz`` next to this file: the 64 axial-force traces.  The GPU test
(``tests/test_gpu_ensemble.py``) checks that the engine's ensemble mean lies
inside the reference ensemble's 95 % interval.
Usage: ``python tests/golden/make_ensemble.py``.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refload  # noqa: E402

CASE = dict(nrows=2, ncols=2, pCa=4.5, z_line=900.0, duration_ms=100, replicates=64, rng_seed=0)


def main(out_path=os.path.join(HERE, 'ensemble.npz')):
    R = refload.load()
    rs, rd = R.params.get_skeletal_params()
    topo = R.geo.SarcTopology.create(nrows=CASE['nrows'], ncols=CASE['ncols'], static_params=rs, dynamic_params=rd)
    t0 = time.time()
    res = R.sim.run(topo, duration_ms=CASE['duration_ms'], pCa=CASE['pCa'], z_line=CASE['z_line'],
                    replicates=CASE['replicates'], dynamic_params=rd, static_params=rs, rng_seed=CASE['rng_seed'])
    force = np.asarray(res.metrics['axial_force'], np.float32).reshape(CASE['replicates'], -1)
    np.savez_compressed(out_path, axial_force=force, **{k: np.asarray(v) for k, v in CASE.items()})
    print(f"wrote {out_path}: {force.shape} in {time.time() - t0:.0f} s")


if __name__ == '__main__':
    main()
