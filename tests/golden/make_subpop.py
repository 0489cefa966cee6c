"""Generate the subpopulation fixtures by running the reference's own Python source.

TEST INFRASTRUCTURE.  Like ``make_golden.py``: runs ``multifil_jax`` (the
reference checkout named by ``MULTIFIL_REF``) under the NumPy JAX stand-in in
``jaxshim/`` and writes ``subpop.npz`` next to this file:

* ``run_<case>__<metric>``  the 52 metrics of ``simulation.run(...,
  subpopulation=...)`` for the cases in ``CASES`` (mean field, random and
  C-zone populations; a swept list of mean-field fractions; dynamic spacing);
* ``masks_random__xb|tm``   ``generate_random_masks_batch`` labels
  (core/subpopulation.py:213-253) for seed 3, fractions 0.3 / 0.6, 2x2;
* ``masks_czone__xb|tm``    the C-zone labels of a 2x2 lattice with a tm_*
  scale (core/subpopulation.py:179-210).

Usage: ``MULTIFIL_REF=<checkout> python tests/golden/make_subpop.py`` (about a minute).
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refload  # noqa: E402

# name: (nrows, ncols, preset, subpopulation spec, run kwargs).  The spec is
# (constructor, args, kwargs) of the reference's Subpopulation; 'sweep' is a
# list of such specs (a sweep axis).
CASES = {
    'mf_1x1': (1, 1, 'skeletal', ('mean_field', (0.5,), dict(xb_r34_coeff=2.0, tm_k_01=0.5)),
               dict(pCa=4.5, z_line=900.0, duration_ms=25)),
    'mfxb_2x2': (2, 2, 'skeletal', ('mean_field', (0.3,), dict(xb_r01_coeff=2.5, xb_r23_coeff=0.5)),
                 dict(pCa=5.0, z_line=900.0, duration_ms=15)),
    'rand_2x2': (2, 2, 'skeletal', ('random', (0.3,), dict(seed=3, xb_r01_coeff=3.0, tm_J_C=2.0)),
                 dict(pCa=5.0, z_line=900.0, duration_ms=15, replicates=2)),
    'czone_2x2': (2, 2, 'cardiac', ('c_zone', (), dict(xb_r23_coeff=0.5)),
                  dict(pCa=4.5, z_line=900.0, duration_ms=15)),
    'czone_tm_1x1': (1, 1, 'skeletal', ('c_zone', (), dict(xb_r12_coeff=2.0, tm_k_12=1.5)),
                     dict(pCa=5.5, z_line=950.0, duration_ms=15)),
    'sweep_mf_1x1': (1, 1, 'skeletal', [('mean_field', (f,), dict(xb_r34_coeff=3.0)) for f in (0.0, 0.5, 1.0)],
                     dict(pCa=4.5, z_line=900.0, duration_ms=12)),
    'mf_dyn_1x1': (1, 1, 'skeletal', ('mean_field', (0.5,), dict(xb_r01_coeff=2.0, tm_k_01=0.7)),
                   dict(pCa=4.5, z_line=950.0, duration_ms=12, K_lat=5.0, nu=0.5)),
}


def build(SP, topo, spec):
    ctor, args, kw = spec
    if ctor == 'c_zone':
        return SP.Subpopulation.c_zone(topo, *args, **kw)
    return getattr(SP.Subpopulation, ctor)(*args, **kw)


def main(out_path=os.path.join(HERE, 'subpop.npz')):
    R = refload.load()
    SP = importlib.import_module('multifil_jax.core.subpopulation')
    data = {}
    rs, rd = R.params.get_skeletal_params()
    _, cd = R.params.get_cardiac_params()
    for name, (nr, nc, preset, spec, kw) in CASES.items():
        d = cd if preset == 'cardiac' else rd
        topo = R.geo.SarcTopology.create(nrows=nr, ncols=nc, static_params=rs, dynamic_params=d)
        sub = [build(SP, topo, s) for s in spec] if isinstance(spec, list) else build(SP, topo, spec)
        res = R.sim.run(topo, dynamic_params=d, static_params=rs, rng_seed=0, subpopulation=sub, **kw)
        for k, v in res.metrics.items():
            data[f'run_{name}__{k}'] = np.asarray(v)
        data[f'run_{name}__rng_key'] = np.asarray(res.rng_key)
        print(name, np.asarray(res.metrics['axial_force']).shape)
    t22 = R.geo.SarcTopology.create(nrows=2, ncols=2, static_params=rs, dynamic_params=rd)
    xb, tm = SP.generate_random_masks_batch(3, np.asarray([0.3, 0.6], np.float32), t22, 2)
    data['masks_random__xb'] = np.asarray(xb)
    data['masks_random__tm'] = np.asarray(tm)
    cz = SP.Subpopulation.c_zone(t22, tm_k_01=2.0, xb_r01_coeff=2.0)
    data['masks_czone__xb'] = np.asarray(cz.xb_mask)
    data['masks_czone__tm'] = np.asarray(cz.tm_mask)
    data['masks_czone__fractions'] = np.asarray(cz.fractions)
    np.savez_compressed(out_path, **data)
    print(f'wrote {out_path}: {len(data)} arrays, {os.path.getsize(out_path) / 1e3:.0f} kB')


if __name__ == '__main__':
    main()
