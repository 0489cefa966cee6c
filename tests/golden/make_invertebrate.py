"""Generate the invertebrate / superlattice / legacy-face fixtures from the reference source.

TEST INFRASTRUCTURE.  Like ``make_golden.py``: runs ``multifil_jax`` (the
reference checkout named by ``MULTIFIL_REF``) under the NumPy JAX stand-in in
``jaxshim/`` and writes ``invertebrate.npz`` next to this file:

* ``topo_<name>__<field>``  every SarcTopology array of the lattices in
  ``LATTICES`` (SarcTopology.create, core/sarc_geometry.py:379-645 with the
  edge-lattice, registration, superlattice and legacy branches);
* ``run_<name>__<metric>``  the 52 metrics of short ``simulation.run`` calls
  on those lattices (``RUNS``).

Usage: ``MULTIFIL_REF=<checkout> python tests/golden/make_invertebrate.py``.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refload  # noqa: E402
from make_golden import TOPO_FIELDS  # noqa: E402

# name: (nrows, ncols, preset, StaticParams overrides)
LATTICES = {
    'leth_2x2': (2, 2, 'lethocerus', {}),
    'leth_4x2': (4, 2, 'lethocerus', {}),
    'dros_2x3': (2, 3, 'drosophila', {}),
    'legacy_2x2': (2, 2, 'skeletal', {'legacy_crown_geometry': True}),
    'vert4_2x2': (2, 2, 'skeletal', {'n_xb_per_crown': 4, 'crown_rotation_deg': 33.75}),
}

# name: (lattice, run kwargs)
RUNS = {
    'leth_2x2': ('leth_2x2', dict(pCa=4.5, z_line=1550.0, duration_ms=10)),
    'dros_2x3': ('dros_2x3', dict(pCa=5.0, z_line=1525.0, duration_ms=6)),
    'legacy_2x2': ('legacy_2x2', dict(pCa=4.5, z_line=900.0, duration_ms=12)),
}


def params_of(R, preset, overrides):
    s, d = {'lethocerus': R.params.get_lethocerus_params, 'drosophila': R.params.get_drosophila_params,
            'skeletal': R.params.get_skeletal_params}[preset]()
    return (s.replace(**overrides) if overrides else s), d


def main(out_path=os.path.join(HERE, 'invertebrate.npz')):
    R = refload.load()
    data = {}
    topos = {}
    for name, (nr, nc, preset, ov) in LATTICES.items():
        s, d = params_of(R, preset, ov)
        t = R.geo.SarcTopology.create(nrows=nr, ncols=nc, static_params=s, dynamic_params=d)
        topos[name] = (t, s, d)
        for f in TOPO_FIELDS:
            data[f'topo_{name}__{f}'] = np.asarray(getattr(t, f))
        data[f'topo_{name}__ints'] = np.array([t.n_thick, t.n_crowns, t.n_thin, t.n_sites, t.n_titin,
                                               t.n_xb_per_crown, t.n_faces_per_thin, t.max_sites_per_face,
                                               t.total_xbs, t.n_xb_bins])
        print(name, t.n_thick, t.n_thin, t.n_sites, t.total_xbs)
    for name, (lat, kw) in RUNS.items():
        t, s, d = topos[lat]
        res = R.sim.run(t, dynamic_params=d, static_params=s, rng_seed=0, **kw)
        for k, v in res.metrics.items():
            data[f'run_{name}__{k}'] = np.asarray(v)
        data[f'run_{name}__rng_key'] = np.asarray(res.rng_key)
        print(name, np.asarray(res.metrics['axial_force'])[..., :4])
    np.savez_compressed(out_path, **data)
    print(f'wrote {out_path}: {len(data)} arrays, {os.path.getsize(out_path) / 1e3:.0f} kB')


if __name__ == '__main__':
    main()
