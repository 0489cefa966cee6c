"""Generate golden fixtures by running the reference's own Python source.

TEST INFRASTRUCTURE.  Runs ``multifil_jax`` (the reference checkout named by
``MULTIFIL_REF``) under the NumPy JAX stand-in in ``jaxshim/`` and writes
``golden.npz`` next to this file:

* ``topo_RxC__<field>``   every SarcTopology array for a few lattice sizes
  (``SarcTopology.create``, sarc_geometry.py:379-645);
* ``expm__*``             the reference ``expm_pade6_batch`` on the 400
  crossbridge bins and 27 tropomyosin generators (transitions.py:99-190);
* ``run_<case>__<metric>`` the 52 metrics of ``simulation.run`` for short
  runs (fixed and dynamic lattice spacing, sweeps, traces, cardiac, x64);
* ``steps_2x2__*``        per-step integer state arrays and node positions
  from calling the reference ``timestep`` directly.

Randomness flows through ``jax.random`` -> the stand-in -> ``oracle.prng``, so
these fixtures pin everything except the jax.random layering itself.
Usage: ``python tests/golden/make_golden.py`` (about a minute).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import refload  # noqa: E402

TOPO_SIZES = [(1, 1), (2, 2), (2, 3), (3, 1), (4, 4)]
TOPO_FIELDS = ('xb_to_thin_id', 'xb_to_thin_face', 'xb_to_site_indices', 'xb_valid', 'thick_to_thin',
               'thin_to_thick', 'face_to_sites', 'n_sites_per_face', 'titin_connections', 'crown_offsets',
               'crown_rests', 'binding_offsets', 'binding_rests', 'tm_chains', 'thick_starts', 'thin_starts',
               'xb_bin_edges', 'xb_bin_centers', 'tm_prev_neighbor', 'tm_next_neighbor')

# name: (nrows, ncols, preset, run kwargs)
RUNS = {
    'skel_1x1': (1, 1, 'skeletal', dict(pCa=4.5, z_line=900.0, duration_ms=40)),
    'skel_2x2': (2, 2, 'skeletal', dict(pCa=4.5, z_line=900.0, duration_ms=40)),
    'card_2x2_z950': (2, 2, 'cardiac', dict(pCa=5.0, z_line=950.0, duration_ms=25)),
    'sweep_2x2': (2, 2, 'skeletal', dict(pCa=[4.0, 5.5, 7.0], z_line=900.0, duration_ms=12, replicates=2)),
    'dynls_1x1': (1, 1, 'skeletal', dict(pCa=4.5, z_line='ramp', duration_ms=20, K_lat=5.0, nu=0.5)),
    'dynls_2x2': (2, 2, 'skeletal', dict(pCa=4.5, z_line=950.0, duration_ms=12, K_lat=5.0, nu=0.5)),
    'sine_2x2': (2, 2, 'skeletal', dict(pCa=4.5, z_line='sine', duration_ms=30)),
    'poisson_1x1': (1, 1, 'skeletal', dict(pCa=5.0, z_line='ramp', duration_ms=15, nu=0.5)),
    'x64_2x2': (2, 2, 'skeletal', dict(pCa=4.5, z_line=900.0, duration_ms=12)),
}


def _trace(kind, n):
    t = np.arange(n, dtype=np.float64)
    if kind == 'ramp':
        return 900.0 + 0.5 * t
    if kind == 'sine':
        return 900.0 + 2.0 * np.sin(2 * np.pi * 50.0 * t / 1000.0)
    raise ValueError(kind)


def main(out_path=os.path.join(HERE, 'golden.npz')):
    R = refload.load()
    import jax
    data = {}
    rs, rd = R.params.get_skeletal_params()
    _, cd = R.params.get_cardiac_params()

    for nr, nc in TOPO_SIZES:
        t = R.geo.SarcTopology.create(nrows=nr, ncols=nc, static_params=rs, dynamic_params=rd)
        for f in TOPO_FIELDS:
            data[f'topo_{nr}x{nc}__{f}'] = np.asarray(getattr(t, f))
        data[f'topo_{nr}x{nc}__ints'] = np.array([t.n_thick, t.n_crowns, t.n_thin, t.n_sites, t.n_titin,
                                                  t.n_xb_per_crown, t.n_faces_per_thin,
                                                  t.max_sites_per_face, t.total_xbs, t.n_xb_bins])

    # expm on the crossbridge bin grid and the 27 tropomyosin generators
    t22 = R.geo.SarcTopology.create(nrows=2, ncols=2, static_params=rs, dynamic_params=rd)
    st = R.state.realize_state(t22, rd, 900.0, 4.5, 14.0)
    for pCa, d in [(4.5, 14.0), (6.0, 12.5)]:
        c = rd.copy(pCa=pCa, lattice_spacing=d)
        Q, _ = R.trans._build_xb_Q_bins(st, c, t22)
        tag = f'{pCa}_{d}'
        data[f'expm__Q_{tag}'] = np.asarray(Q)
        data[f'expm__P_{tag}'] = np.asarray(R.trans.expm_pade6_batch(Q * 1.0, t22.eye_6))
        Qa = Q.at[..., 4, :].set(0.0).at[..., 0, :].set(0.0)
        data[f'expm__Pabs_{tag}'] = np.asarray(R.trans.expm_pade6_batch(Qa * 1.0, t22.eye_6))
        ca = 10.0 ** (-c.pCa)
        Qt = R.trans._compute_unique_tm_Q_matrices(ca, c.tm_J_C, c.tm_J_M, c).reshape(27, 4, 4)
        data[f'expm__Qtm_{tag}'] = np.asarray(Qt)
        data[f'expm__Ptm_{tag}'] = np.asarray(R.trans.expm_pade6_batch(Qt * 1.0, t22.eye_4))

    # short runs through the public run()
    for name, (nr, nc, preset, kw) in RUNS.items():
        x64 = name.startswith('x64')
        jax.config.update('jax_enable_x64', x64)
        R2 = R
        if x64:
            rs2, rd2 = R.params.get_skeletal_params()
        else:
            rs2, rd2 = rs, (cd if preset == 'cardiac' else rd)
        topo = R2.geo.SarcTopology.create(nrows=nr, ncols=nc, static_params=rs2, dynamic_params=rd2)
        kw = dict(kw)
        n = int(kw['duration_ms'])
        if isinstance(kw.get('z_line'), str):
            kw['z_line'] = _trace(kw['z_line'], n)
        res = R2.sim.run(topo, dynamic_params=rd2, static_params=rs2, rng_seed=0, **kw)
        for k, v in res.metrics.items():
            data[f'run_{name}__{k}'] = np.asarray(v)
        data[f'run_{name}__lattice_spacing_trace'] = np.asarray(res.lattice_spacing)
        data[f'run_{name}__rng_key'] = np.asarray(res.rng_key)
        jax.config.update('jax_enable_x64', False)

    # per-step states through the reference timestep()
    topo = t22
    pp = R.state.build_preconditioner_params(topo.n_thick, topo.n_crowns, topo.n_thin, topo.n_sites,
                                             rd.thick_k, rd.thin_k)
    pre = R.solver.build_prefactored_preconditioner(pp)
    s0 = R.state.realize_state(topo, rd, 900.0, 4.5, 14.0)
    s0 = R.geometry.update_nearest_neighbors(s0, rd, topo)
    s0, _, _, _ = R.solver.solve_equilibrium(s0, rd, topo, n_cg_steps=6, n_newton_steps=4)
    key = jax.random.split(jax.random.PRNGKey(7), 1)[0]
    drivers = R.state.Drivers(pCa=np.float32(4.5), z_line=np.float32(900.0), lattice_spacing=np.float32(14.0))
    rec = {k: [] for k in ('xb_states', 'xb_bound_to', 'tm_states', 'thin_bound_to', 'thick_axial',
                           'thin_axial', 'residual', 'iters')}
    s = s0
    data['steps_2x2__init_thick_axial'] = np.asarray(s0.thick.axial)
    data['steps_2x2__init_thin_axial'] = np.asarray(s0.thin.axial)
    data['steps_2x2__key0'] = np.asarray(key)
    for _ in range(20):
        s, key, res_, _ls, it = R.timestep.timestep(s, rd, drivers, topo, key, dt=1.0, n_cg_steps=6,
                                                    n_newton_steps=4, precond_params=pp,
                                                    prefactored_precond=pre)
        rec['xb_states'].append(np.asarray(s.thick.xb_states).reshape(-1))
        rec['xb_bound_to'].append(np.asarray(s.thick.xb_bound_to).reshape(-1))
        rec['tm_states'].append(np.asarray(s.thin.tm_states))
        rec['thin_bound_to'].append(np.asarray(s.thin.bound_to))
        rec['thick_axial'].append(np.asarray(s.thick.axial))
        rec['thin_axial'].append(np.asarray(s.thin.axial))
        rec['residual'].append(float(res_))
        rec['iters'].append(int(it))
    for k, v in rec.items():
        data[f'steps_2x2__{k}'] = np.asarray(v)

    np.savez_compressed(out_path, **data)
    print(f'wrote {out_path}: {len(data)} arrays, {os.path.getsize(out_path) / 1e3:.0f} kB')


if __name__ == '__main__':
    main()
