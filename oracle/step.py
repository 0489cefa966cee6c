"""One condition, one timestep: kinetics, Newton-CG equilibrium, 52 metrics.

TEST INFRASTRUCTURE (oracle).  Restates timestep.py:65-199,
kernels/solver.py:329-771, simulation.py:633-729 and metrics_fn.py:79-417 on
top of ``oracle.physics``.  ``Condition`` carries the scan state of one
simulation; ``run_condition`` is the per-condition body of ``_run_sim_kernel``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import physics as ph
from . import prng

METRIC_KEYS = (
    'axial_force', 'solver_residual', 'z_line', 'pCa', 'lattice_spacing',
    'n_bound', 'n_xb_drx', 'n_xb_loose', 'n_xb_tight_1', 'n_xb_tight_2', 'n_xb_free_2', 'n_xb_srx',
    'frac_xb_bound', 'frac_xb_drx', 'frac_xb_loose', 'frac_xb_tight_1', 'frac_xb_tight_2',
    'frac_xb_free_2', 'frac_xb_srx',
    'n_tm_state_0', 'n_tm_state_1', 'n_tm_state_2', 'n_tm_state_3',
    'frac_tm_state_0', 'frac_tm_state_1', 'frac_tm_state_2', 'frac_tm_state_3',
    'actin_permissiveness', 'frac_tm_state_2_overlap', 'frac_tm_state_3_overlap',
    'frac_tm_available_overlap', 'n_overlap_sites',
    'atp_consumed', 'newly_bound',
    'thick_displace_mean', 'thick_displace_max', 'thick_displace_min', 'thick_displace_std',
    'thin_displace_mean', 'thin_displace_max', 'thin_displace_min', 'thin_displace_std',
    'thick_energy_first_avg', 'thick_energy_first_delta_avg', 'titin_energy_avg', 'titin_energy_delta_avg',
    'work_thick', 'work_thick_mean', 'atp_expected_p', 'xb_tear_expected', 'work_per_atp', 'newton_iters')
assert len(METRIC_KEYS) == 52


@dataclass
class Condition:
    thick_x: np.ndarray
    thin_x: np.ndarray
    xb_state: np.ndarray
    xb_bound: np.ndarray
    xb_nearest: np.ndarray
    xb_dist: np.ndarray
    tm: np.ndarray
    thin_bound: np.ndarray

    def copy(self):
        return Condition(*[getattr(self, f).copy() for f in
                           ('thick_x', 'thin_x', 'xb_state', 'xb_bound', 'xb_nearest', 'xb_dist',
                            'tm', 'thin_bound')])


@dataclass
class Tables:
    """Per-step probability tables (depend on pCa, spacing and dt only)."""
    P_tm: np.ndarray
    P_xb: np.ndarray
    s_tm: np.ndarray = field(default=None)
    s_xb: np.ndarray = field(default=None)


def _pop_generators(gen, p, sp, family, dt):
    """Generators of one rate family with subpopulations (transitions.py:580-596,
    :957-976): the wild-type set when no population scales the family, the
    fraction-weighted sum sum_k f_k Q_k (mean field, Python ``sum`` order), or
    the K sets stacked on a leading axis (explicit labels)."""
    if sp is None or not sp[family]:
        return gen(p)
    Qk = [gen(ph.param_dict(r, dt)) for r in sp['rows']]
    if not sp['explicit']:
        f = np.asarray(sp['frac'], dtype=np.float32).astype(dt)
        return sum(f[k] * Qk[k] for k in range(len(Qk)))
    return np.stack(Qk)


def _expm_any(Q, with_s=False):
    """expm_pade6 over any leading shape (K stacked sets included)."""
    n = Q.shape[-1]
    r = ph.expm_pade6(Q.reshape(-1, n, n), with_s=with_s)
    if with_s:
        return r[0].reshape(Q.shape), r[1].reshape(Q.shape[:-2])
    return r.reshape(Q.shape)


def tables(topo, p, pCa, d, dt_ms, dt, sp=None):
    """Sampling tables at (pCa, d); with a subpopulation ``sp`` (see
    ``subpop_spec``) the blended or per-population sets."""
    Qt = _pop_generators(lambda q: ph.tm_Q27(q, dt(pCa), dt), p, sp, 'tm', dt)
    Qx = _pop_generators(lambda q: ph.xb_Q_bins(topo, q, dt(pCa), dt(d), dt), p, sp, 'xb', dt)
    P_tm, s_tm = _expm_any(Qt * dt(dt_ms), with_s=True)
    P_xb, s_xb = _expm_any(Qx * dt(dt_ms), with_s=True)
    return Tables(P_tm, P_xb, s_tm, s_xb)


def absorbing_table(topo, p, pCa, d, dt_ms, dt, sp=None):
    Qx = _pop_generators(lambda q: ph.xb_Q_bins(topo, q, dt(pCa), dt(d), dt), p, sp, 'xb', dt)
    return _expm_any(ph.absorbing(Qx) * dt(dt_ms))


def subpop_spec(rows, fractions, explicit, xb, tm, xb_label=None, tm_label=None):
    """One condition's subpopulation for the oracle: K parameter rows, the K
    fractions, which rate families the populations change, and the labels of
    the explicit modes."""
    return dict(rows=np.asarray(rows, np.float32), frac=np.asarray(fractions, np.float32), explicit=bool(explicit),
                xb=bool(xb), tm=bool(tm),
                xb_label=None if xb_label is None else np.asarray(xb_label, np.int64),
                tm_label=None if tm_label is None else np.asarray(tm_label, np.int64))


def _labels(sp, family):
    if sp is None or not sp['explicit'] or not sp[family]:
        return None
    return sp[family + '_label']


# ---------------------------------------------------------------------------
# Equilibrium solve (solver.py:329-771)
# ---------------------------------------------------------------------------

def tolerance(p, dt):
    return max(p['solver_tol'], max(p['thick_k'] * dt(1e-4), dt(ph.MIN_FLOAT32_TOLERANCE)))


def pcg(Av, M, b, n_cg):
    """6-step preconditioned CG from x0 = 0 (solver.py:329-366)."""
    dt = b.dtype.type
    r = b.copy()
    z = M(r)
    pv = z
    rz = np.dot(r, z)
    x = np.zeros_like(b)
    for _ in range(n_cg):
        Ap = Av(pv)
        pAp = np.dot(pv, Ap)
        alpha = rz / (pAp + dt(1e-30))
        x = x + alpha * pv
        r = r - alpha * Ap
        z = M(r)
        rz_new = np.dot(r, z)
        beta = rz_new / (rz + dt(1e-30))
        pv = z + beta * pv
        rz = rz_new
    return x


def solve_fixed(topo, p, c: Condition, z, ls, n_newton, n_cg, dt, precond):
    """Newton with max|F| > tol exit; non-finite steps zeroed (solver.py:369-495)."""
    fm = ph.ForceModel(topo, p, c.xb_state, c.xb_bound, z, dt)
    d = dt(ls)
    x = np.concatenate([c.thick_x.reshape(-1), c.thin_x.reshape(-1)]).astype(dt)
    tol = tolerance(p, dt)
    f = fm.residual(x, d)
    it = 0
    while np.max(np.abs(f)) > tol and it < n_newton:
        dx = pcg(lambda v: -fm.jvp(x, d, v), precond, f, n_cg)
        dx = np.where(np.isfinite(dx), dx, dt(0.0))
        x = x + dx
        f = fm.residual(x, d)
        it += 1
    xt, xn = fm.split(x)
    return xt.copy(), xn.copy(), np.max(np.abs(f)), it, d


def solve_dynamic(topo, p, c: Condition, z, d_init, K_lat, d_ref, n_newton, n_cg, dt, precond):
    """Augmented (n+1) Newton with the lattice spacing as an unknown (solver.py:599-656)."""
    fm = ph.ForceModel(topo, p, c.xb_state, c.xb_bound, z, dt)
    K = dt(K_lat)
    dref = dt(d_ref)
    x0 = np.concatenate([c.thick_x.reshape(-1), c.thin_x.reshape(-1)]).astype(dt)
    d0 = dt(d_init)
    J_dd = fm.J_dd(x0, d0, K)
    d_inv = dt(-1.0) / J_dd
    n = x0.shape[0]

    def R(xa):
        return np.concatenate([fm.residual(xa[:n], xa[n]), [fm.radial(xa[:n], xa[n], K, dref)]]).astype(dt)

    def Av(xa, va):
        ax, rd = fm.jvp(xa[:n], xa[n], va[:n], va[n], K)
        return -np.concatenate([ax, [rd]]).astype(dt)

    def M(va):
        return np.concatenate([precond(va[:n]), [d_inv * va[n]]]).astype(dt)

    tol = tolerance(p, dt)
    xa = np.concatenate([x0, [d0]]).astype(dt)
    f = R(xa)
    it = 0
    while np.max(np.abs(f)) > tol and it < n_newton:
        dx = pcg(lambda v: Av(xa, v), M, f, n_cg)
        dx = np.where(np.isfinite(dx), dx, dt(0.0))
        xa = xa + dx
        xa[n] = max(xa[n], dt(1.0))
        f = R(xa)
        it += 1
    xt, xn = fm.split(xa[:n])
    return xt.copy(), xn.copy(), np.max(np.abs(f)), it, xa[n]


# ---------------------------------------------------------------------------
# Initial state (state.py:191-262, simulation.py:633-642)
# ---------------------------------------------------------------------------

def initial_condition(topo, p, z0, n_newton, n_cg, dt, precond):
    c = Condition(
        thick_x=topo.crown_offsets.astype(dt).copy(),
        thin_x=(dt(z0) - topo.binding_offsets).astype(dt),
        xb_state=np.zeros(topo.total_xbs, np.int8),
        xb_bound=np.full(topo.total_xbs, -1, np.int32),
        xb_nearest=np.zeros(topo.total_xbs, np.int32),
        xb_dist=np.zeros((topo.total_xbs, 2), dt),
        tm=np.zeros((topo.n_thin, topo.n_sites), np.int8),
        thin_bound=np.full((topo.n_thin, topo.n_sites), -1, np.int32))
    c.xb_nearest, c.xb_dist = ph.nearest_sites(c.thick_x, c.thin_x, topo, p['lattice_spacing'], dt)
    xt, xn, _, _, _ = solve_fixed(topo, p, c, p['z_line'], p['lattice_spacing'], n_newton, n_cg, dt, precond)
    c.thick_x, c.thin_x = xt, xn
    return c


# ---------------------------------------------------------------------------
# Metrics (metrics_fn.py:79-417)
# ---------------------------------------------------------------------------

def metrics(topo, p, old: Condition, new: Condition, z, pCa, ls, pre_thick, force, resid, iters,
            P_abs, dt, thin_rest_cum, xb_labels=None):
    f32 = dt
    nx = f32(new.xb_state.size)
    nt = f32(new.tm.size)
    xb_new = new.xb_state
    xb_old = old.xb_state
    cnt = [f32(np.sum(xb_new == k)) for k in range(6)]
    n_bound = f32(np.sum((xb_new >= 1) & (xb_new <= 3)))
    tmc = [f32(np.sum(new.tm == k)) for k in range(4)]
    perm_mean = np.mean((new.tm == 3).astype(dt))
    near = topo.crown_offsets.min() - dt(13.0)
    far = topo.crown_offsets.max() + dt(13.0)
    om = (new.thin_x >= near) & (new.thin_x <= far) & (new.thin_x > 0.0)
    n_ov = f32(np.sum(om))
    n2 = f32(np.sum((new.tm == 2) & om))
    n3 = f32(np.sum((new.tm == 3) & om))
    atp = f32(np.sum((xb_old == 3) & ((xb_new == 4) | (xb_new == 0))))
    newly = f32(np.sum((xb_old == 0) & (xb_new == 1)))
    tdisp = (new.thick_x - topo.crown_offsets).reshape(-1)
    ndisp = (new.thin_x - thin_rest_cum).reshape(-1)
    k = p['thick_k']
    L0 = topo.crown_offsets[:, 0]
    e_new = f32(0.5) * k * (new.thick_x[:, 0] - L0) ** 2
    e_old = f32(0.5) * k * (old.thick_x[:, 0] - L0) ** 2
    a, b, r0 = p['titin_a'], p['titin_b'], p['titin_rest']

    def tit_e(xl):
        ad = z - xl
        L = np.sqrt(ad ** 2 + ls ** 2)
        return (a / b) * (np.exp(b * (L - r0)) - f32(1.0))
    te_new = tit_e(new.thick_x[:, -1])
    te_old = tit_e(old.thick_x[:, -1])
    dxm = new.thick_x - pre_thick
    work = force * np.mean(dxm)
    work_mean = work / f32(topo.n_thick * topo.n_crowns)
    # expected exits from the absorbing generator, on the pre-step geometry
    perm = ph.permissiveness(old.tm, old.xb_nearest, topo)
    key = ph.xb_bin_key(old.xb_dist[:, 0], perm, topo)
    Pk = P_abs[key] if xb_labels is None else P_abs[xb_labels, key]
    s_old = xb_old.astype(np.int32)
    atp_p = np.sum((s_old == 3).astype(dt) * Pk[:, 3, 4])
    tear = np.sum(((s_old == 2) | (s_old == 3)).astype(dt) * Pk[np.arange(s_old.size), s_old, 0])
    wpa = work / atp_p if atp_p > 0.01 else f32(0.0)
    vals = [force, resid, z, pCa, ls, n_bound, *cnt,
            n_bound / nx, *[c_ / nx for c_ in cnt],
            *tmc, *[c_ / nt for c_ in tmc], perm_mean,
            n2 / n_ov, n3 / n_ov, (n2 + n3) / n_ov, n_ov, atp, newly,
            np.mean(tdisp), np.max(tdisp), np.min(tdisp), np.std(tdisp),
            np.mean(ndisp), np.max(ndisp), np.min(ndisp), np.std(ndisp),
            np.mean(e_new), np.mean(e_new - e_old), np.mean(te_new), np.mean(te_new - te_old),
            work, work_mean, atp_p, tear, wpa, iters]
    return np.array(vals, dtype=np.float64)


# ---------------------------------------------------------------------------
# Timestep (timestep.py:65-199 + simulation.py:679-721)
# ---------------------------------------------------------------------------

def timestep(topo, p, c: Condition, z, pCa, ls_drv, dz, u_thin, u_xb, tab: Tables, n_newton, n_cg,
             dt, precond, dt_ms, K_lat=None, d_ref=None, P_abs=None, thin_rest_cum=None,
             want_metrics=True, tab_abs_fn=None, sp=None):
    """Advance one condition by one step; returns (new condition, metrics row, extras)."""
    old = c.copy()
    old.thin_x = (old.thin_x + dt(dz)).astype(dt)
    pre_thick = old.thick_x.copy()
    s = old.copy()
    # kinetics (timestep.py:97-129)
    s.xb_nearest, s.xb_dist = ph.nearest_sites(s.thick_x, s.thin_x, topo, dt(ls_drv), dt)
    s.tm = ph.thin_transitions(s.tm, s.thin_bound, tab.P_tm, topo, u_thin, labels=_labels(sp, 'tm'))
    s.xb_state, s.xb_bound, s.thin_bound = ph.thick_transitions(
        s.xb_state, s.xb_bound, s.thin_bound, s.xb_nearest, s.xb_dist[:, 0], s.tm, tab.P_xb, topo, u_xb,
        labels=_labels(sp, 'xb'))
    # mechanics
    if K_lat is None:
        xt, xn, res, it, new_ls = solve_fixed(topo, p, s, z, ls_drv, n_newton, n_cg, dt, precond)
    else:
        xt, xn, res, it, new_ls = solve_dynamic(topo, p, s, z, ls_drv, K_lat, d_ref, n_newton, n_cg, dt,
                                                precond)
    s.thick_x, s.thin_x = xt, xn
    force = np.sum((s.thick_x[:, 0] - topo.crown_offsets[:, 0]) * p['thick_k'])
    row = None
    if want_metrics:
        if P_abs is None:
            P_abs = tab_abs_fn(new_ls)
        row = metrics(topo, p, old, s, dt(z), dt(pCa), dt(new_ls), pre_thick, force, res, it, P_abs, dt,
                      thin_rest_cum, xb_labels=_labels(sp, 'xb'))
    return s, row, dict(force=force, residual=res, iters=it, ls=new_ls)


def thin_rest_cumsum(topo, dt):
    return ph.cumsum_jax(topo.binding_rests.astype(np.float32), axis=1).astype(dt)


def run_condition(topo, prow, z_tr, pCa_tr, ls_tr, key, dt_ms=1.0, n_newton=4, n_cg=6, dt=np.float32,
                  K_lat=None, nu=0.0, uniforms=None, record_states=False, partitionable=None,
                  hoist_tables=True, udtype=np.float32, subpop=None):
    """The per-condition body of ``_run_sim_kernel`` (simulation.py:633-729).

    Returns ``(metrics [52, T], info)``; ``info['uniforms']`` holds the draws
    used, ``info['states']`` per-step snapshots when ``record_states``.
    ``uniforms`` (list of (u_thin, u_xb)) replaces the PRNG draws.
    ``subpop`` (``subpop_spec``) runs the condition with mixed populations
    (simulation.py:658-676).
    """
    dt = np.dtype(dt).type
    p = ph.param_dict(prow, dt)
    precond = ph.Preconditioner(topo, p, dt)
    T = len(z_tr)
    z_tr = np.asarray(z_tr, dtype=dt)
    pCa_tr = np.asarray(pCa_tr, dtype=dt)
    ls_tr = np.asarray(ls_tr, dtype=dt)
    dz = np.concatenate([np.zeros(1, dt), np.diff(z_tr)]).astype(dt)
    c = initial_condition(topo, p, z_tr[0], n_newton, n_cg, dt, precond)
    thin_cum = thin_rest_cumsum(topo, dt)
    key = np.asarray(key, dtype=np.uint32)
    cur_ls = ls_tr[0]
    l0 = z_tr[0]
    out = np.zeros((52, T))
    used, states = [], []
    cache = {}

    def get_tab(pCa, d):
        k = (float(pCa), float(d))
        if not hoist_tables or k not in cache:
            cache.clear()
            cache[k] = tables(topo, p, pCa, d, dt_ms, dt, sp=subpop)
        return cache[k]
    abs_cache = {}

    def get_abs(pCa, d):
        k = (float(pCa), float(d))
        if not hoist_tables or k not in abs_cache:
            abs_cache.clear()
            abs_cache[k] = absorbing_table(topo, p, pCa, d, dt_ms, dt, sp=subpop)
        return abs_cache[k]

    for t in range(T):
        if uniforms is not None:
            u_thin, u_xb = uniforms[t]
        else:
            u_thin, u_xb, key = prng.step_uniforms(key, topo.n_sites_total, topo.total_xbs, udtype,
                                                    partitionable)
        used.append((u_thin, u_xb))
        if K_lat is None:
            ls_drv = ls_tr[t]
            d_ref = None
        else:
            ls_drv = cur_ls
            d_ref = ls_tr[t] * (l0 / z_tr[t]) ** dt(nu)
        tab = get_tab(pCa_tr[t], ls_drv)
        c, row, ex = timestep(topo, p, c, z_tr[t], pCa_tr[t], ls_drv, dz[t], u_thin.astype(dt),
                              u_xb.astype(dt), tab, n_newton, n_cg, dt, precond, dt_ms, K_lat=K_lat,
                              d_ref=d_ref, thin_rest_cum=thin_cum,
                              tab_abs_fn=lambda d_new, t_=t: get_abs(pCa_tr[t_], d_new), sp=subpop)
        out[:, t] = row
        cur_ls = ex['ls']
        if record_states:
            states.append(c.copy())
    return out, dict(uniforms=used, states=states, key=key)
