"""Helpers that drive the oracle the way run() drives the CUDA engine (test-only)."""
import numpy as np

from oracle import step as OS


def plan_subpop(plan, b):
    """The oracle's subpopulation spec of condition b of a BatchPlan (None without one)."""
    sp = plan.subpop
    if sp is None:
        return None
    return OS.subpop_spec(sp.rows[b], sp.fractions[b], sp.explicit, sp.xb, sp.tm,
                          None if sp.xb_label is None else sp.xb_label[b],
                          None if sp.tm_label is None else sp.tm_label[b])


def oracle_plan(topo, plan, static, dtype=np.float32, udtype=np.float32, params=None, **kw):
    """Metrics [B, 52, T] of every condition of a BatchPlan, computed by the oracle."""
    B, T = plan.total, plan.n_steps
    out = np.zeros((B, 52, T))
    infos = []
    for b in range(B):
        row = plan.params[b] if params is None else params[b]
        K = float(plan.K_lat[b]) if plan.dynamic_ls else None
        m, info = OS.run_condition(topo, row, plan.z[b], plan.pCa[b], plan.ls[b], plan.keys[b],
                                   dt_ms=plan.dt, n_newton=static.n_newton_steps, n_cg=static.n_cg_steps,
                                   dt=dtype, K_lat=K, nu=float(plan.nu[b]), udtype=udtype,
                                   subpop=plan_subpop(plan, b), **kw)
        out[b] = m
        infos.append(info)
    return out, infos


COUNT_KEYS = ('n_bound', 'n_xb_drx', 'n_xb_loose', 'n_xb_tight_1', 'n_xb_tight_2', 'n_xb_free_2', 'n_xb_srx',
              'n_tm_state_0', 'n_tm_state_1', 'n_tm_state_2', 'n_tm_state_3', 'atp_consumed', 'newly_bound')
# Metrics that are float32 rounding noise by construction: the residual sits
# below the float32 floor of the force balance, and the deltas/work are
# differences of nearly equal numbers.  Compared with an absolute bound.
NOISE_ABS = {'solver_residual': 0.76, 'titin_energy_delta_avg': 0.05, 'thick_energy_first_delta_avg': 0.05,
             'work_thick': 0.5, 'work_thick_mean': 1e-3, 'work_per_atp': 2.0, 'newton_iters': 4}


def first_divergence(a, b, keys, solver=True):
    """First step where any integer count metric differs (None if never).

    With ``solver`` the Newton iteration count is included: when the float32
    residual sits at its noise floor (~0.75 pN at thick_k=7500) the
    accept-or-iterate decision depends on rounding, and a different decision
    moves the lattice by a whole Newton step -- the deterministic analogue of
    a stochastic divergence.
    """
    idx = [keys.index(k) for k in COUNT_KEYS + (('newton_iters',) if solver else ())]
    diff = np.any(a[..., idx, :] != b[..., idx, :], axis=tuple(range(a.ndim - 2)) + (a.ndim - 2,))
    w = np.where(diff)[0]
    return int(w[0]) if len(w) else None


def compare_metrics(a, b, keys, rtol=1e-5, upto=None):
    """Max relative error per metric over steps [0, upto); noise metrics by absolute bound."""
    bad = {}
    sl = slice(0, upto)
    for k, name in enumerate(keys):
        x, y = a[..., k, sl], b[..., k, sl]
        if name in NOISE_ABS:
            e = np.max(np.abs(x - y)) if x.size else 0.0
            if e > NOISE_ABS[name]:
                bad[name] = float(e)
            continue
        e = np.max(np.abs(x - y) / np.maximum(np.abs(y), 1.0)) if x.size else 0.0
        if e > rtol:
            bad[name] = float(e)
    return bad
