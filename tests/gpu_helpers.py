"""Drive the CUDA engine the way the parity tests need (injected uniforms, traces)."""
import numpy as np

from oracle import step as OS, prng


def tt(a, dtype=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda().contiguous()


def keys_tensor(keys):
    import torch
    return tt(np.asarray(keys, np.uint32).astype(np.int64)).to(torch.int32).contiguous()


def run_engine(eng, topos, params, z, pCa, ls, keys, n_steps=None, K_lat=None, nu=None, dt=None, flags=0,
               u_thin=None, u_xb=None, traces=False, chunk_steps=0):
    import torch
    B, T = np.asarray(z).shape
    ns = np.full(B, T, np.int32) if n_steps is None else np.asarray(n_steps, np.int32)
    res = eng.run_batch(topos, tt(params, torch.float32), tt(z, torch.float32), tt(pCa, torch.float32),
                        tt(ls, torch.float32), tt(ns), keys_tensor(keys),
                        K_lat=tt(np.zeros(B) if K_lat is None else K_lat, torch.float32),
                        nu=tt(np.zeros(B) if nu is None else nu, torch.float32),
                        dt=tt(np.ones(B) if dt is None else dt, torch.float32), flags=flags,
                        u_thin=None if u_thin is None else tt(u_thin, torch.float32),
                        u_xb=None if u_xb is None else tt(u_xb, torch.float32),
                        want_x_trace=traces, want_state_trace=traces, chunk_steps=chunk_steps)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in res.items()}


def oracle_with_states(topo, row, z, pCa, ls, key, dtype=np.float32, K_lat=None, nu=0.0, uniforms=None):
    return OS.run_condition(topo, row, z, pCa, ls, key, dt=dtype, K_lat=K_lat, nu=nu, uniforms=uniforms,
                            record_states=True)


def state_divergence(res, b, info, topo, T):
    """First step where the engine's integer state arrays differ from the oracle's."""
    X, S = topo.total_xbs, topo.n_sites_total
    st, bt = res['state_trace'][b], res['bound_trace'][b]
    for t in range(T):
        o = info['states'][t]
        if not (np.array_equal(st[t, :X], o.xb_state) and np.array_equal(st[t, X:X + S], o.tm.reshape(-1))
                and np.array_equal(bt[t, :X], o.xb_bound)
                and np.array_equal(bt[t, X:X + S], o.thin_bound.reshape(-1))):
            return t
    return None


def oracle_positions(info, topo):
    return np.stack([np.concatenate([s.thick_x.reshape(-1), s.thin_x.reshape(-1)]) for s in info['states']])


def oracle_tables(topo, row, pCa, d, dtype):
    """The oracle's sampling tables at (pCa, d): (P_tm [27,4,4], P_xb [2*n_bins,6,6])."""
    from oracle import physics as ph
    p = ph.param_dict(row, dtype)
    tab = OS.tables(topo, p, pCa, d, 1.0, dtype)
    return tab.P_tm, tab.P_xb


def divergence_cause(topo, row, pCa, d, dtype, info, res, b, t):
    """Why the engine's step t differs from the oracle's (fixed spacing, constant pCa).

    Returns (cause, margin): 'draw' with the smallest distance between a
    uniform and a threshold of the oracle's cumulative row, over the heads and
    sites whose new state differs; 'bin' with the smallest distance of such a
    head's axial offset to a bin edge (nm); 'newton' when no integer state
    differs (the accept-or-iterate decision of the Newton loop, the residual
    being at its floor).
    """
    from oracle import physics as ph
    X, S = topo.total_xbs, topo.n_sites_total
    st = res['state_trace'][b, t]
    o = info['states'][t]
    u_thin, u_xb = info['uniforms'][t]
    prev = info['states'][t - 1] if t > 0 else None
    old_xb = prev.xb_state.astype(np.int32) if prev is not None else np.zeros(X, np.int32)
    old_tm = prev.tm if prev is not None else np.zeros((topo.n_thin, topo.n_sites), np.int8)
    P_tm, P_xb = oracle_tables(topo, row, pCa, d, dtype)
    heads = np.flatnonzero(st[:X] != o.xb_state)
    sites = np.flatnonzero(st[X:X + S] != o.tm.reshape(-1))
    if heads.size == 0 and sites.size == 0:
        return 'newton', None
    margins, bins = [], []
    if heads.size:
        perm = ph.permissiveness(o.tm, o.xb_nearest, topo)
        key = ph.xb_bin_key(o.xb_dist[:, 0], perm, topo)
        cum = np.cumsum(P_xb[key[heads], old_xb[heads]].astype(np.float64), axis=1)
        margins.append(np.min(np.abs(cum - np.asarray(u_xb, np.float64)[heads, None]), axis=1))
        bins.append(np.min(np.abs(o.xb_dist[heads, 0][:, None].astype(np.float64)
                                  - topo.xb_bin_edges[None, :].astype(np.float64)), axis=1))
    if sites.size:
        cfg = ph.tm_config(old_tm, topo.tm_prev_neighbor, topo.tm_next_neighbor)
        s_old = old_tm.reshape(-1).astype(np.int32)
        cum = np.cumsum(P_tm[cfg[sites], s_old[sites]].astype(np.float64), axis=1)
        margins.append(np.min(np.abs(cum - np.asarray(u_thin, np.float64)[sites, None]), axis=1))
    m = float(np.min(np.concatenate(margins)))
    if bins and float(np.min(np.concatenate(bins))) < 1e-4:
        return 'bin', float(np.min(np.concatenate(bins)))
    return 'draw', m


def float32_force_floor(topo, d):
    """Force change of two float32 roundings of every thick filament's M-line
    node (pN): the force reads absolute float32 positions (~58 nm there)."""
    x0 = np.float32(np.max(np.abs(topo.crown_offsets[:, 0])))
    return topo.n_thick * float(d.thick_k) * 2.0 * float(np.spacing(x0))
