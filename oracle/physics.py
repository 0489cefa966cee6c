"""Physics of one condition: rates, Pade expm, sampling, nearest sites, forces, JVPs.

TEST INFRASTRUCTURE (oracle).  Plain NumPy restatement of the reference,
function by function, in a selectable float dtype (float32 reproduces the
reference's single-precision path; float64 is the FP64 oracle).  Operation
order follows the reference expressions so float32 results agree to
rounding; every function cites the lines it restates.

Conventions: ``p`` is a dict of the 44 DynamicParams values already cast to
the working dtype; topology arrays keep their float32 values (as the
reference's do, even under ``jax_enable_x64``).
"""
from __future__ import annotations

import numpy as np

from multifil_jax_b200.params import DYNAMIC_FIELDS

N_TITIN_PER_THICK = 6            # forces.py:104, :630
HEAD_REACH = 13.0                # geometry.py:224
RATE_CAP = 10000.0               # rate_functions.py:383,462,516,558,620
MIN_FLOAT32_TOLERANCE = 0.25     # solver.py:104
# Pade(6,6) coefficients, stored as float32 by the reference (transitions.py:84-92)
PADE6_B = np.array([1.0, 1.0 / 2.0, 1.0 / 9.0, 1.0 / 72.0, 1.0 / 1008.0, 1.0 / 30240.0,
                    1.0 / 1209600.0], dtype=np.float32)


def param_dict(row, dt):
    return {name: dt(row[i]) for i, name in enumerate(DYNAMIC_FIELDS)}


# ---------------------------------------------------------------------------
# JAX reassociation orders
# ---------------------------------------------------------------------------

def assoc_scan(fn, elems, axis=-1):
    """``lax.associative_scan`` with JAX's odd/even recursion order.

    ``elems`` is a tuple of arrays scanned along ``axis``; ``fn(left, right)``
    combines two tuples.  Used for the Thomas substitutions (solver.py:165-219)
    and for ``jnp.cumsum`` (lowered to this scan on CPU/GPU).
    """
    elems = tuple(np.moveaxis(e, axis, 0) for e in elems)

    def rec(es):
        n = es[0].shape[0]
        if n < 2:
            return es
        red = fn(tuple(e[0:-1:2] for e in es), tuple(e[1::2] for e in es))
        odd = rec(red)
        if n % 2 == 0:
            even = fn(tuple(o[:-1] for o in odd), tuple(e[2::2] for e in es))
        else:
            even = fn(odd, tuple(e[2::2] for e in es))
        even = tuple(np.concatenate([e[0:1], v], axis=0) for e, v in zip(es, even))
        out = []
        for ev, od in zip(even, odd):
            r = np.empty((ev.shape[0] + od.shape[0],) + ev.shape[1:], dtype=np.result_type(ev, od))
            r[0::2] = ev
            r[1::2] = od
            out.append(r)
        return tuple(out)
    return tuple(np.moveaxis(o, 0, axis) for o in rec(elems))


def cumsum_jax(x, axis=-1):
    """``jnp.cumsum`` = associative scan with ``+`` (JAX association order)."""
    return assoc_scan(lambda a, b: (a[0] + b[0],), (x,), axis=axis)[0]


# ---------------------------------------------------------------------------
# Matrix exponential (transitions.py:99-190)
# ---------------------------------------------------------------------------

def _matmul(a, b):
    """Batched matmul with a left-to-right sum over the inner index."""
    n = a.shape[-1]
    out = a[..., :, 0:1] * b[..., 0:1, :]
    for j in range(1, n):
        out = out + a[..., :, j:j + 1] * b[..., j:j + 1, :]
    return out


def _lu_solve(A, B):
    """Batched solve with LU and partial pivoting (first max as pivot)."""
    A = A.copy()
    B = B.copy()
    m, n = A.shape[0], A.shape[-1]
    rows = np.arange(m)
    for k in range(n):
        piv = k + np.argmax(np.abs(A[:, k:, k]), axis=1)
        sw = piv != k
        if np.any(sw):
            r = rows[sw]
            tmp = A[r, k, :].copy()
            A[r, k, :] = A[r, piv[sw], :]
            A[r, piv[sw], :] = tmp
            tmp = B[r, k, :].copy()
            B[r, k, :] = B[r, piv[sw], :]
            B[r, piv[sw], :] = tmp
        for i in range(k + 1, n):
            l = A[:, i, k] / A[:, k, k]
            A[:, i, k + 1:] = A[:, i, k + 1:] - l[:, None] * A[:, k, k + 1:]
            B[:, i, :] = B[:, i, :] - l[:, None] * B[:, k, :]
    X = np.empty_like(B)
    for i in range(n - 1, -1, -1):
        acc = B[:, i, :]
        for j in range(i + 1, n):
            acc = acc - A[:, i, j:j + 1] * X[:, j, :]
        X[:, i, :] = acc / A[:, i, i:i + 1]
    return X


def expm_pade6(A, with_s=False):
    """exp(A) for a batch of small matrices: scale by 2^-s, Pade(6,6), square s times.

    Restates expm_pade6_batch (transitions.py:99-190) including the 18-trip
    masked squaring cap, row renormalisation and the NaN -> 1/n guard.
    """
    dt = A.dtype
    n = A.shape[-1]
    a_norms = np.max(np.sum(np.abs(A), axis=2), axis=1)
    s = np.maximum(0, np.ceil(np.log2(a_norms / dt.type(0.5) + dt.type(1e-10))).astype(np.int32))
    scale = np.power(dt.type(2.0), s.astype(dt))[:, None, None]
    As = A / scale
    eye = np.eye(n, dtype=np.float32)
    b = PADE6_B
    A2 = _matmul(As, As)
    A4 = _matmul(A2, A2)
    A6 = _matmul(A4, A2)
    inner = b[1] * eye + b[3] * A2 + b[5] * A4
    U = _matmul(As, inner)
    V = b[0] * eye + b[2] * A2 + b[4] * A4 + b[6] * A6
    R = _lu_solve((V - U).astype(dt), (V + U).astype(dt))
    for i in range(18):
        sq = i < s
        if not np.any(sq):
            break
        R2 = _matmul(R, R)
        R = np.where(sq[:, None, None], R2, R)
    R = R / np.sum(R, axis=2, keepdims=True)
    R = np.where(np.isnan(R), dt.type(1.0 / n), R).astype(dt)
    return (R, s) if with_s else R


# ---------------------------------------------------------------------------
# Rate matrices
# ---------------------------------------------------------------------------

def tm_Q27(p, pCa, dt):
    """27 tropomyosin generators indexed 9*n2 + 3*n3 + nclosed (transitions.py:434-513)."""
    ca = dt(10.0) ** (-pCa)
    lv = np.array([0, 1, 2], dtype=np.float32)
    n2, n3, nc = [g.reshape(-1) for g in np.meshgrid(lv, lv, lv, indexing='ij')]
    JC, JM = p['tm_J_C'], p['tm_J_M']
    h = JC * n2 + JM * n3 - dt(0.5) * (JC + JM) * nc
    fwd = np.exp(dt(0.5) * h)
    bwd = np.exp(dt(-0.5) * h)
    k01 = p['tm_k_01'] * ca * fwd
    k12 = p['tm_k_12'] * fwd
    k23 = p['tm_k_23'] * fwd
    k30 = np.broadcast_to(p['tm_k_30'], (27,)).astype(h.dtype)
    k10 = (p['tm_k_01'] / p['tm_Keq_01']) * bwd
    k21 = (p['tm_k_12'] / p['tm_Keq_12']) * bwd
    k32 = (p['tm_k_23'] / p['tm_Keq_23']) * bwd
    Q = np.zeros((27, 4, 4), dtype=h.dtype)
    Q[:, 0, 0] = -k01
    Q[:, 0, 1] = k01
    Q[:, 1, 0] = k10
    Q[:, 1, 1] = -(k10 + k12)
    Q[:, 1, 2] = k12
    Q[:, 2, 1] = k21
    Q[:, 2, 2] = -(k21 + k23)
    Q[:, 2, 3] = k23
    Q[:, 3, 0] = k30
    Q[:, 3, 2] = k32
    Q[:, 3, 3] = -(k30 + k32)
    return Q


def xb_Q(x, d, perm, p, pCa, dt):
    """6x6 crossbridge generators at axial offsets ``x`` and spacing ``d``.

    Restates xb_rate_matrix (transitions.py:632-804) with the rate laws of
    rate_functions.py:318-753 (caps, NaN guards, log-space reverse rates).
    """
    x = x.astype(dt)
    y = np.full(x.shape, d, dtype=dt)
    perm = perm.astype(dt)
    ca = dt(10.0) ** (-pCa)
    r = np.sqrt(x ** 2 + y ** 2)
    th = np.arctan2(y, x)
    half = dt(0.5)
    kt = dt(1.3810e-23) * (p['temp_celsius'] + dt(273.15)) * dt(1e21)
    Ew = (half * p['xb_g_k_weak'] * (r - p['xb_g_rest_weak']) ** 2
          + half * p['xb_c_k_weak'] * (th - p['xb_c_rest_weak']) ** 2) / kt
    Es = (half * p['xb_g_k_strong'] * (r - p['xb_g_rest_strong']) ** 2
          + half * p['xb_c_k_strong'] * (th - p['xb_c_rest_strong']) ** 2) / kt
    Ediff = Ew - Es
    U_drx = p['xb_U_DRX']
    U_loose = p['xb_U_loose'] + Ew
    U_t1 = p['xb_U_tight_1'] + Es
    U_t2 = p['xb_U_tight_2'] + Es
    f_s = p['xb_g_k_strong'] * (r - p['xb_g_rest_strong']) + (dt(1.0) / r) * p['xb_c_k_strong'] * (
        th - p['xb_c_rest_strong'])
    cap = dt(RATE_CAP)
    with np.errstate(all='ignore'):
        r01 = perm * p['xb_r01_coeff'] * np.exp(-Ew)
        r01 = np.where(np.isnan(r01), dt(0.0), r01)
        r10 = np.exp(np.log(r01 + dt(0.005)) - (U_drx - U_loose))
        r10 = np.minimum(r10, cap)
        r10 = np.where(np.isnan(r10), cap, r10)
        r12 = p['xb_r12_coeff'] * np.exp(np.minimum(Ediff, dt(30.0)) / dt(2.0))
        r12 = np.where(np.isnan(r12), dt(0.0), r12)
        r21 = np.minimum(np.exp(np.log(r12) - (U_loose - U_t1)), cap)
        r23 = np.minimum(p['xb_r23_coeff'] * np.exp(-f_s * p['xb_delta_23'] / kt), cap)
        r32 = np.exp(np.minimum(np.log(r23 + dt(1e-30)) + (U_t2 - U_t1), np.log(cap)))
        r34 = np.minimum(p['xb_r34_coeff'] * np.exp(f_s * p['xb_delta_34'] / kt), cap)
    ones = np.ones(x.shape, dtype=dt)
    r43 = dt(0.0) * ones
    r40 = p['xb_r40'] * ones
    r04 = p['xb_r04'] * ones
    k0, kmax, b, ca50 = p['xb_srx_k0'], p['xb_srx_kmax'], p['xb_srx_b'], p['xb_srx_ca50']
    r50 = (k0 + ((kmax - k0) * ca ** b) / (ca50 ** b + ca ** b)) * ones
    r05 = p['xb_r05'] * ones
    Q = np.zeros(x.shape + (6, 6), dtype=dt)
    Q[:, 0, 0] = -(r01 + r04 + r05)
    Q[:, 0, 1] = r01
    Q[:, 0, 4] = r04
    Q[:, 0, 5] = r05
    Q[:, 1, 0] = r10
    Q[:, 1, 1] = -(r10 + r12)
    Q[:, 1, 2] = r12
    Q[:, 2, 1] = r21
    Q[:, 2, 2] = -(r21 + r23)
    Q[:, 2, 3] = r23
    Q[:, 3, 2] = r32
    Q[:, 3, 3] = -(r32 + r34)
    Q[:, 3, 4] = r34
    Q[:, 4, 0] = r40
    Q[:, 4, 3] = r43
    Q[:, 4, 4] = -(r43 + r40)
    Q[:, 5, 0] = r50
    Q[:, 5, 5] = -r50
    return Q


def xb_Q_bins(topo, p, pCa, d, dt):
    """(2*n_bins, 6, 6): permissiveness-0 block then permissiveness-1 block
    (transitions.py:807-922)."""
    c = topo.xb_bin_centers
    nb = c.shape[0]
    q0 = xb_Q(c, d, np.zeros(nb), p, pCa, dt)
    q1 = xb_Q(c, d, np.ones(nb), p, pCa, dt)
    return np.concatenate([q0, q1], axis=0)


def absorbing(Q):
    """Rows 4 then 0 zeroed (transitions.py:1077)."""
    Q = Q.copy()
    Q[..., 4, :] = 0
    Q[..., 0, :] = 0
    return Q


def xb_bin_key(x_axial, perm, topo):
    """ap*n_bins + clip(digitize(x, edges) - 1, 0, n_bins-1) (transitions.py:915-920)."""
    nb = topo.xb_bin_centers.shape[0]
    b = np.clip(np.digitize(x_axial, topo.xb_bin_edges) - 1, 0, nb - 1)
    return perm.astype(np.int32) * nb + b


def sample(prob, u):
    """argmax(u < cumsum(p)), 0 when no entry qualifies (transitions.py:619-620,1164-1165)."""
    cum = cumsum_jax(prob, axis=1)
    return np.argmax(u[:, None] < cum, axis=1)


# ---------------------------------------------------------------------------
# Nearest binding site (geometry.py:60-262)
# ---------------------------------------------------------------------------

def nearest_sites(thick_x, thin_x, topo, ls, dt):
    nxb = topo.n_xb_per_crown
    base = np.repeat(thick_x, nxb, axis=1).reshape(-1)
    head = base + dt(HEAD_REACH)
    npf = topo.n_sites_per_face[topo.xb_to_thin_id, topo.xb_to_thin_face]
    sites = topo.xb_to_site_indices
    fpos = thin_x[topo.xb_to_thin_id[:, None], sites]
    dist = np.abs(fpos - head[:, None])
    mask = (np.arange(sites.shape[1])[None, :] < npf[:, None]) & (fpos > 0.0)
    md = np.where(mask, dist, np.inf)
    k = np.argmin(md, axis=1)
    nearest = sites[np.arange(sites.shape[0]), k].astype(np.int32)
    axial = thin_x[topo.xb_to_thin_id, nearest] - base
    dist2 = np.stack([axial, np.full(axial.shape, ls, dtype=axial.dtype)], axis=1)
    return nearest, dist2


# ---------------------------------------------------------------------------
# Transitions
# ---------------------------------------------------------------------------

def tm_config(tm, prev, nxt):
    """9*n2 + 3*n3 + n_closed over same-chain neighbours (transitions.py:384-431)."""
    n_thin, n_sites = tm.shape
    idx = np.arange(n_sites)[None, :]
    rows = np.arange(n_thin)[:, None]
    pr = prev != idx
    nr = nxt != idx
    tp = tm[rows, prev]
    tn = tm[rows, nxt]

    def cnt(pred):
        return ((pred(tp) & pr).astype(np.int32) + (pred(tn) & nr).astype(np.int32)).clip(max=2)
    n2 = cnt(lambda s: s == 2)
    n3 = cnt(lambda s: s == 3)
    nc = cnt(lambda s: (s == 0) | (s == 1))
    return (n2 * 9 + n3 * 3 + nc).reshape(-1)


def thin_transitions(tm, thin_bound, P_tm, topo, u, labels=None):
    """New tm_states (transitions.py:516-625), with the bound-and-open lock.

    ``labels`` (per site): ``P_tm`` holds one 27-table set per population and
    each site reads its own population's set (transitions.py:586-596)."""
    cfg = tm_config(tm, topo.tm_prev_neighbor, topo.tm_next_neighbor)
    s = tm.reshape(-1).astype(np.int32)
    prob = P_tm[cfg, s] if labels is None else P_tm[np.asarray(labels), cfg, s]
    locked = (s == 3) & (thin_bound.reshape(-1) >= 0)
    lock_row = np.array([0.0, 0.0, 0.0, 1.0], dtype=prob.dtype)
    prob = np.where(locked[:, None], lock_row, prob)
    return sample(prob, u).reshape(tm.shape).astype(np.int8)


def permissiveness(tm, nearest, topo):
    n_sites = tm.shape[1]
    st = tm[topo.xb_to_thin_id, np.clip(nearest, 0, n_sites - 1)]
    return (st == 3).astype(np.float32) * topo.xb_valid.astype(np.float32)


def thick_transitions(xb_state, xb_bound, thin_bound, nearest, x_axial, tm, P_bins, topo, u, labels=None):
    """Sample crossbridge states and update the binding bookkeeping.

    ``labels`` (per head): ``P_bins`` holds one bin grid per population and a
    head reads its own population's grid (transitions.py:925-994).

    Restates thick_transitions (transitions.py:1081-1245).  The two scatters
    into ``thin.bound_to`` are applied in crossbridge-index order with the last
    writer winning, which is how XLA executes duplicate-index scatters on CPU.
    """
    n_sites = tm.shape[1]
    perm = permissiveness(tm, nearest, topo)
    key = xb_bin_key(x_axial, perm, topo)
    old = xb_state.astype(np.int32)
    prob = P_bins[key, old] if labels is None else P_bins[np.asarray(labels), key, old]
    new = sample(prob, u)
    old_b = (old >= 1) & (old <= 3)
    new_b = (new >= 1) & (new <= 3)
    binding = ~old_b & new_b
    unbinding = old_b & ~new_b
    tb = thin_bound.reshape(-1)
    site = np.clip(nearest, 0, n_sites - 1)
    tgt = topo.xb_to_thin_id * n_sites + site
    occupied = tb[tgt] >= 0
    can_bind = binding & (perm > 0.5) & ~occupied
    new_xb_bound = np.where(can_bind, nearest, np.where(unbinding, -1, xb_bound)).astype(np.int32)
    # STEP 1: clear the sites of unbinding heads (every head writes)
    i1 = topo.xb_to_thin_id * n_sites + np.clip(xb_bound, 0, n_sites - 1)
    v1 = np.where(unbinding & (xb_bound >= 0), -1, tb[i1])
    t1 = tb.copy()
    for k in range(i1.shape[0]):
        t1[i1[k]] = v1[k]
    # STEP 2: claim nearest sites (every head writes)
    v2 = np.where(can_bind, np.arange(tgt.shape[0]), t1[tgt])
    t2 = t1.copy()
    for k in range(tgt.shape[0]):
        t2[tgt[k]] = v2[k]
    new = np.where(binding & ~can_bind, 0, new)
    return new.astype(np.int8), new_xb_bound, t2.reshape(thin_bound.shape).astype(np.int32)


# ---------------------------------------------------------------------------
# Forces (forces.py) and their derivatives
# ---------------------------------------------------------------------------

class ForceModel:
    """Axial residual F(x) of one condition and its directional derivatives.

    ``F`` restates compute_forces_vectorized (forces.py:425-500); the
    derivatives are the analytic forms of what ``jax.jvp``/``jax.grad``
    evaluate in the solver (solver.py:413,633), including the dynamic lattice
    spacing terms (forces.py:649-749, solver.py:502-596).
    """

    def __init__(self, topo, p, xb_state, xb_bound, z, dt):
        self.t = topo
        self.p = p
        self.dt = dt
        self.z = dt(z)
        nxb = topo.n_xb_per_crown
        s = xb_state.astype(np.int32)
        self.bound = (s >= 1) & (s <= 3) & (xb_bound >= 0)
        strong = (s == 2) | (s == 3)
        self.c_rest = np.where(strong, p['xb_c_rest_strong'], p['xb_c_rest_weak']).astype(dt)
        self.c_k = np.where(strong, p['xb_c_k_strong'], p['xb_c_k_weak']).astype(dt)
        self.g_rest = np.where(strong, p['xb_g_rest_strong'], p['xb_g_rest_weak']).astype(dt)
        self.g_k = np.where(strong, p['xb_g_k_strong'], p['xb_g_k_weak']).astype(dt)
        n_sites = topo.n_sites
        self.site_idx = (np.clip(topo.xb_to_thin_id, 0, topo.n_thin - 1) * n_sites
                         + np.clip(xb_bound, 0, n_sites - 1))
        self.crown_idx = np.arange(topo.total_xbs) // nxb
        self.n_thick_nodes = topo.n_thick * topo.n_crowns

    def split(self, x):
        t = self.t
        return (x[:self.n_thick_nodes].reshape(t.n_thick, t.n_crowns),
                x[self.n_thick_nodes:].reshape(t.n_thin, t.n_sites))

    # -- primal ------------------------------------------------------------
    def _titin(self, x_last, d):
        p, dt = self.p, self.dt
        ad = self.z - x_last
        L = np.sqrt(ad ** 2 + d ** 2)
        arg = p['titin_b'] * (L - p['titin_rest'])
        clipped = (arg < -100.0) | (arg > 100.0)
        Ft = np.maximum(p['titin_a'] * np.exp(np.clip(arg, dt(-100.0), dt(100.0))), dt(0.0))
        return ad, L, Ft, clipped

    def _xb_geom(self, xt, xn, d):
        base = np.repeat(xt.reshape(-1), self.t.n_xb_per_crown)
        bs = xn.reshape(-1)[self.site_idx]
        xd = bs - base
        r = np.sqrt(xd ** 2 + d ** 2)
        rs = np.where(r > 1e-10, r, self.dt(1e-10))
        cos = xd / rs
        sin = d / rs
        th = np.arctan2(d, xd)
        return xd, r, rs, cos, sin, th

    def xb_forces(self, xt, xn, d):
        xd, r, rs, cos, sin, th = self._xb_geom(xt, xn, d)
        f = self.g_k * (r - self.g_rest) * cos - (self.dt(1.0) / rs) * self.c_k * (th - self.c_rest) * sin
        return np.where(self.bound, f, self.dt(0.0))

    def residual(self, x, d):
        t, p, dt = self.t, self.p, self.dt
        xt, xn = self.split(x)
        # thick backbone + titin (forces.py:82-162)
        aw = np.concatenate([np.zeros((t.n_thick, 1), dt), xt], axis=1)
        spring = (np.diff(aw, axis=1) - t.crown_rests) * p['thick_k']
        ad, L, Ft, _ = self._titin(xt[:, -1], d)
        cosang = np.where(L > 0, ad / L, dt(0.0))
        tit = N_TITIN_PER_THICK * (Ft * cosang)
        Fthick = np.diff(np.concatenate([spring, tit[:, None]], axis=1), axis=1)
        # thin backbone (forces.py:210-242)
        az = np.concatenate([xn, np.full((t.n_thin, 1), self.z, dt)], axis=1)
        sp = (np.diff(az, axis=1) - t.binding_rests) * p['thin_k']
        Fthin = np.diff(np.concatenate([np.zeros((t.n_thin, 1), dt), sp], axis=1), axis=1)
        # crossbridges (forces.py:277-418)
        f = self.xb_forces(xt, xn, d)
        fc = f.reshape(-1, t.n_xb_per_crown)
        acc = fc[:, 0]
        for j in range(1, t.n_xb_per_crown):
            acc = acc + fc[:, j]
        fthin = np.zeros(t.n_thin * t.n_sites, dtype=dt)
        np.add.at(fthin, self.site_idx, -f)
        return np.concatenate([(Fthick + acc.reshape(t.n_thick, t.n_crowns)).reshape(-1),
                               (Fthin + fthin.reshape(t.n_thin, t.n_sites)).reshape(-1)])

    def radial(self, x, d, K_lat, d_ref):
        """F_rad = -K(d - d_ref) - sum f_xb_radial - sum titin_radial (solver.py:502-528)."""
        dt = self.dt
        xt, xn = self.split(x)
        xd, r, rs, cos, sin, th = self._xb_geom(xt, xn, d)
        fr = self.g_k * (r - self.g_rest) * sin + (dt(1.0) / rs) * self.c_k * (th - self.c_rest) * cos
        fxb = np.sum(np.where(self.bound, fr, dt(0.0)))
        ad, L, Ft, _ = self._titin(xt[:, -1], d)
        Ls = np.where(L > 1e-10, L, dt(1e-10))
        ftit = np.sum(N_TITIN_PER_THICK * Ft * (d / Ls))
        return -K_lat * (d - d_ref) + (-fxb) + (-ftit)

    # -- derivatives --------------------------------------------------------
    def _xb_partials(self, xt, xn, d):
        """df/dx, df/dd (= dfr/dx) and dfr/dd per crossbridge (zero if unbound)."""
        dt = self.dt
        xd, r, rs, cos, sin, th = self._xb_geom(xt, xn, d)
        gk, g0, ck, c0 = self.g_k, self.g_rest, self.c_k, self.c_rest
        dth = th - c0
        inv_r2 = dt(1.0) / (r * r)
        f_x = gk * (cos * cos + (dt(1.0) - g0 / r) * sin * sin) + ck * inv_r2 * (dt(2.0) * dth * sin * cos + sin * sin)
        f_d = gk * sin * cos * (g0 / r) - ck * inv_r2 * (sin * cos + dth * (cos * cos - sin * sin))
        fr_d = gk * (sin * sin + (r - g0) * cos * cos / r) + ck * inv_r2 * (cos * cos - dt(2.0) * dth * sin * cos)
        z0 = dt(0.0)
        return (np.where(self.bound, f_x, z0), np.where(self.bound, f_d, z0),
                np.where(self.bound, fr_d, z0))

    def _titin_partials(self, x_last, d):
        """d(titin axial)/dx_last, d(titin axial)/dd (= d(titin radial)/dx_last), d(radial)/dd."""
        p, dt = self.p, self.dt
        ad, L, Ft, clipped = self._titin(x_last, d)
        b = np.where(clipped, dt(0.0), p['titin_b'])
        n = dt(N_TITIN_PER_THICK)
        a_x = -n * Ft * (b * ad * ad / (L * L) + d * d / (L * L * L))
        a_d = n * Ft * ad * d * (b / (L * L) - dt(1.0) / (L * L * L))
        r_d = n * Ft * (b * d * d / (L * L) + ad * ad / (L * L * L))
        return a_x, a_d, r_d

    def jvp(self, x, d, v, vd=None, K_lat=None):
        """J @ [v, vd] of the axial residual (and of the radial row when ``vd`` is given)."""
        t, p, dt = self.t, self.p, self.dt
        xt, xn = self.split(x)
        vt, vn = self.split(v)
        # thick backbone
        vw = np.concatenate([np.zeros((t.n_thick, 1), dt), vt], axis=1)
        s_dot = np.diff(vw, axis=1) * p['thick_k']
        a_x, a_d, r_d = self._titin_partials(xt[:, -1], d)
        tit_dot = a_x * vt[:, -1]
        if vd is not None:
            tit_dot = tit_dot + a_d * vd
        Jt = np.diff(np.concatenate([s_dot, tit_dot[:, None]], axis=1), axis=1)
        # thin backbone
        vz = np.concatenate([vn, np.zeros((t.n_thin, 1), dt)], axis=1)
        sp_dot = np.diff(vz, axis=1) * p['thin_k']
        Jn = np.diff(np.concatenate([np.zeros((t.n_thin, 1), dt), sp_dot], axis=1), axis=1)
        # crossbridges
        f_x, f_d, fr_d = self._xb_partials(xt, xn, d)
        base_v = np.repeat(vt.reshape(-1), t.n_xb_per_crown)
        dxd = vn.reshape(-1)[self.site_idx] - base_v
        fdot = f_x * dxd
        if vd is not None:
            fdot = fdot + f_d * vd
        fc = fdot.reshape(-1, t.n_xb_per_crown)
        acc = fc[:, 0]
        for j in range(1, t.n_xb_per_crown):
            acc = acc + fc[:, j]
        fthin = np.zeros(t.n_thin * t.n_sites, dtype=dt)
        np.add.at(fthin, self.site_idx, -fdot)
        out = np.concatenate([(Jt + acc.reshape(t.n_thick, t.n_crowns)).reshape(-1),
                              (Jn + fthin.reshape(t.n_thin, t.n_sites)).reshape(-1)])
        if vd is None:
            return out
        # radial row: d/dx of -sum fr (fr_x = f_d); d(titin radial)/dx_last = -a_d
        rad = (-np.sum(f_d * dxd) + np.sum(a_d * vt[:, -1])
               + (-K_lat - np.sum(fr_d) - np.sum(r_d)) * vd)
        return out, rad

    def J_dd(self, x, d, K_lat):
        xt, _ = self.split(x)
        _, _, fr_d = self._xb_partials(xt, self.split(x)[1], d)
        _, _, r_d = self._titin_partials(xt[:, -1], d)
        return -K_lat - np.sum(fr_d) - np.sum(r_d)


# ---------------------------------------------------------------------------
# Thomas preconditioner (solver.py:104-322, state.py:269-316)
# ---------------------------------------------------------------------------

def thomas_factors(n, k, first_boundary, dt):
    """Negated, regularised single-filament tridiagonal factor.

    thick: diag 2k (last k), thin: diag 2k (first k); off-diagonals -k after
    negation; +1e-9 on the diagonal (solver.py:243-282).
    """
    k = dt(k)
    diag = np.full(n, dt(-2.0) * k, dtype=dt)
    if first_boundary:
        diag[0] = dt(-1.0) * k
    else:
        diag[-1] = dt(-1.0) * k
    diag = -diag + dt(1e-9)
    off = np.full(n - 1, -k, dtype=dt)
    md = [diag[0]]
    mult = []
    for i in range(1, n):
        m = off[i - 1] / md[i - 1]
        mult.append(m)
        md.append(diag[i] - m * off[i - 1])
    inv = (dt(1.0) / np.array(md, dtype=dt)).astype(dt)
    return inv, off, np.array(mult, dtype=dt)


def _compose(l, r):
    return (r[0] * l[0], r[0] * l[1] + r[1])


def thomas_apply(fac, rhs):
    """Forward and back substitution as affine-map associative scans (solver.py:165-219).

    ``rhs`` has shape (n_filaments, n); scans run along the last axis.
    """
    inv, upper, mult = fac
    dt = rhs.dtype
    nf = rhs.shape[0]
    a_f = np.broadcast_to(np.concatenate([np.ones(1, dt), -mult]), rhs.shape)
    _, y = assoc_scan(_compose, (a_f, rhs), axis=1)
    a_b = np.concatenate([-upper * inv[:-1], np.zeros(1, dt)])
    a_b = np.broadcast_to(a_b[::-1], rhs.shape)
    _, xr = assoc_scan(_compose, (a_b, (y * inv)[:, ::-1]), axis=1)
    return xr[:, ::-1]


class Preconditioner:
    def __init__(self, topo, p, dt):
        self.t = topo
        self.thick = thomas_factors(topo.n_crowns, p['thick_k'], False, dt)
        self.thin = thomas_factors(topo.n_sites, p['thin_k'], True, dt)
        self.nt = topo.n_thick * topo.n_crowns

    def __call__(self, v):
        t = self.t
        a = thomas_apply(self.thick, v[:self.nt].reshape(t.n_thick, t.n_crowns))
        b = thomas_apply(self.thin, v[self.nt:].reshape(t.n_thin, t.n_sites))
        return np.concatenate([a.reshape(-1), b.reshape(-1)])
