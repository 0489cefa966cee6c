"""Operation counts of one timestep of the reference algorithm, by phase.

TEST INFRASTRUCTURE (oracle).  ``python -m oracle.opcount`` prints the
counts; the 2x2 figures are the roofline numerator ``bench.py`` uses (as
constants, checked against a fresh count by ``tests/test_opcount.py``).  The
oracle's own timestep
(``oracle.step.timestep``, which restates timestep.py:65-199 and
solver.py:329-771) is run once on arrays of :class:`Counted`, an ndarray
subclass that counts every floating-point element operation NumPy performs
on it, attributed to the phase that is running:

* ``flops``: add, subtract, multiply, divide, negate, abs, min/max, square
  (an FMA would count 2), including reductions (``n - 1`` per reduced row),
  scans and ``ufunc.at`` scatters;
* ``sfu``: transcendental and root calls (exp, log, sqrt, arctan2, power,
  ...), one per element, counted apart from the flops;
* comparisons, selects, gathers and integer work are not counted.

The matrix exponentials are the one exception.  The reference runs a fixed
18-trip masked squaring loop for every matrix (transitions.py:181); the
algorithm needs ``s`` squarings for a matrix of norm 2^s (what this build's
kernel does), so ``expm_flops`` counts each matrix's Pade(6,6) evaluation, LU
solve and its own ``s`` squarings from the operation counts of those steps.

Phases: nearest (geometry.py:60-262), tm_kinetics (transitions.py:516-625),
xb_kinetics (:1081-1245), residual, jvp, precond and cg_vector (the Newton-CG
solve, solver.py:329-427), metrics (metrics_fn.py:154-417), tables (the 27
tropomyosin and 400 crossbridge generators and their expm,
transitions.py:434-513, 632-922) and absorbing (the metrics' absorbing-chain
expm, :1029-1078).  Tables and absorbing are counted per build: a kernel
that holds (pCa, lattice spacing) fixed builds them once per condition.
"""
from __future__ import annotations

import contextlib
from collections import defaultdict

import numpy as np

from . import physics as ph
from . import step as OS

_FLOP_UFUNCS = {'add', 'subtract', 'multiply', 'divide', 'true_divide', 'negative', 'absolute', 'fabs',
                'maximum', 'minimum', 'fmax', 'fmin', 'square', 'reciprocal', 'positive'}
_SFU_UFUNCS = {'exp', 'exp2', 'log', 'log2', 'log10', 'sqrt', 'arctan2', 'arctan', 'power', 'float_power',
               'sin', 'cos', 'tanh', 'expm1', 'log1p', 'cbrt'}

_state = {'phase': None, 'counts': None}


def _bump(kind, n):
    if _state['counts'] is not None and _state['phase'] is not None and n > 0:
        _state['counts'][_state['phase']][kind] += int(n)


def _plain(x):
    return x.view(np.ndarray) if isinstance(x, Counted) else x


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, Counted):
        return x.view(Counted)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


class Counted(np.ndarray):
    """An ndarray whose floating-point element operations are counted."""

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        args = [_plain(x) for x in inputs]
        if 'out' in kwargs:
            kwargs['out'] = tuple(_plain(o) for o in kwargs['out'])
        result = getattr(ufunc, method)(*args, **kwargs)
        floating = any(np.issubdtype(np.asarray(a).dtype, np.floating) for a in args
                       if isinstance(a, (np.ndarray, np.generic, float)))
        if floating:
            kind = 'flops' if ufunc.__name__ in _FLOP_UFUNCS else ('sfu' if ufunc.__name__ in _SFU_UFUNCS else None)
            if ufunc.__name__ == 'matmul' and method == '__call__':
                a, b = np.asarray(args[0]), np.asarray(args[1])
                _bump('flops', 2 * np.asarray(result).size * a.shape[-1])
            elif kind is not None:
                if method == '__call__':
                    _bump(kind, np.asarray(result).size)
                elif method in ('reduce',):
                    a = np.asarray(args[0])
                    _bump(kind, a.size - np.asarray(result).size)
                elif method in ('accumulate',):
                    _bump(kind, np.asarray(args[0]).size)
                elif method == 'at':
                    _bump(kind, np.size(args[1]) if not isinstance(args[1], tuple) else np.size(args[1][0]))
        if method == 'at':
            return None
        return _wrap(result)

    def __array_function__(self, func, types, args, kwargs):
        # NumPy's own implementation on the counted arrays, so that the ufuncs
        # it applies inside (np.sum, np.diff, np.cumsum, np.mean, ...) are counted
        return _wrap(super().__array_function__(func, types, args, kwargs))


@contextlib.contextmanager
def phase(name):
    prev = _state['phase']
    _state['phase'] = name
    try:
        yield
    finally:
        _state['phase'] = prev


def expm_flops(n: int, s: np.ndarray) -> int:
    """Flops of expm_pade6 (transitions.py:99-190) on matrices of size n with
    squaring counts s: the 1-norm, the scaling, three products for A^2, A^4,
    A^6 and one for U, the V and inner sums, the LU with partial pivoting of
    (V - U) and its solve for the n columns of (V + U), then s squarings and
    the row renormalisation."""
    s = np.asarray(s, dtype=np.int64)
    mm = 2 * n ** 3 - n ** 2                      # one n x n product
    norm = n * n + (n * n - n) + (n - 1)          # abs, row sums, max
    scale = n * n
    sums = 2 * n * n + 3 * n * n + 3 * n * n      # V - U, V + U; inner (3 terms); V (4 terms)
    lu = sum(2 * (n - k - 1) * (n - k - 1) + (n - k - 1) + 2 * (n - k - 1) * n for k in range(n))
    back = n * n * (n - 1) + n * n                # back substitution, one division per entry
    renorm = n * (n - 1) + n * n
    per = norm + scale + 4 * mm + sums + lu + back + renorm
    return int(per * s.size + mm * int(s.sum()))


class _Tracer:
    """Runs the oracle's functions under the phase each belongs to, counting calls."""

    def __init__(self):
        self.saved = []
        self.calls = defaultdict(int)

    def patch(self, owner, name, label):
        fn = getattr(owner, name)
        calls = self.calls

        def traced(*a, **k):
            calls[label] += 1
            with phase(label):
                return fn(*a, **k)
        self.saved.append((owner, name, fn))
        setattr(owner, name, traced)

    def restore(self):
        for owner, name, fn in reversed(self.saved):
            setattr(owner, name, fn)
        self.saved.clear()


def count_timestep(topo, row, c: OS.Condition, z: float, pCa: float, ls: float, u_thin, u_xb,
                   n_newton=4, n_cg=6, dt=np.float32, dt_ms=1.0, K_lat=None, d_ref=None):
    """Counts of one oracle timestep from condition ``c`` (fixed spacing when
    ``K_lat`` is None).  Returns (counts {phase: {'flops', 'sfu'}}, next
    condition, extras of the step)."""
    dt = np.dtype(dt).type
    p = ph.param_dict(row, dt)
    pre = ph.Preconditioner(topo, p, dt)
    counts = defaultdict(lambda: defaultdict(int))
    _state['counts'] = counts
    tr = _Tracer()
    try:
        # table builds (the generators counted here, their expm by expm_flops)
        with phase('tables'):
            Q_tm = ph.tm_Q27(p, _wrap(np.asarray(dt(pCa))), dt)
            Q_xb = ph.xb_Q_bins(topo, p, _wrap(np.asarray(dt(pCa))), dt(ls), dt)
        P_tm, s_tm = ph.expm_pade6(np.asarray(_plain(Q_tm)) * dt(dt_ms), with_s=True)
        P_xb, s_xb = ph.expm_pade6(np.asarray(_plain(Q_xb)) * dt(dt_ms), with_s=True)
        counts['tables']['flops'] += expm_flops(4, s_tm) + expm_flops(6, s_xb)
        Pa, s_a = ph.expm_pade6(ph.absorbing(np.asarray(_plain(Q_xb))) * dt(dt_ms), with_s=True)
        counts['absorbing']['flops'] += expm_flops(6, s_a)
        tab = OS.Tables(P_tm, P_xb, s_tm, s_xb)
        tr.patch(ph, 'nearest_sites', 'nearest')
        tr.patch(ph, 'thin_transitions', 'tm_kinetics')
        tr.patch(ph, 'thick_transitions', 'xb_kinetics')
        tr.patch(ph.ForceModel, 'residual', 'residual')
        tr.patch(ph.ForceModel, 'radial', 'residual')
        tr.patch(ph.ForceModel, 'jvp', 'jvp')
        tr.patch(ph.ForceModel, 'J_dd', 'residual')
        tr.patch(ph.Preconditioner, '__call__', 'precond')
        tr.patch(OS, 'metrics', 'metrics')
        cw = c.copy()
        for f in ('thick_x', 'thin_x', 'xb_dist'):
            setattr(cw, f, _wrap(getattr(cw, f)))
        thin_cum = OS.thin_rest_cumsum(topo, dt)
        with phase('cg_vector'):  # whatever the solver does outside the named pieces
            nc, row_m, ex = OS.timestep(topo, p, cw, z, pCa, ls, 0.0, _wrap(np.asarray(u_thin, dt)),
                                        _wrap(np.asarray(u_xb, dt)), tab, n_newton, n_cg, dt, pre, dt_ms,
                                        K_lat=K_lat, d_ref=d_ref, P_abs=Pa, thin_rest_cum=thin_cum)
    finally:
        tr.restore()
        _state['counts'] = None
    out = {k: dict(v) for k, v in counts.items()}
    out['calls'] = dict(tr.calls)
    tr.calls.clear()
    for f in ('thick_x', 'thin_x', 'xb_dist'):
        setattr(nc, f, np.asarray(_plain(getattr(nc, f))))
    return out, nc, ex


def unit_counts(topo, row, pCa=4.5, z=900.0, ls=14.0, T=20, key=None, n_newton=4, n_cg=6):
    """Counts per unit of work over T steps of a fixed-spacing isometric run:
    per step (nearest sites, both kinetics, the metrics, the first residual),
    per Newton iteration (one residual, n_cg JVPs, n_cg + 1 preconditioner
    applications, the CG vector updates), per table build and per absorbing
    table build.  A step then costs per_step + iterations x per_newton flops,
    and a launch adds one build of each table per (pCa, spacing) it meets."""
    from . import prng
    dt = np.float32
    p = ph.param_dict(row, dt)
    pre = ph.Preconditioner(topo, p, dt)
    c = OS.initial_condition(topo, p, z, n_newton, n_cg, dt, pre)
    key = prng.split(prng.PRNGKey(0), 1)[0] if key is None else np.asarray(key, np.uint32)
    tot = defaultdict(lambda: defaultdict(float))
    calls = defaultdict(int)
    iters = 0
    build = None
    for t in range(T):
        ut, ux, key = prng.step_uniforms(key, topo.n_sites_total, topo.total_xbs)
        cnt, c, ex = count_timestep(topo, row, c, z, pCa, ls, ut, ux, n_newton, n_cg)
        iters += ex['iters']
        for k, v in cnt.pop('calls').items():
            calls[k] += v
        if build is None:
            build = {k: int(cnt[k]['flops']) for k in ('tables', 'absorbing')}
        for ph_name, kinds in cnt.items():
            for kind, v in kinds.items():
                tot[ph_name][kind] += v
    per_call = {k: {kind: v / max(calls[k], 1) for kind, v in tot[k].items()}
                for k in ('residual', 'jvp', 'precond')}
    fixed_phases = ('nearest', 'tm_kinetics', 'xb_kinetics', 'metrics')

    def f(kind):
        step = sum(tot[k][kind] for k in fixed_phases) / T + per_call['residual'].get(kind, 0.0)
        newton = (per_call['residual'].get(kind, 0.0) + n_cg * per_call['jvp'].get(kind, 0.0)
                  + (n_cg + 1) * per_call['precond'].get(kind, 0.0)
                  + (tot['cg_vector'][kind] / iters if iters else 0.0))
        return step, newton
    step_f, newton_f = f('flops')
    step_s, newton_s = f('sfu')
    return {'per_step_flops': step_f, 'per_newton_flops': newton_f, 'per_step_sfu': step_s,
            'per_newton_sfu': newton_s, 'table_build_flops': build['tables'],
            'absorbing_build_flops': build['absorbing'], 'mean_newton_iters': iters / T, 'steps': T,
            'phases_per_step': {k: {kind: v / T for kind, v in kinds.items()} for k, kinds in tot.items()
                                if k not in ('tables', 'absorbing')},
            'calls': dict(calls)}


if __name__ == '__main__':
    import json
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    s_, d_ = get_skeletal_params()
    for n in (1, 2, 3, 4):
        t_ = SarcTopology.create(n, n, s_, d_)
        print(json.dumps({'lattice': f'{n}x{n}', **unit_counts(t_, d_.param_row())}))
