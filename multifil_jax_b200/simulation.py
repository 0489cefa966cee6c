"""``run()``: the reference's public entry point on the CUDA engine.

Mirrors ``multifil_jax/simulation.py:754-1165`` (sweep expansion, per-field
parameter tables, key split, Poisson lattice-spacing pre-computation, result
data cube, residual warning); the result type is
:class:`multifil_jax_b200.result.SimulationResult`.  The per-condition time loop --
the reference's ``jit(vmap(scan(timestep)))`` -- runs in the fused sm_100a
kernel through :mod:`multifil_jax_b200.engine`; there is no CPU path.

Sweep axes are Cartesian-producted in the reference's fixed order (z_line,
pCa, lattice_spacing, K_lat, nu, dynamic_params fields / candidates) and
results come back shaped ``(sweep_1, ..., replicates, time)``.
"""
from __future__ import annotations

import time
import warnings
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple, Union

import numpy as np

from .params import DYNAMIC_FIELDS, DynamicParams, StaticParams, N_PARAMS
from .topology import SarcTopology
from .result import MetricsDict, SimulationResult
from .subpopulation import ResolvedSubpop, Subpopulation  # noqa: F401

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

BATCH_BUCKETS = (1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384)

PRECISIONS = ('float32', 'mixed')


def get_bucket_size(actual_size: int) -> int:
    """Next power-of-two bucket (reference ``simulation.py:434-450``).

    The CUDA engine needs no shape buckets; this is kept because the
    reference's returned ``rng_key`` is the last key of the padded batch.
    """
    for b in BATCH_BUCKETS:
        if b >= actual_size:
            return b
    return actual_size


# ---------------------------------------------------------------------------
# sweep expansion (host glue; simulation.py:848-1048)
# ---------------------------------------------------------------------------

@dataclass
class BatchPlan:
    """Every per-condition input of one run(), flattened to B = grid x replicates rows."""
    n_steps: int
    dt: float
    params: np.ndarray        # [B, 44] float32
    z: np.ndarray             # [B, T] float32
    pCa: np.ndarray
    ls: np.ndarray
    keys: np.ndarray          # [B, 2] uint32
    K_lat: np.ndarray         # [B] float32, already x n_thick when dynamic
    nu: np.ndarray            # [B] float32
    dynamic_ls: bool
    grid_shape: Tuple[int, ...]
    replicates: int
    axis_names: List[str]
    coords: Dict[str, list]
    rng_key: np.ndarray
    topology_config: Dict = field(default_factory=dict)
    subpop: Optional['ResolvedSubpop'] = None  # per-condition populations (None: one population)

    @property
    def total(self) -> int:
        return self.params.shape[0]

    @property
    def const_drivers(self) -> bool:
        """Whether z, pCa and ls each hold one value per condition for every
        step (time stride 0), so that [B] values can replace the traces."""
        return self.n_steps > 0 and all(a.ndim == 2 and a.strides[1] == 0 for a in (self.z, self.pCa, self.ls))


def _split_keys(seed: int, n: int) -> np.ndarray:
    from .engine import prng_key, prng_split
    if n == 0:
        return np.zeros((0, 2), np.uint32)
    return prng_split(prng_key(seed), n)


def plan_batch(topology: SarcTopology, duration_ms: float = 1000.0, dt: float = 1.0,
               pCa=4.5, z_line=900.0, lattice_spacing=14.0, K_lat=None, nu=0.0, dynamic_params=None,
               static_params: Optional[StaticParams] = None, replicates: int = 1, rng_seed: int = 0,
               subpopulation=None) -> BatchPlan:
    """Expand run()'s arguments into per-condition arrays (no device work)."""
    if replicates < 1:
        raise ValueError("replicates must be >= 1")
    n_steps = int(duration_ms / dt)
    if dynamic_params is None or isinstance(dynamic_params, (dict, list)):
        base = DynamicParams()
    elif isinstance(dynamic_params, DynamicParams):
        base = dynamic_params
    else:
        raise ValueError(f"dynamic_params must be DynamicParams, dict, or list, got {type(dynamic_params)}")
    is_dyn = K_lat is not None

    def as_trace(v):
        a = np.asarray(v, dtype=float)
        return np.full(n_steps, float(a)) if a.ndim == 0 else a

    axes: List[Tuple[str, list]] = []
    wf_tables: Dict[str, np.ndarray] = {}
    wf_sweeps = set()
    ptables: Dict[str, np.ndarray] = {}
    paxis: Dict[str, str] = {}
    for name, value in (('z_line', z_line), ('pCa', pCa), ('lattice_spacing', lattice_spacing)):
        if isinstance(value, list):
            if not value:
                raise ValueError(f"{name} sweep list is empty")
            if all(np.ndim(v) == 0 for v in value):  # scalar sweep: one constant per value, broadcast in wave()
                wf_tables[name] = np.asarray(value, dtype=float).astype(np.float32)[:, None]
            else:
                rows = [as_trace(v) for v in value]
                if any(r.shape != (n_steps,) for r in rows):
                    raise ValueError(f"{name} trace length != n_steps {n_steps}")
                wf_tables[name] = np.stack(rows).astype(np.float32)
            trace_sweep = any(not isinstance(v, (int, float)) and np.asarray(v).ndim == 1
                              and len(np.asarray(v)) == n_steps for v in value)
            coords = ([np.asarray(wf_tables[name][i]) for i in range(len(value))] if trace_sweep
                      else list(value))
            axes.append((name, coords))
            wf_sweeps.add(name)
        else:
            arr = np.asarray(value)
            if arr.ndim > 0 and arr.shape[0] != n_steps:
                raise ValueError(f"{name} array length {arr.shape[0]} != n_steps {n_steps}")
            # a scalar stays one value (a [1, 1] table): held for every step
            wf_tables[name] = (np.full((1, 1), float(arr), np.float32) if arr.ndim == 0
                               else as_trace(value).astype(np.float32)[None, :])
    if isinstance(K_lat, list):
        axes.append(('K_lat', list(K_lat)))
    if isinstance(nu, list):
        axes.append(('nu', list(nu)))
    if isinstance(dynamic_params, list):
        if not dynamic_params:
            raise ValueError("dynamic_params candidate list is empty")
        axes.append(('candidates', list(range(len(dynamic_params)))))
        for name in DYNAMIC_FIELDS:
            ptables[name] = np.stack([np.asarray(getattr(dp, name), np.float32) for dp in dynamic_params])
            paxis[name] = 'candidates'
    elif isinstance(dynamic_params, dict):
        for pname, pval in dynamic_params.items():
            if pname not in DYNAMIC_FIELDS:
                raise ValueError(f"Unknown dynamic_params field '{pname}'. Valid: {list(DYNAMIC_FIELDS)}")
            if isinstance(pval, list):
                axes.append((pname, list(pval)))
                ptables[pname] = np.asarray(pval, np.float32)
                paxis[pname] = pname
    elif isinstance(dynamic_params, DynamicParams):
        for name in DYNAMIC_FIELDS:
            arr = np.asarray(getattr(dynamic_params, name))
            if arr.ndim > 0 and arr.shape[0] > 1:
                axes.append((name, list(arr.tolist())))
                ptables[name] = arr.astype(np.float32)
                paxis[name] = name
    # a list of Subpopulations is a candidate-style sweep axis (simulation.py:945-953)
    if isinstance(subpopulation, list):
        if isinstance(dynamic_params, list):
            raise ValueError("Cannot sweep a dynamic_params list and a subpopulation list simultaneously "
                             "(both are candidate-style axes).")
        if not subpopulation:
            raise ValueError("subpopulation list is empty")
        axes.append(('subpopulation', list(range(len(subpopulation)))))

    if axes:
        grids = np.meshgrid(*[np.arange(len(c)) for _, c in axes], indexing='ij')
        batch = grids[0].size
        flat = {name: np.repeat(g.reshape(-1), replicates) for (name, _), g in zip(axes, grids)}
    else:
        batch = 1
        flat = {}
    total = batch * replicates
    grid_shape = tuple(len(c) for _, c in axes)
    axis_names = [n for n, _ in axes] + ['replicates', 'time']
    coords = {n: c for n, c in axes}
    coords['replicates'] = list(range(replicates))
    coords['time'] = (np.arange(n_steps) * dt).tolist()

    def wave(name):
        tab = wf_tables[name]
        if name in wf_sweeps:
            return np.broadcast_to(tab[flat[name]], (total, n_steps))
        return np.broadcast_to(tab[0], (total, n_steps))
    # read-only broadcast views: a driver constant in time has time stride 0
    # (BatchPlan.const_drivers), and nothing [B, T] is materialised for it
    z_b, p_b, l_b = wave('z_line'), wave('pCa'), wave('lattice_spacing')
    if isinstance(K_lat, list):
        K_b = np.asarray(K_lat, np.float32)[flat['K_lat']]
    elif is_dyn:
        K_b = np.full(total, float(K_lat), np.float32)
    else:
        K_b = np.zeros(total, np.float32)
    if isinstance(nu, list):
        nu_b = np.asarray(nu, np.float32)[flat['nu']]
    else:
        nu_b = np.full(total, float(nu), np.float32)
    if is_dyn:
        K_b = (K_b * np.float32(topology.n_thick)).astype(np.float32)
    ls_is_trace = not isinstance(lattice_spacing, list) and np.asarray(lattice_spacing).ndim > 0
    nonzero_nu = any(v != 0.0 for v in nu) if isinstance(nu, list) else float(nu) != 0.0
    if not is_dyn and not ls_is_trace and nonzero_nu and n_steps > 0:
        d0 = l_b[:, 0:1]
        l_b = (d0 * (z_b[:, 0:1] / z_b) ** nu_b[:, None]).astype(np.float32)

    # one constant row, then the swept columns
    row = np.empty(N_PARAMS, np.float32)
    for j, name in enumerate(DYNAMIC_FIELDS):
        if isinstance(dynamic_params, dict) and name in dynamic_params and name not in paxis:
            row[j] = float(dynamic_params[name])
        else:
            row[j] = float(np.asarray(getattr(base, name)).reshape(-1)[0])
    params = np.tile(row, (total, 1))
    for j, name in enumerate(DYNAMIC_FIELDS):
        if name in paxis:
            params[:, j] = ptables[name][flat[paxis[name]]]
    assert params.shape == (total, N_PARAMS)
    from .subpopulation import resolve_subpopulation
    subpop = resolve_subpopulation(subpopulation, topology, params,
                                   flat['subpopulation'] if isinstance(subpopulation, list) else None)
    keys = _split_keys(rng_seed, total)
    padded = get_bucket_size(total)
    if padded > total:
        last_key = _split_keys(rng_seed + 1, padded - total)[-1]
    else:
        last_key = keys[-1]
    tcfg = {'n_thick': topology.n_thick, 'n_crowns': topology.n_crowns, 'n_thin': topology.n_thin,
            'n_sites': topology.n_sites, 'n_titin': topology.n_titin, 'total_xbs': topology.total_xbs,
            'n_faces_per_thin': topology.n_faces_per_thin}
    if is_dyn:
        tcfg['K_lat'] = K_lat
        tcfg['K_lat_eff'] = (float(K_lat * topology.n_thick) if not isinstance(K_lat, list)
                             else [float(k * topology.n_thick) for k in K_lat])
        tcfg['nu'] = nu
    return BatchPlan(n_steps=n_steps, dt=float(dt), params=params, z=z_b, pCa=p_b, ls=l_b, keys=keys,
                     K_lat=K_b, nu=nu_b, dynamic_ls=is_dyn, grid_shape=grid_shape, replicates=replicates,
                     axis_names=axis_names, coords=coords, rng_key=last_key, topology_config=tcfg,
                     subpop=subpop)


def assemble_result(plan: BatchPlan, metrics: np.ndarray, static_params: StaticParams, rng_seed: int,
                    verbose: bool = False, key_major: bool = False) -> SimulationResult:
    """[B, 52, T] metrics ([52, B, T] with ``key_major``) -> data-cube
    SimulationResult with the residual warning.  Float metrics are views of
    ``metrics`` (no copies); ``newton_iters`` is converted to int32."""
    shape = plan.grid_shape + (plan.replicates, plan.n_steps)
    md = MetricsDict()
    for k, name in enumerate(METRIC_KEYS):
        v = (metrics[k] if key_major else metrics[:, k, :]).reshape(shape)
        md[name] = v.astype(np.int32) if name == 'newton_iters' else np.asarray(v, dtype=np.float32)
    max_res = float(np.max(md['solver_residual'])) if md['solver_residual'].size else 0.0
    tol = static_params.solver_residual_tol
    if max_res > tol:
        warnings.warn(f"Solver max residual {max_res:.2f} pN exceeds threshold {tol} pN "
                      f"(set via StaticParams.solver_residual_tol)")
    if verbose:
        print(f"Result shape: {md['axial_force'].shape}")
        print(f"Max solver residual: {max_res:.4f} pN")
    return SimulationResult(
        metrics=md, rng_key=plan.rng_key, z_line=plan.z.reshape(shape), pCa=plan.pCa.reshape(shape),
        lattice_spacing=plan.ls.reshape(shape), final_state=None, metadata={'master_seed': rng_seed},
        dt=plan.dt, name="run", grid_shape=plan.grid_shape, axis_names=plan.axis_names,
        coords=plan.coords, topology_config=plan.topology_config)


def run(topology: SarcTopology, duration_ms: float = 1000.0, dt: float = 1.0,
        pCa: Union[float, List[float], np.ndarray] = 4.5,
        z_line: Union[float, List[float], np.ndarray] = 900.0,
        lattice_spacing: Union[float, List[float], np.ndarray] = 14.0,
        K_lat: Union[float, List[float], None] = None, nu: Union[float, List[float]] = 0.0,
        dynamic_params=None, static_params: Optional[StaticParams] = None, replicates: int = 1,
        rng_seed: int = 0, unroll: int = 1, minibatch_size: Optional[int] = "auto", verbose: bool = False,
        subpopulation=None, *, precision: str = 'float32', device: Optional[int] = None,
        chunk_steps: int = 0) -> SimulationResult:
    """Run a muscle simulation sweep on the GPU (reference ``simulation.py:754-1165``).

    Same arguments, errors and result as the reference; ``unroll`` is accepted
    and has no effect (the fused kernel has no scan to unroll).  Keyword-only
    extensions: ``precision`` ``'float32'`` reproduces the reference's
    single-precision arithmetic, ``'mixed'`` stores node displacements and
    keeps the Newton residual test and large-norm expm squarings in float64;
    ``device`` picks the CUDA device; ``chunk_steps`` > 0 splits the time loop
    into launches of that many steps replayed from a CUDA graph.
    """
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}")
    sp = static_params if static_params is not None else StaticParams()
    plan = plan_batch(topology, duration_ms, dt, pCa, z_line, lattice_spacing, K_lat, nu, dynamic_params,
                      sp, replicates, rng_seed, subpopulation)
    if verbose:
        print(f"Grid shape: {plan.grid_shape}, axes: {plan.axis_names}, total: {plan.total}")
    from .engine import execute_plan, MF_STATUS_NONFINITE
    status = np.zeros(plan.total, np.int32)
    metrics = execute_plan(topology, plan, sp, precision=precision, device=device,
                           minibatch_size=minibatch_size, chunk_steps=chunk_steps, key_major=True,
                           status_out=status)
    bad = np.flatnonzero(status & MF_STATUS_NONFINITE)
    if bad.size:
        warnings.warn(f"{bad.size} of {plan.total} conditions produced a non-finite Newton update or residual "
                      f"(first: condition {int(bad[0])}); the update was zeroed, as the reference does")
    return assemble_result(plan, metrics, sp, rng_seed, verbose, key_major=True)


def run_conditions(conditions: List[dict], *, static_params: Optional[StaticParams] = None,
                   precision: str = 'float32', device: Optional[int] = None, chunk_steps: int = 0,
                   autotune: bool = False) -> List[MetricsDict]:
    """Run independent conditions on different lattices and durations in one launch.

    The reference needs one ``run()`` per (lattice, n_steps) pair, both being
    JIT shapes; here every condition is one CTA of the same persistent launch,
    grouped by CTA size.  Each condition is a dict with ``topology``,
    ``duration_ms``, and optionally ``dt`` (1.0), ``pCa`` (4.5), ``z_line``
    (900.0), ``lattice_spacing`` (14.0), ``K_lat`` (None: fixed spacing; else
    the reference's per-thick-filament value, multiplied by ``n_thick`` as in
    ``simulation.py:1002-1003``), ``nu`` (0.0), ``dynamic_params`` (the
    skeletal defaults) and ``key`` (uint32[2]; default ``split(PRNGKey(0), B)[i]``).
    Scalars only: one constant driver value per condition; the parameter
    row itself keeps the DynamicParams constants, as ``run()`` does (the
    initial equilibrium uses them, ``simulation.py:633-642``).  Either every
    condition gives ``K_lat`` or none does.  ``autotune`` measures the CTA size
    of every distinct lattice first (``autotune.autotune_many``).

    Returns one MetricsDict per condition, each key an array of that
    condition's ``n_steps``.
    """
    import torch
    from .engine import get_engine, MF_FLAG_DYNAMIC_LS, MF_FLAG_PRECISE, prng_key, prng_split
    from .params import get_skeletal_params
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}")
    sp = static_params if static_params is not None else StaticParams()
    B = len(conditions)
    if B == 0:
        return []
    dyn = [c.get('K_lat') is not None for c in conditions]
    if any(dyn) and not all(dyn):
        raise ValueError("either every condition gives K_lat (dynamic lattice spacing) or none does")
    default_keys = prng_split(prng_key(0), B)
    _, d_default = get_skeletal_params()
    steps = []
    for c in conditions:
        dt = float(c.get('dt', 1.0))
        if dt <= 0:
            raise ValueError("dt must be positive")
        steps.append(int(float(c['duration_ms']) / dt))
    if min(steps) < 1:
        raise ValueError("every condition needs at least one timestep")
    T = max(steps)
    P = np.zeros((B, 44), np.float32)
    # one driver value per condition, held for every step (MF_FLAG_CONST_DRIVERS)
    Z = np.zeros(B, np.float32)
    PC = np.zeros(B, np.float32)
    L = np.zeros(B, np.float32)
    K = np.zeros(B, np.float32)
    NU = np.zeros(B, np.float32)
    DT = np.zeros(B, np.float32)
    KEYS = np.zeros((B, 2), np.uint32)
    for i, c in enumerate(conditions):
        dp = c.get('dynamic_params') or d_default
        z, pca, ls = float(c.get('z_line', 900.0)), float(c.get('pCa', 4.5)), float(c.get('lattice_spacing', 14.0))
        P[i] = dp.param_row()  # the constants, as run() passes them
        Z[i], PC[i], L[i] = z, pca, ls
        if dyn[i]:
            K[i] = np.float32(float(c['K_lat']) * c['topology'].n_thick)
        NU[i] = float(c.get('nu', 0.0))
        DT[i] = float(c.get('dt', 1.0))
        KEYS[i] = np.asarray(c['key'], np.uint32) if c.get('key') is not None else default_keys[i]
    topos = [c['topology'] for c in conditions]
    eng = get_engine(device)
    dev = torch.device('cuda', eng.device)
    flags = (MF_FLAG_DYNAMIC_LS if all(dyn) else 0) | (MF_FLAG_PRECISE if precision == 'mixed' else 0)
    from .engine import upload, host_metrics
    if autotune:
        from .autotune import autotune_many, choose_batch_sizes
        picks = autotune_many(topos, precision=precision, device=device, dynamic_ls=all(dyn))
        Ts = min(T, 20)  # the batch itself, a few steps long

        def run_short():
            with torch.cuda.device(dev):
                a = upload(dev, P, Z, PC, L, np.minimum(np.asarray(steps, np.int32), Ts),
                           KEYS.view(np.int32), K, NU, DT)
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                eng.run_batch(topos, *a[:6], K_lat=a[6], nu=a[7], dt=a[8], n_newton=sp.n_newton_steps,
                              n_cg=sp.n_cg_steps, flags=flags, chunk_steps=chunk_steps,
                              residual_warn=sp.solver_residual_tol, n_time=Ts)
                torch.cuda.synchronize(dev)
                return time.perf_counter() - t0
        choose_batch_sizes(topos, picks, run_short, precision=precision, device=device)
    with torch.cuda.device(dev):
        dP, dZ, dPC, dL, dN, dKY, dK, dNU, dDT = upload(dev, P, Z, PC, L, np.asarray(steps, np.int32),
                                                        KEYS.view(np.int32), K, NU, DT)
        hm = host_metrics(len(conditions), T)  # written by the kernels over the bus
        eng.run_batch(topos, dP, dZ, dPC, dL, dN, dKY, K_lat=dK, nu=dNU, dt=dDT,
                      n_newton=sp.n_newton_steps, n_cg=sp.n_cg_steps, flags=flags, chunk_steps=chunk_steps,
                      residual_warn=sp.solver_residual_tol, metrics_out=hm, n_time=T)
        torch.cuda.current_stream(dev).synchronize()
        m = hm.numpy()
    out = []
    for i, n in enumerate(steps):
        md = MetricsDict()
        for k, name in enumerate(METRIC_KEYS):
            v = m[i, k, :n]
            md[name] = v.astype(np.int32) if name == 'newton_iters' else v.copy()
        out.append(md)
    return out


__all__ = ['run', 'run_conditions', 'SimulationResult', 'MetricsDict', 'METRIC_KEYS', 'BATCH_BUCKETS',
           'get_bucket_size', 'plan_batch', 'assemble_result', 'BatchPlan']
