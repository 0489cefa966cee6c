"""The public halves of a timestep on caller-owned states.

Drop-in for the reference's functional timestep API (``timestep.py:65-199``,
``core/state.py:69-262``, ``kernels/geometry.py:186-262``,
``kernels/solver.py:663-771``): ``realize_state``, ``update_nearest_neighbors``,
``kinetics_step``, ``solve_equilibrium``, ``timestep`` and
``create_and_equilibrate``, for coupled solvers that step several sarcomeres
and solve between kinetics and equilibrium themselves.

A :class:`State` holds torch CUDA tensors in the reference's layout, either
one state (``thick.axial`` of shape ``(n_thick, n_crowns)``) or a batch of B
states (a leading axis of B on every field).  Each call runs ``mf_step_states``
(one CTA per state, the fused kernel's own phase code) on copies of the
inputs and returns new tensors, so the functions stay pure as in the
reference.  Arithmetic is the reference's float32.  Random keys are
``uint32[2]`` (or ``[B, 2]``) arrays; the transitions advance them exactly as
``jax.random`` does (``timestep.py:120,125``).
"""
from __future__ import annotations

import ctypes
from typing import NamedTuple, Optional, Sequence

import numpy as np

from .engine import (EngineError, get_engine, device_pops, MF_FLAG_ORIGINAL_PRNG, N_PARAMS, MF_POP_EXPLICIT,
                     MF_POP_XB, MF_POP_TM)
from .params import DynamicParams, DYNAMIC_FIELDS

MF_PHASE_NEAREST = 1
MF_PHASE_TRANSITIONS = 2
MF_PHASE_EQUILIBRIUM = 4
MF_PHASE_KINETICS = MF_PHASE_NEAREST | MF_PHASE_TRANSITIONS
MF_PHASE_TIMESTEP = MF_PHASE_KINETICS | MF_PHASE_EQUILIBRIUM


class ThickState(NamedTuple):
    axial: 'object'           # (n_thick, n_crowns) float32
    xb_states: 'object'       # (n_thick, n_crowns, n_xb_per_crown) int8
    xb_bound_to: 'object'     # same, int32 (-1 unbound)
    xb_nearest_bs: 'object'   # same, int32
    xb_distances: 'object'    # (..., 2) float32: axial offset, radial spacing


class ThinState(NamedTuple):
    axial: 'object'           # (n_thin, n_sites) float32
    tm_states: 'object'       # (n_thin, n_sites) int8
    bound_to: 'object'        # (n_thin, n_sites) int32 (-1 unbound)


class State(NamedTuple):
    thick: ThickState
    thin: ThinState


class Drivers(NamedTuple):
    """Per-step overrides of pCa, z_line and lattice spacing; NaN = the constant."""
    pCa: 'object' = float('nan')
    z_line: 'object' = float('nan')
    lattice_spacing: 'object' = float('nan')


class mf_state_batch(ctypes.Structure):
    _fields_ = [
        ('B', ctypes.c_int32), ('topo_id', ctypes.c_int32), ('phases', ctypes.c_int32), ('flags', ctypes.c_int32),
        ('dt', ctypes.c_float), ('n_newton', ctypes.c_int32), ('n_cg', ctypes.c_int32),
        ('thick_axial', ctypes.c_void_p), ('xb_states', ctypes.c_void_p), ('xb_bound_to', ctypes.c_void_p),
        ('xb_nearest_bs', ctypes.c_void_p), ('xb_distances', ctypes.c_void_p), ('thin_axial', ctypes.c_void_p),
        ('tm_states', ctypes.c_void_p), ('thin_bound_to', ctypes.c_void_p), ('keys', ctypes.c_void_p),
        ('params', ctypes.c_void_p), ('pCa', ctypes.c_void_p), ('z_line', ctypes.c_void_p),
        ('lattice_spacing', ctypes.c_void_p), ('K_lat', ctypes.c_void_p), ('d_ref', ctypes.c_void_p),
        ('residual_out', ctypes.c_void_p), ('ls_out', ctypes.c_void_p), ('iters_out', ctypes.c_void_p),
        ('status_out', ctypes.c_void_p),
        ('n_pops', ctypes.c_int32), ('pop_flags', ctypes.c_int32), ('label_stride', ctypes.c_int32),
        ('pop_params', ctypes.c_void_p), ('pop_frac', ctypes.c_void_p), ('xb_label', ctypes.c_void_p),
        ('tm_label', ctypes.c_void_p), ('u_thin', ctypes.c_void_p), ('u_xb', ctypes.c_void_p),
    ]


def _torch():
    import torch
    return torch


def _bind(lib):
    fn = lib.mf_step_states
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(mf_state_batch), ctypes.c_void_p]
    return fn


def _device(device):
    torch = _torch()
    if not torch.cuda.is_available():
        raise EngineError("multifil_jax_b200 needs a CUDA device; none is available")
    return torch.device('cuda', torch.cuda.current_device() if device is None else device)


def realize_state(topology, constants: DynamicParams, z_line: float, pCa: float, lattice_spacing: float,
                  batch: Optional[int] = None, device=None) -> State:
    """Initial state (reference ``core/state.py:191-262``): crowns at their
    offsets, binding sites at ``z_line - binding_offsets``, every head and site
    in state 0, nothing bound.  ``batch``: B identical states."""
    torch = _torch()
    dev = _device(device)
    t = topology
    lead = () if batch is None else (int(batch),)
    xshape = lead + (t.n_thick, t.n_crowns, t.n_xb_per_crown)

    def rep(a, dtype):
        x = torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
        return x.expand(lead + tuple(x.shape)).contiguous() if lead else x
    thick = ThickState(
        axial=rep(np.asarray(t.crown_offsets, np.float32), torch.float32),
        xb_states=torch.zeros(xshape, dtype=torch.int8, device=dev),
        xb_bound_to=torch.full(xshape, -1, dtype=torch.int32, device=dev),
        xb_nearest_bs=torch.zeros(xshape, dtype=torch.int32, device=dev),
        xb_distances=torch.zeros(xshape + (2,), dtype=torch.float32, device=dev))
    thin = ThinState(
        axial=rep((np.float32(z_line) - np.asarray(t.binding_offsets, np.float32)).astype(np.float32), torch.float32),
        tm_states=torch.zeros(lead + (t.n_thin, t.n_sites), dtype=torch.int8, device=dev),
        bound_to=torch.full(lead + (t.n_thin, t.n_sites), -1, dtype=torch.int32, device=dev))
    return State(thick, thin)


def _batch_of(state: State, topology) -> int:
    ax = state.thick.axial
    if tuple(ax.shape[-2:]) != (topology.n_thick, topology.n_crowns):
        raise ValueError(f"thick.axial shape {tuple(ax.shape)} does not match the topology")
    if ax.dim() == 2:
        return 0
    if ax.dim() == 3:
        return int(ax.shape[0])
    raise ValueError("a State has one optional leading batch axis")


def _rows(constants, B: int) -> np.ndarray:
    """DynamicParams (scalar or per-state fields) -> [B, 44] float32 rows."""
    cols = []
    for name in DYNAMIC_FIELDS:
        v = np.asarray(getattr(constants, name), np.float32).reshape(-1)
        if v.size not in (1, B):
            raise ValueError(f"DynamicParams field {name} has {v.size} values for {B} states")
        cols.append(np.broadcast_to(v, (B,)))
    return np.ascontiguousarray(np.stack(cols, axis=1), dtype=np.float32)


def _per_state(v, B: int, name: str) -> np.ndarray:
    a = np.asarray(v, np.float32).reshape(-1)
    if a.size not in (1, B):
        raise ValueError(f"{name}: {a.size} values for {B} states")
    return np.ascontiguousarray(np.broadcast_to(a, (B,)), dtype=np.float32)


def _keys(rng_key, B: int):
    k = np.asarray(rng_key.cpu().numpy() if hasattr(rng_key, 'cpu') else rng_key, dtype=np.uint32)
    if k.shape == (2,):
        k = np.broadcast_to(k, (B, 2))
    if k.shape != (B, 2):
        raise ValueError(f"rng_key must be uint32[2] or [B, 2], got {k.shape}")
    return np.ascontiguousarray(k)


def _subpop_pops(xb_subpop, tm_subpop, topology, B: int):
    """The reference's (mode, constants_k, extra) tuples -> run_batch ``pops`` arrays."""
    from .subpopulation import ResolvedSubpop
    sub = [s for s in (xb_subpop, tm_subpop) if s is not None]
    if not sub:
        return None
    mode, ck, _ = sub[0]
    for s in sub[1:]:
        if s[0] != mode or len(s[1]) != len(ck):
            raise ValueError("xb_subpop and tm_subpop must share one mode and population list")
    if mode not in ('mean_field', 'explicit'):
        raise ValueError(f"unknown subpopulation mode '{mode}'")
    K = len(ck)
    rows = np.stack([_rows(c, B) for c in ck], axis=1)
    explicit = mode == 'explicit'
    frac = np.zeros((B, K), np.float32)
    xl = tl = None
    if not explicit:
        frac[:] = np.asarray(sub[0][2], np.float32).reshape(-1)[:K]
    else:
        def lab(s, n):
            if s is None:
                return np.zeros((B, n), np.int8)
            a = np.asarray(s[2].cpu().numpy() if hasattr(s[2], 'cpu') else s[2]).reshape(-1, n)
            return np.ascontiguousarray(np.broadcast_to(a, (B, n)), dtype=np.int8)
        xl, tl = lab(xb_subpop, topology.total_xbs), lab(tm_subpop, topology.n_sites_total)
    return ResolvedSubpop(K=K, explicit=explicit, xb=xb_subpop is not None, tm=tm_subpop is not None,
                          rows=rows.astype(np.float32), fractions=frac, xb_label=xl, tm_label=tl)


def _step(state: State, constants, topology, phases: int, drivers: Optional[Drivers] = None, rng_key=None,
          dt: float = 1.0, K_lat=None, d_ref=None, tolerance=None, n_newton_steps: int = 16, n_cg_steps: int = 6,
          xb_subpop=None, tm_subpop=None, partitionable: bool = True, uniforms=None):
    torch = _torch()
    B0 = _batch_of(state, topology)
    B = max(B0, 1)
    dev = state.thick.axial.device
    eng = get_engine(dev.index)
    fn = _bind(eng.lib)
    up = eng.upload(topology)
    X, S = topology.total_xbs, topology.n_sites_total
    flat = lambda t, dtype, n: t.detach().to(device=dev, dtype=dtype).reshape(B, n).clone().contiguous()
    thick_ax = flat(state.thick.axial, torch.float32, topology.n_thick * topology.n_crowns)
    xbs = flat(state.thick.xb_states, torch.int8, X)
    xbb = flat(state.thick.xb_bound_to, torch.int32, X)
    xbn = flat(state.thick.xb_nearest_bs, torch.int32, X)
    xbd = flat(state.thick.xb_distances, torch.float32, 2 * X)
    thin_ax = flat(state.thin.axial, torch.float32, S)
    tms = flat(state.thin.tm_states, torch.int8, S)
    tmb = flat(state.thin.bound_to, torch.int32, S)
    rows = _rows(constants, B)
    if tolerance is not None:
        rows[:, DYNAMIC_FIELDS.index('solver_tol')] = np.float32(tolerance)
    keys = _keys(rng_key if rng_key is not None else np.zeros(2, np.uint32), B)
    host = [rows, keys.view(np.int32)]
    drv = drivers if drivers is not None else Drivers()
    for v, name in ((drv.pCa, 'pCa'), (drv.z_line, 'z_line'), (drv.lattice_spacing, 'lattice_spacing')):
        host.append(_per_state(v.cpu().numpy() if hasattr(v, 'cpu') else v, B, name))
    dyn = K_lat is not None
    if dyn:
        if d_ref is None:
            raise ValueError("d_ref is required when K_lat is given")
        host += [_per_state(K_lat, B, 'K_lat'), _per_state(d_ref, B, 'd_ref')]
    from .engine import upload
    with torch.cuda.device(dev):
        d_arrays = upload(dev, *host)
        d_rows, d_keys, d_pca, d_z, d_ls = d_arrays[:5]
        d_K, d_dref = (d_arrays[5], d_arrays[6]) if dyn else (None, None)
        resid = torch.zeros(B, dtype=torch.float32, device=dev)
        ls_out = torch.zeros(B, dtype=torch.float32, device=dev)
        iters = torch.zeros(B, dtype=torch.int32, device=dev)
        status = torch.zeros(B, dtype=torch.int32, device=dev)
        sb = mf_state_batch()
        sb.B, sb.topo_id, sb.phases = B, up.topo_id, int(phases)
        sb.flags = 0 if partitionable else MF_FLAG_ORIGINAL_PRNG
        sb.dt, sb.n_newton, sb.n_cg = float(dt), int(n_newton_steps), int(n_cg_steps)
        sb.thick_axial, sb.xb_states, sb.xb_bound_to = thick_ax.data_ptr(), xbs.data_ptr(), xbb.data_ptr()
        sb.xb_nearest_bs, sb.xb_distances, sb.thin_axial = xbn.data_ptr(), xbd.data_ptr(), thin_ax.data_ptr()
        sb.tm_states, sb.thin_bound_to, sb.keys = tms.data_ptr(), tmb.data_ptr(), d_keys.data_ptr()
        sb.params, sb.pCa, sb.z_line, sb.lattice_spacing = d_rows.data_ptr(), d_pca.data_ptr(), d_z.data_ptr(), d_ls.data_ptr()
        sb.K_lat = d_K.data_ptr() if dyn else None
        sb.d_ref = d_dref.data_ptr() if dyn else None
        sb.residual_out, sb.ls_out, sb.iters_out, sb.status_out = (resid.data_ptr(), ls_out.data_ptr(),
                                                                   iters.data_ptr(), status.data_ptr())
        sp = _subpop_pops(xb_subpop, tm_subpop, topology, B)
        keep = []
        if sp is not None:
            pops = device_pops(sp, dev)
            keep.append(pops)
            sb.n_pops = sp.K
            sb.pop_flags = pops['flags']
            sb.pop_params, sb.pop_frac = pops['rows'].data_ptr(), pops['fractions'].data_ptr()
            if sp.explicit:
                sb.label_stride = int(pops['xb_label'].shape[1])
                sb.xb_label, sb.tm_label = pops['xb_label'].data_ptr(), pops['tm_label'].data_ptr()
        if uniforms is not None:
            ut = torch.as_tensor(np.ascontiguousarray(uniforms[0], np.float32).reshape(B, S), device=dev)
            ux = torch.as_tensor(np.ascontiguousarray(uniforms[1], np.float32).reshape(B, X), device=dev)
            keep += [ut, ux]
            sb.u_thin, sb.u_xb = ut.data_ptr(), ux.data_ptr()
        s = torch.cuda.current_stream(dev)
        rc = fn(eng.h, ctypes.byref(sb), ctypes.c_void_p(s.cuda_stream))
        if rc:
            msg = eng.lib.mf_last_error(eng.h)
            raise EngineError(f"mf_step_states failed ({rc}): {msg.decode() if msg else ''}")
    lead = () if B0 == 0 else (B0,)
    t = topology
    new = State(
        ThickState(thick_ax.view(lead + (t.n_thick, t.n_crowns)), xbs.view(lead + (t.n_thick, t.n_crowns, t.n_xb_per_crown)),
                   xbb.view(lead + (t.n_thick, t.n_crowns, t.n_xb_per_crown)),
                   xbn.view(lead + (t.n_thick, t.n_crowns, t.n_xb_per_crown)),
                   xbd.view(lead + (t.n_thick, t.n_crowns, t.n_xb_per_crown, 2))),
        ThinState(thin_ax.view(lead + (t.n_thin, t.n_sites)), tms.view(lead + (t.n_thin, t.n_sites)),
                  tmb.view(lead + (t.n_thin, t.n_sites))))
    new_keys = d_keys.view(torch.int32).cpu().numpy().view(np.uint32).reshape(B, 2)
    out_key = new_keys[0].copy() if B0 == 0 else new_keys.copy()
    sq = (lambda x: x[0]) if B0 == 0 else (lambda x: x)
    return new, out_key, sq(resid), sq(ls_out), sq(iters), sq(status)


def _resolved(constants: DynamicParams, drivers: Drivers) -> DynamicParams:
    """constants.with_drivers of the resolved drivers (NaN -> the constant), as
    kinetics_step returns them (timestep.py:96-103)."""
    def pick(d, c):
        d = np.asarray(d.cpu().numpy() if hasattr(d, 'cpu') else d, np.float32)
        c = np.asarray(c, np.float32)
        return np.where(np.isnan(d), c, d)
    return constants.with_drivers(pick(drivers.pCa, constants.pCa), pick(drivers.z_line, constants.z_line),
                                  pick(drivers.lattice_spacing, constants.lattice_spacing))


def update_nearest_neighbors(state: State, constants: DynamicParams, topology, **kw) -> State:
    """Nearest binding site and offsets of every head (kernels/geometry.py:186-262)."""
    new, *_ = _step(state, constants, topology, MF_PHASE_NEAREST, **kw)
    return new


def kinetics_step(state: State, constants: DynamicParams, drivers: Drivers, topology, rng_key, *, dt: float,
                  xb_subpop=None, tm_subpop=None, **kw):
    """Kinetics half of a timestep (timestep.py:65-129): nearest sites,
    tropomyosin then crossbridge transitions.  Returns ``(state, rng_key,
    resolved_constants)``; positions are left out of equilibrium."""
    new, key, *_ = _step(state, constants, topology, MF_PHASE_KINETICS, drivers, rng_key, dt=dt,
                         xb_subpop=xb_subpop, tm_subpop=tm_subpop, **kw)
    return new, key, _resolved(constants, drivers)


def solve_equilibrium(state: State, constants: DynamicParams, topology, K_lat=None, d_ref=None,
                      tolerance: Optional[float] = None, n_newton_steps: int = 16, n_cg_steps: int = 6,
                      precond_params=None, prefactored_precond=None, **kw):
    """Newton-CG force balance of the filament nodes (kernels/solver.py:663-771),
    with the lattice spacing as an extra unknown when ``K_lat`` (already x
    n_thick) is given.  ``constants`` carry z_line and the (initial) spacing.
    Returns ``(state, residual, new_lattice_spacing, n_iters)``."""
    new, _, resid, ls, iters, _ = _step(state, constants, topology, MF_PHASE_EQUILIBRIUM, K_lat=K_lat, d_ref=d_ref,
                                        tolerance=tolerance, n_newton_steps=n_newton_steps,
                                        n_cg_steps=n_cg_steps, **kw)
    return new, resid, ls, iters


def timestep(state: State, constants: DynamicParams, drivers: Drivers, topology, rng_key, *, dt: float,
             K_lat=None, d_ref=None, solver_tol: Optional[float] = None, n_cg_steps: int = 6,
             n_newton_steps: int = 16, precond_params=None, prefactored_precond=None, xb_subpop=None,
             tm_subpop=None, **kw):
    """One whole timestep (timestep.py:132-199): kinetics, then the equilibrium
    solve at the resolved drivers.  Returns ``(new_state, rng_key,
    solver_residual, new_ls, n_iters)``."""
    new, key, resid, ls, iters, _ = _step(state, constants, topology, MF_PHASE_TIMESTEP, drivers, rng_key, dt=dt,
                                          K_lat=K_lat, d_ref=d_ref, tolerance=solver_tol,
                                          n_newton_steps=n_newton_steps, n_cg_steps=n_cg_steps,
                                          xb_subpop=xb_subpop, tm_subpop=tm_subpop, **kw)
    return new, key, resid, ls, iters


def create_and_equilibrate(topology, constants: DynamicParams, z_line: float, pCa: float, lattice_spacing: float,
                           n_cg_steps: int = 6, n_newton_steps: int = 4, batch: Optional[int] = None,
                           device=None) -> State:
    """realize_state, nearest sites and one equilibrium solve with the constants
    (simulation.py:633-642; the constants' z_line and spacing, not the arguments,
    drive the nearest-site search and the solve)."""
    s = realize_state(topology, constants, z_line, pCa, lattice_spacing, batch=batch, device=device)
    s = update_nearest_neighbors(s, constants, topology)
    s, _, _, _ = solve_equilibrium(s, constants, topology, n_newton_steps=n_newton_steps, n_cg_steps=n_cg_steps)
    return s


__all__ = ['State', 'ThickState', 'ThinState', 'Drivers', 'realize_state', 'update_nearest_neighbors',
           'kinetics_step', 'solve_equilibrium', 'timestep', 'create_and_equilibrate', 'MF_PHASE_NEAREST',
           'MF_PHASE_TRANSITIONS', 'MF_PHASE_EQUILIBRIUM', 'MF_PHASE_KINETICS', 'MF_PHASE_TIMESTEP']
