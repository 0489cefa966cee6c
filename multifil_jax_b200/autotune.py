"""Per-lattice CTA-size autotuner for the fused step kernel.

Each condition runs in one CTA whose thread count trades per-condition latency
(more threads: fewer nodes per thread, more lanes in the Thomas scans) against
how many conditions share an SM (fewer threads: more resident CTAs, cheaper
barriers).  The best point depends on the lattice (nodes, heads) and on how
many conditions are in flight, so it is measured: a short run of the actual
kernel on a synthetic batch of that lattice for every candidate size, the
fastest kept for the lattice and precision mode through ``mf_tune_threads_mode``.
"""
from __future__ import annotations

import time
from typing import Dict, Iterable, Optional, Tuple

import numpy as np

from .engine import MF_FLAG_PRECISE, get_engine

CANDIDATES = (128, 256, 384, 512, 1024)
_CACHE: Dict[Tuple, int] = {}


def autotune(topology, n_conditions: int = 256, steps: int = 20, precision: str = 'float32',
             candidates: Iterable[int] = CANDIDATES, device: Optional[int] = None, verbose: bool = False,
             dynamic_ls: bool = False) -> int:
    """Measure every candidate CTA size on this lattice; keep and return the best.

    ``dynamic_ls`` measures with the lattice spacing solved as an unknown
    (K_lat 5, nu 0.5), where the per-step table rebuilds dominate.
    """
    import torch
    from .params import get_skeletal_params
    key = (topology.size_key(), int(n_conditions), precision, bool(dynamic_ls))
    eng = get_engine(device)
    if key in _CACHE:
        eng.tune_threads(topology, _CACHE[key], precision)
        return _CACHE[key]
    dev = torch.device('cuda', eng.device)
    B, T = int(n_conditions), int(steps)
    _, d = get_skeletal_params()
    from .engine import prng_key, prng_split
    P = torch.as_tensor(np.tile(d.param_row(), (B, 1)), device=dev)
    Z = torch.full((B, T), 900.0, device=dev)
    PC = torch.as_tensor(np.repeat(np.linspace(4.0, 7.0, B, dtype=np.float32)[:, None], T, 1), device=dev)
    L = torch.full((B, T), 14.0, device=dev)
    NS = torch.full((B,), T, dtype=torch.int32, device=dev)
    K = torch.as_tensor(prng_split(prng_key(0), B).astype(np.int64), device=dev).to(torch.int32)
    flags = MF_FLAG_PRECISE if precision == 'mixed' else 0
    kw = {}
    if dynamic_ls:
        from .engine import MF_FLAG_DYNAMIC_LS
        flags |= MF_FLAG_DYNAMIC_LS
        kw = dict(K_lat=torch.full((B,), 5.0 * topology.n_thick, device=dev),
                  nu=torch.full((B,), 0.5, device=dev))
    best, best_t = None, float('inf')
    for nt in candidates:
        try:
            eng.tune_threads(topology, nt, precision)
        except Exception:
            continue  # does not fit in shared memory at this size
        eng.run_batch(topology, P, Z, PC, L, NS, K, flags=flags, **kw)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        eng.run_batch(topology, P, Z, PC, L, NS, K, flags=flags, **kw)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        if verbose:
            print(f"autotune {topology.nrows}x{topology.ncols} B={B}: {nt} threads {dt * 1e3:.2f} ms")
        if dt < best_t:
            best, best_t = nt, dt
    if best is None:
        raise RuntimeError("no CTA size fits this lattice")
    eng.tune_threads(topology, best, precision)
    _CACHE[key] = best
    return best


def autotune_many(topologies, n_conditions: int = 256, **kw) -> Dict[Tuple[int, int], int]:
    """Tune every distinct lattice of an uneven batch."""
    out = {}
    seen = set()
    for t in topologies:
        k = t.size_key()
        if k in seen:
            continue
        seen.add(k)
        out[(t.nrows, t.ncols)] = autotune(t, n_conditions=n_conditions, **kw)
    return out


def choose_batch_sizes(topologies, picks: Dict[Tuple[int, int], int], run_short, precision: str = 'float32',
                       device: Optional[int] = None, repeats: int = 2) -> Dict[Tuple[int, int], int]:
    """Check the per-lattice sizes on the batch itself.

    Per-lattice sizes are measured on a batch of one lattice.  In an uneven
    batch every distinct CTA size becomes its own launch, and several partly
    filled launches can lose to one fuller launch at a common size.
    ``run_short()`` runs the actual batch for a few steps and returns its time
    in seconds.  The per-lattice sizes and the largest of them used for every
    lattice are both timed, and the faster one is kept.  Returns the kept
    sizes.
    """
    eng = get_engine(device)
    distinct = {}
    for t in topologies:
        distinct.setdefault((t.nrows, t.ncols), t)
    sizes = {picks[k] for k in distinct if k in picks}
    if len(sizes) <= 1:
        return dict(picks)

    def timed():
        run_short()  # warm-up (graph and allocation of this grouping)
        return min(run_short() for _ in range(repeats))

    t_per = timed()
    common = max(sizes)
    uniform = {}
    for k, t in distinct.items():
        try:
            eng.tune_threads(t, common, precision)
            uniform[k] = common
        except Exception:
            eng.tune_threads(t, picks[k], precision)  # the common size does not fit this lattice
            uniform[k] = picks[k]
    t_uni = timed()
    if t_uni <= t_per:
        return uniform
    for k, t in distinct.items():
        eng.tune_threads(t, picks[k], precision)
    return dict(picks)
