"""Mixed motor populations: one lattice, several kinetic parameter sets.

Behaviour of the reference's ``core/subpopulation.py`` (``Subpopulation``
with its ``mean_field``, ``random`` and ``c_zone`` constructors,
``generate_random_masks_batch``) and of the run()-side resolution in
``simulation.py:485-577``:

* Population 0 is the wild type; every other population multiplies named
  ``xb_*`` / ``tm_*`` DynamicParams fields by a factor.  Mechanics always keep
  the wild-type values.
* ``mean_field``: every unit sees the fraction-weighted sum of the K
  populations' generators, ``Q = sum_k f_k Q_k``, exponentiated once
  (``transitions.py:580-585,967-971``).
* ``random`` / ``c_zone`` (the "explicit" modes): every head and binding site
  carries a population label; each population's generators are exponentiated
  and a unit reads its own population's table (``transitions.py:586-596,
  973-976``).  ``random`` draws labels per simulation from
  ``split(PRNGKey(seed), n_sims)``; ``c_zone`` labels the crowns (and, when a
  ``tm_*`` field is scaled, the sites) inside an axial band.

On the device a resolved subpopulation is a set of per-condition arrays
(:class:`ResolvedSubpop`): K parameter rows, K fractions, and int8 labels per
head and per site.  The CUDA kernel builds the K table sets (or the blended
one) with the same table builder as the single-population path.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from .params import DYNAMIC_FIELDS, DynamicParams

# Default cardiac C-zone band (nm from the M-line): crowns whose axial offset
# lies in it belong to the modified population (reference core/subpopulation.py:74-75).
C_ZONE_MIN_NM = 350.0
C_ZONE_MAX_NM = 650.0

# populations per condition the kernel accepts (include/multifil_b200.h MF_MAX_POPS)
MAX_POPS = 4

_FIELD_INDEX = {n: i for i, n in enumerate(DYNAMIC_FIELDS)}


def _checked_scales(scales: Dict[str, float]) -> Dict[str, float]:
    unknown = sorted(set(scales) - set(DYNAMIC_FIELDS))
    if unknown:
        raise ValueError(f"Unknown subpopulation scale field(s): {unknown}. "
                         f"Valid DynamicParams fields: {list(DYNAMIC_FIELDS)}")
    return {k: float(v) for k, v in scales.items()}


@dataclass
class Subpopulation:
    """K populations of motors (index 0 = wild type).

    ``scales[k]`` maps DynamicParams field names to multiplicative factors;
    ``fractions`` are the K blend weights (float32, summing to one) and the
    label probabilities of ``random``.  ``mode`` is ``'mean_field'``,
    ``'random'`` or ``'c_zone'``.  ``xb_mask`` / ``tm_mask`` hold fixed int
    labels per head / site (``c_zone``); ``seed`` drives ``random``.
    """
    scales: List[Dict[str, float]]
    fractions: np.ndarray
    mode: str
    xb_mask: Optional[np.ndarray] = None
    tm_mask: Optional[np.ndarray] = None
    seed: Optional[int] = None

    @property
    def K(self) -> int:
        return len(self.scales)

    def scaled_fields(self) -> tuple:
        """Every field some population scales, sorted by name."""
        return tuple(sorted({f for s in self.scales for f in s}))

    def scale_array(self, field_names: Sequence[str]) -> np.ndarray:
        """(K, F) float32 factors in ``field_names`` order (1 where a population leaves a field)."""
        return np.array([[float(s.get(f, 1.0)) for f in field_names] for s in self.scales], dtype=np.float32)

    def apply_scales(self, constants: DynamicParams) -> List[DynamicParams]:
        """The K populations' DynamicParams: each scale dict multiplied onto ``constants``
        (population 0, with no scales, is ``constants`` itself)."""
        out = []
        for s in self.scales:
            if not s:
                out.append(constants)
            else:
                out.append(constants.copy(**{f: np.asarray(getattr(constants, f), np.float32) * np.float32(v)
                                             for f, v in s.items()}))
        return out

    @classmethod
    def mean_field(cls, fraction: float, **scales) -> 'Subpopulation':
        """Every unit follows the fraction-weighted blend of the wild-type and
        modified generators; no labels, still one exponential per table."""
        return cls(scales=[{}, _checked_scales(scales)],
                   fractions=np.asarray([1.0 - fraction, fraction], dtype=np.float32), mode='mean_field')

    @classmethod
    def random(cls, fraction: float, seed: int = 0, **scales) -> 'Subpopulation':
        """Each head and site is independently modified with probability
        ``fraction``; labels are drawn per simulation from ``seed``."""
        return cls(scales=[{}, _checked_scales(scales)],
                   fractions=np.asarray([1.0 - fraction, fraction], dtype=np.float32), mode='random',
                   seed=seed)

    @classmethod
    def c_zone(cls, topology, c_zone_min_nm: float = C_ZONE_MIN_NM, c_zone_max_nm: float = C_ZONE_MAX_NM,
               **scales) -> 'Subpopulation':
        """Heads on crowns whose axial offset lies in [min, max] nm are modified
        (and, when a ``tm_*`` field is scaled, the sites in the same band)."""
        sc = _checked_scales(scales)
        xb_mask, tm_mask = c_zone_masks(topology, c_zone_min_nm, c_zone_max_nm, sc)
        frac = float(np.mean(xb_mask))
        return cls(scales=[{}, sc], fractions=np.asarray([1.0 - frac, frac], dtype=np.float32), mode='c_zone',
                   xb_mask=xb_mask, tm_mask=tm_mask)


def c_zone_masks(topology, lo_nm: float, hi_nm: float, scales: Dict[str, float]):
    """Int32 labels per head and per site of an axial band (reference
    ``core/subpopulation.py:179-210``): heads inherit their crown's membership;
    sites are labelled by their rest position only when a ``tm_*`` field is scaled."""
    off = np.asarray(topology.crown_offsets)
    inside = ((off >= lo_nm) & (off <= hi_nm)).astype(np.int32)
    xb = np.repeat(inside[:, :, None], topology.n_xb_per_crown, axis=2).reshape(-1)
    if any(f.startswith('tm_') for f in scales):
        pos = np.cumsum(np.asarray(topology.binding_rests), axis=1)
        tm = ((pos >= lo_nm) & (pos <= hi_nm)).astype(np.int32).reshape(-1)
    else:
        tm = np.zeros(topology.n_thin * topology.n_sites, dtype=np.int32)
    return xb, tm


def generate_random_masks_batch(seed: int, p_mut_b, topology, total_batch: int):
    """Per-simulation Bernoulli labels (reference ``core/subpopulation.py:213-253``).

    Simulation i uses key ``split(PRNGKey(seed), total_batch)[i]``, split once
    more into a head key and a site key; a unit is modified where its
    ``uniform`` draw is below ``p_mut_b[i]``.  Returns int32 arrays
    ``[total_batch, total_xbs]`` and ``[total_batch, n_sites_total]``.
    """
    from .engine import prng_key, prng_split, prng_uniform
    X, S = topology.total_xbs, topology.n_sites_total
    p = np.asarray(p_mut_b, dtype=np.float32).reshape(-1)
    keys = prng_split(prng_key(int(seed)), total_batch) if total_batch else np.zeros((0, 2), np.uint32)
    xb = np.zeros((total_batch, X), np.int32)
    tm = np.zeros((total_batch, S), np.int32)
    for i in range(total_batch):
        kx, kt = prng_split(keys[i], 2)
        xb[i] = prng_uniform(kx, X) < p[i]
        tm[i] = prng_uniform(kt, S) < p[i]
    return xb, tm


@dataclass
class ResolvedSubpop:
    """Per-condition device inputs of a subpopulation run (B conditions, K populations).

    ``explicit`` selects labelled tables (``random`` / ``c_zone``) over the
    blend; ``xb`` / ``tm`` say which rate family the populations change (a
    family no population scales keeps the wild-type tables, as the reference's
    ``subpop_has_xb`` / ``subpop_has_tm`` flags do).
    """
    K: int
    explicit: bool
    xb: bool
    tm: bool
    rows: np.ndarray       # [B, K, 44] float32 parameter rows
    fractions: np.ndarray  # [B, K] float32
    xb_label: Optional[np.ndarray] = None  # [B, total_xbs] int8
    tm_label: Optional[np.ndarray] = None  # [B, n_sites_total] int8

    def take(self, s: int, e: int) -> 'ResolvedSubpop':
        """Rows s:e of every per-condition array."""
        cut = lambda a: None if a is None else a[s:e]
        return ResolvedSubpop(self.K, self.explicit, self.xb, self.tm, self.rows[s:e], self.fractions[s:e],
                              cut(self.xb_label), cut(self.tm_label))


def resolve_subpopulation(subpopulation, topology, params: np.ndarray, variant_index: Optional[np.ndarray]):
    """Subpopulation (or list of them, a sweep axis) -> :class:`ResolvedSubpop` or None.

    ``params`` is the run's [B, 44] parameter rows; ``variant_index`` gives
    each condition's element of a swept list (None: one object for all).
    Errors follow the reference (``simulation.py:514-577``).
    """
    if subpopulation is None:
        return None
    subs = list(subpopulation) if isinstance(subpopulation, list) else [subpopulation]
    for s in subs:
        if not isinstance(s, Subpopulation):
            raise TypeError(f"subpopulation must be a Subpopulation or a list of them, got {type(s).__name__}")
    modes = {s.mode for s in subs}
    if len(modes) > 1:
        raise ValueError(f"All swept subpopulations must share one mode; got {sorted(modes)}")
    Ks = {s.K for s in subs}
    if len(Ks) > 1:
        raise ValueError(f"All swept subpopulations must have the same K; got {sorted(Ks)}")
    mode, K = subs[0].mode, subs[0].K
    if mode not in ('mean_field', 'random', 'c_zone'):
        raise ValueError(f"Unknown subpopulation mode '{mode}'")
    if K > MAX_POPS:
        raise ValueError(f"at most {MAX_POPS} populations are supported, got {K}")
    fields = sorted({f for s in subs for f in s.scaled_fields()})
    bad = [f for f in fields if not (f.startswith('xb_') or f.startswith('tm_'))]
    if bad:
        raise ValueError(f"Subpopulation scales must be xb_* or tm_* fields; got {sorted(bad)}")
    B = params.shape[0]
    scale_v = np.stack([s.scale_array(fields) for s in subs])            # [V, K, F]
    frac_v = np.stack([np.asarray(s.fractions, np.float32) for s in subs])  # [V, K]
    idx = np.zeros(B, np.int64) if variant_index is None else np.asarray(variant_index, np.int64)
    scale_b, frac_b = scale_v[idx], frac_v[idx]                           # [B, K, F], [B, K]
    rows = np.repeat(params[:, None, :].astype(np.float32), K, axis=1)
    for j, f in enumerate(fields):
        c = _FIELD_INDEX[f]
        rows[:, :, c] = (params[:, None, c].astype(np.float32) * scale_b[:, :, j]).astype(np.float32)
    has_xb = any(f.startswith('xb_') for f in fields)
    has_tm = any(f.startswith('tm_') for f in fields)
    res = ResolvedSubpop(K=K, explicit=mode != 'mean_field', xb=has_xb, tm=has_tm, rows=rows,
                         fractions=frac_b.astype(np.float32))
    if res.explicit:
        if mode == 'c_zone':
            xv = np.stack([np.asarray(s.xb_mask) for s in subs])
            tv = np.stack([np.asarray(s.tm_mask) for s in subs])
            xl, tl = xv[idx], tv[idx]
        else:
            seeds = {int(s.seed or 0) for s in subs}
            if len(seeds) > 1:
                raise ValueError(f"All swept 'random' subpopulations must share one seed; got {sorted(seeds)}")
            xl, tl = generate_random_masks_batch(subs[0].seed or 0, frac_b[:, 1], topology, B)
        if xl.shape[1] != topology.total_xbs or tl.shape[1] != topology.n_sites_total:
            raise ValueError("subpopulation masks do not match the topology's head / site counts")
        if np.any((xl < 0) | (xl >= K)) or np.any((tl < 0) | (tl >= K)):
            raise ValueError(f"subpopulation labels must lie in [0, {K})")
        res.xb_label = np.ascontiguousarray(xl, dtype=np.int8)
        res.tm_label = np.ascontiguousarray(tl, dtype=np.int8)
    return res


__all__ = ['Subpopulation', 'c_zone_masks', 'generate_random_masks_batch', 'resolve_subpopulation',
           'ResolvedSubpop', 'C_ZONE_MIN_NM', 'C_ZONE_MAX_NM', 'MAX_POPS']
