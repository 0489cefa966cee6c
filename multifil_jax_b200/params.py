"""Physical parameters of the half-sarcomere model.

Two kinds, mirroring the reference package (``multifil_jax/core/params.py``):

* :class:`StaticParams` -- structure.  Every field fixes an array shape or a
  solver cap; changing one means a new :class:`~multifil_jax_b200.topology.SarcTopology`.
  Reference: ``core/params.py:563-733``.
* :class:`DynamicParams` -- the 44 sweepable physics values, each stored as a
  float32 scalar (or a float32 vector when a field is swept).  Reference:
  ``core/params.py:73-556`` (defaults, in this exact order) and ``:739-857``.

On the device a condition's parameters travel as one float32 row of 44 values
in :data:`DYNAMIC_FIELDS` order; ``param_row()`` builds it.
"""
from __future__ import annotations

import dataclasses
import warnings
from dataclasses import dataclass, asdict
from typing import Any, Dict, Tuple

import numpy as np

# Field name -> skeletal default.  Order is the device parameter-row layout and
# the reference's DYNAMIC_FIELDS order (core/params.py:73-556).
_DEFAULTS: Dict[str, float] = {
    # backbone springs (pN/nm per segment)
    'thick_k': 7500.0,
    'thin_k': 5500.0,
    # two-spring crossbridge head: converter (angular) and globular (linear)
    'xb_c_rest_weak': 0.82309,
    'xb_c_rest_strong': 1.27758,
    'xb_c_k_weak': 8.0,
    'xb_c_k_strong': 40.0,
    'xb_g_rest_weak': 19.93,
    'xb_g_rest_strong': 16.47,
    'xb_g_k_weak': 0.4,
    'xb_g_k_strong': 5.0,
    # titin exponential spring
    'titin_a': 43.0,
    'titin_b': 0.004,
    'titin_rest': 215.0,
    # tropomyosin rates / equilibria / Ising couplings
    'tm_k_01': 100000.0,
    'tm_k_12': 1.0,
    'tm_k_23': 0.1,
    'tm_k_30': 0.2,
    'tm_Keq_01': 500000.0,
    'tm_Keq_12': 130.0,
    'tm_Keq_23': 0.1,
    'tm_J_C': 0.0,
    'tm_J_M': 2.70,
    # crossbridge cycle
    'xb_r01_coeff': 305.99,
    'xb_r12_coeff': 0.6,
    'xb_r23_coeff': 0.15,
    'xb_r34_coeff': 0.6,
    'xb_delta_23': 1.0,
    'xb_delta_34': 0.5,
    'xb_r40': 0.1,
    'xb_r04': 0.01,
    'xb_r05': 0.007,
    'xb_U_DRX': -2.3,
    'xb_U_loose': -4.3,
    'xb_U_tight_1': -15.0,
    'xb_U_tight_2': -21.0,
    # super-relaxed state recruitment (Hill form)
    'xb_srx_k0': 0.007,
    'xb_srx_kmax': 0.4,
    'xb_srx_b': 5.0,
    'xb_srx_ca50': 1e-6,
    # environment / solver
    'temp_celsius': 26.15,
    'solver_tol': 0.3,
    # default driver values
    'pCa': 4.5,
    'z_line': 900.0,
    'lattice_spacing': 14.0,
}

DYNAMIC_FIELDS: Tuple[str, ...] = tuple(_DEFAULTS)
N_PARAMS = len(DYNAMIC_FIELDS)  # 44
PARAM_INDEX = {name: i for i, name in enumerate(DYNAMIC_FIELDS)}

STATIC_FIELDS = frozenset({
    'n_crowns', 'n_polymers_per_thin', 'solver_max_iter', 'actin_geometry',
    'n_newton_steps', 'n_cg_steps', 'solver_residual_tol', 'n_xb_bins',
    'xb_bin_lo', 'xb_bin_hi', 'thick_bare_zone', 'thick_crown_spacing',
    'actin_half_pitch', 'mono_per_poly', 'polymer_base_turns',
    'target_zone_wiggle', 'n_xb_per_crown'})


@dataclass(frozen=True)
class StaticParams:
    """Structural configuration (reference ``core/params.py:563-733``).

    ``actin_geometry`` is ``'vertebrate'`` (1 thick : 2 thin, three faces per
    thin filament) or ``'invertebrate'`` (1 thick : 3 thin, two faces);
    ``n_superlattice_classes`` 3 staggers the thick filaments of the insect
    myosin superlattice; ``legacy_crown_geometry`` uses the fixed crown-face
    table.
    """
    n_crowns: int = 52
    n_polymers_per_thin: int = 15
    solver_max_iter: int = 50
    actin_geometry: str = "vertebrate"
    n_newton_steps: int = 4
    n_cg_steps: int = 6
    solver_residual_tol: float = 1.5
    n_xb_bins: int = 200
    xb_bin_lo: float = -8.0
    xb_bin_hi: float = 35.0
    thick_bare_zone: float = 58.0
    thick_crown_spacing: float = 14.3
    n_superlattice_classes: int = 1
    actin_half_pitch: float = 36.0
    mono_per_poly: int = 26
    polymer_base_turns: float = 12.0
    # float32 round trip of rev/24, as the reference stores it
    target_zone_wiggle: float = float(np.float32(2 * np.pi) / np.float32(24))
    n_xb_per_crown: int = 3
    crown_rotation_deg: float = 60.0
    crown_face_wiggle_deg: float = 15.0
    legacy_crown_geometry: bool = False

    def __post_init__(self):
        # Same validation as core/params.py:702-722.
        if self.legacy_crown_geometry and self.n_xb_per_crown != 3:
            raise ValueError(
                "legacy_crown_geometry=True requires n_xb_per_crown == 3 "
                f"(the legacy face_pattern table has no n={self.n_xb_per_crown} analogue)")
        if self.legacy_crown_geometry and (
                self.crown_rotation_deg != 60.0 or self.crown_face_wiggle_deg != 15.0):
            warnings.warn(
                "legacy_crown_geometry=True ignores crown_rotation_deg/crown_face_wiggle_deg",
                stacklevel=2)
        if self.n_superlattice_classes not in (1, 3):
            raise ValueError(
                f"n_superlattice_classes must be 1 or 3, got {self.n_superlattice_classes}")

    def replace(self, **kwargs) -> 'StaticParams':
        return StaticParams(**{**asdict(self), **kwargs})

    def __repr__(self) -> str:
        return (f"StaticParams(n_crowns={self.n_crowns}, "
                f"n_polymers_per_thin={self.n_polymers_per_thin}, "
                f"actin_geometry='{self.actin_geometry}')")


def _as_f32(value: Any) -> np.ndarray:
    return np.asarray(value, dtype=np.float32)


class DynamicParams:
    """The 44 sweepable physics values (reference ``core/params.py:739-857``).

    Every field is a float32 numpy array: a 0-d scalar normally, or a 1-d
    vector when the field is swept (``run()`` turns a vector of length > 1 into
    a sweep axis, as the reference does at ``simulation.py:943-949``).
    """
    __slots__ = DYNAMIC_FIELDS

    def __init__(self, **kwargs):
        unknown = set(kwargs) - set(DYNAMIC_FIELDS)
        if unknown:
            raise ValueError(f"Unknown parameter: {sorted(unknown)}. Valid: {list(DYNAMIC_FIELDS)}")
        for name, default in _DEFAULTS.items():
            object.__setattr__(self, name, _as_f32(kwargs.get(name, default)))

    def __setattr__(self, name, value):
        raise AttributeError("DynamicParams is immutable; use .copy(**updates)")

    def to_dict(self) -> Dict[str, Any]:
        out = {}
        for name in DYNAMIC_FIELDS:
            v = getattr(self, name)
            out[name] = float(v) if np.ndim(v) == 0 else np.asarray(v).tolist()
        return out

    def copy(self, **updates) -> 'DynamicParams':
        invalid = set(updates) - set(DYNAMIC_FIELDS)
        if invalid:
            raise ValueError(f"Unknown parameter: {sorted(invalid)}. Valid: {list(DYNAMIC_FIELDS)}")
        kw = {name: updates.get(name, getattr(self, name)) for name in DYNAMIC_FIELDS}
        return DynamicParams(**kw)

    def with_drivers(self, pCa, z_line, lattice_spacing) -> 'DynamicParams':
        return self.copy(pCa=pCa, z_line=z_line, lattice_spacing=lattice_spacing)

    def param_row(self) -> np.ndarray:
        """float32[44] device row; every field must be a scalar."""
        row = np.empty(N_PARAMS, dtype=np.float32)
        for i, name in enumerate(DYNAMIC_FIELDS):
            v = getattr(self, name)
            if np.ndim(v) != 0:
                raise ValueError(f"field {name} is a vector; expand the sweep first")
            row[i] = v
        return row

    def __eq__(self, other):
        if not isinstance(other, DynamicParams):
            return NotImplemented
        return all(np.array_equal(getattr(self, n), getattr(other, n)) for n in DYNAMIC_FIELDS)

    __hash__ = None

    def __repr__(self) -> str:
        return (f"DynamicParams(thick_k={float(np.ravel(self.thick_k)[0]):.1f}, "
                f"thin_k={float(np.ravel(self.thin_k)[0]):.1f}, ...)")


def get_skeletal_params() -> Tuple[StaticParams, DynamicParams]:
    """Fast-twitch skeletal preset: the defaults (reference ``core/params.py:860-897``)."""
    return StaticParams(), DynamicParams()


_CARDIAC_OVERRIDES = {
    # reference core/params.py:959-978
    'tm_k_12': 0.5,
    'tm_k_01': 80000.0,
    'tm_Keq_01': 750000.0,
    'tm_k_30': 0.04,
    'xb_r12_coeff': 0.175,
    'xb_r23_coeff': 0.065,
    'xb_r34_coeff': 0.065,
    'xb_r05': 0.2,
    'xb_srx_k0': 0.005,
    'titin_a': 55.0,
    'titin_b': 0.008,
    'titin_rest': 140.0,
}


def get_cardiac_params() -> Tuple[StaticParams, DynamicParams]:
    """Generic cardiac preset (reference ``core/params.py:900-979``)."""
    return StaticParams(), DynamicParams(**_CARDIAC_OVERRIDES)


# Insect indirect flight muscle geometry shared by the two insect presets
# (reference core/params.py:1185-1196 and :1264-1275); the Drosophila preset
# adds the 3-class myosin superlattice.
_IFM_STATIC = {
    'actin_geometry': 'invertebrate',
    'thick_crown_spacing': 14.5,
    'actin_half_pitch': 38.7,
    'mono_per_poly': 28,
    'polymer_base_turns': 13,
    'n_xb_per_crown': 4,
    'crown_rotation_deg': 33.75,
    'target_zone_wiggle': float(np.radians(26.0)),
    'n_crowns': 100,
    'n_polymers_per_thin': 20,
}
_IFM_DYNAMIC = {'titin_a': 40.0, 'titin_b': 0.025, 'titin_rest': 50.0}


def get_lethocerus_params() -> Tuple[StaticParams, DynamicParams]:
    """Lethocerus indirect flight muscle (reference ``core/params.py:982-1202``):
    invertebrate lattice, four heads per crown, 100 crowns, no superlattice."""
    return StaticParams(**_IFM_STATIC), DynamicParams(**_IFM_DYNAMIC)


def get_drosophila_params() -> Tuple[StaticParams, DynamicParams]:
    """Drosophila indirect flight muscle (reference ``core/params.py:1205-1281``):
    the Lethocerus geometry with the 3-class myosin superlattice (lattices need
    an even ``nrows`` and ``ncols`` a multiple of 3)."""
    return StaticParams(**_IFM_STATIC, n_superlattice_classes=3), DynamicParams(**_IFM_DYNAMIC)


def params_table(rows) -> np.ndarray:
    """Stack DynamicParams (all-scalar) into a float32 [B, 44] table."""
    return np.stack([dp.param_row() for dp in rows]).astype(np.float32)


__all__ = ['StaticParams', 'DynamicParams', 'DYNAMIC_FIELDS', 'STATIC_FIELDS', 'N_PARAMS',
           'PARAM_INDEX', 'get_skeletal_params', 'get_cardiac_params', 'get_lethocerus_params',
           'get_drosophila_params', 'params_table']
