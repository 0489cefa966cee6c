"""The data cube that :func:`multifil_jax_b200.run` returns.

Every metric and every driver trace is an array shaped
``(sweep axes..., replicates, time)``.  The sweep axes appear only for
arguments given as lists, in the order run() expands them; the replicate and
time axes are always there.  ``_axis_names`` names every axis and ``coords``
holds the coordinate values of the named sweep axes.

The behaviour a drop-in user relies on is the reference's
(``multifil_jax/simulation.py:96-420``):

* ``mean()`` / ``std()`` collapse the replicate axis (the second-last axis)
  of every metric; the drivers are averaged in both cases, since they do not
  vary between replicates.
* Indexing applies the same key to every array.  An integer removes its axis
  from the names and coordinates, a slice cuts that axis' coordinate list,
  and any other key (an index array, a mask, ``Ellipsis``) leaves the axis
  bookkeeping as it was.
* ``sel(name=value)`` picks coordinate values and drops those axes;
  ``stack`` puts results of one shape side by side on a new leading axis.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

DRIVER_FIELDS = ('z_line', 'pCa', 'lattice_spacing')


class MetricsDict(dict):
    """A dict of metric arrays whose keys also read as attributes
    (``m.axial_force is m['axial_force']``), like the reference's
    ``core/state.py:118-130``."""

    def __getattr__(self, key):
        if key in self:
            return self[key]
        raise AttributeError(key)


def axes_after_index(names: Sequence[str], coords: Dict[str, list], key) -> Tuple[List[str], Dict[str, list]]:
    """Axis names and coordinates of a cube after ``cube[key]``.

    The key's parts are matched to the leading axes.  Integer parts remove
    their axis; slice parts keep it with the coordinates cut the same way;
    axes past the end of the key are untouched.  A part of any other kind
    (or a coordinate list that cannot be sliced) makes the result keep the
    original bookkeeping unchanged.
    """
    parts = key if isinstance(key, tuple) else (key,)
    kept: List[str] = []
    out = dict(coords)
    for axis, part in zip(names, parts):
        if isinstance(part, (int, np.integer)):
            out.pop(axis, None)
        elif isinstance(part, slice):
            kept.append(axis)
            if axis in out:
                try:
                    out[axis] = list(out[axis])[part]
                except Exception:
                    return list(names), dict(coords)
        else:
            return list(names), dict(coords)
    kept.extend(names[len(parts):])
    return kept, out


def _coord_position(values: list, wanted) -> Optional[int]:
    """Position of ``wanted`` in a coordinate list (array-valued coordinates,
    e.g. the traces of a trace sweep, compare element-wise)."""
    for i, v in enumerate(values):
        if isinstance(v, np.ndarray) or isinstance(wanted, np.ndarray):
            if np.shape(v) == np.shape(wanted) and np.array_equal(v, wanted):
                return i
        elif v == wanted:
            return i
    return None


class SimulationResult:
    """Result of :func:`multifil_jax_b200.run`: the 52 metrics and the driver
    traces as numpy arrays over ``(sweep axes..., replicates, time)``.

    Constructor arguments and attributes are the reference's: ``metrics``,
    ``rng_key`` (the key after the batch, for continuation), ``z_line``,
    ``pCa``, ``lattice_spacing``, ``final_state`` (always None),
    ``metadata``, ``dt`` (ms), ``name``, ``grid_shape``, ``axis_names``,
    ``coords`` and ``topology_config``.
    """

    __slots__ = ('metrics', 'rng_key', 'z_line', 'pCa', 'lattice_spacing', 'final_state', 'metadata',
                 'dt', 'name', '_grid_shape', '_axis_names', 'coords', 'topology_config')

    def __init__(self, metrics, rng_key, z_line, pCa, lattice_spacing, final_state=None, metadata=None,
                 dt=1.0, name="", grid_shape=None, axis_names=None, coords=None, topology_config=None):
        self.metrics = metrics if isinstance(metrics, MetricsDict) else MetricsDict(metrics)
        self.rng_key = rng_key
        self.z_line, self.pCa, self.lattice_spacing = z_line, pCa, lattice_spacing
        self.final_state = final_state
        self.metadata = {} if metadata is None else metadata
        self.dt = float(dt)
        self.name = str(name)
        self._grid_shape = grid_shape
        self._axis_names = [] if axis_names is None else axis_names
        self.coords = {} if coords is None else coords
        self.topology_config = {} if topology_config is None else topology_config

    # ---- derived views -------------------------------------------------
    def _derive(self, on_metric, on_driver, axis_names, coords, name=None) -> 'SimulationResult':
        """A new result whose metrics and drivers are transformed arrays of
        this one's; the grid shape follows the new force array."""
        metrics = MetricsDict((k, on_metric(v)) for k, v in self.metrics.items())
        force = metrics['axial_force']
        drivers = {f: on_driver(getattr(self, f)) for f in DRIVER_FIELDS}
        return SimulationResult(metrics=metrics, rng_key=self.rng_key, final_state=None, metadata=self.metadata,
                                dt=self.dt, name=self.name if name is None else name,
                                grid_shape=force.shape[:-1] if force.ndim > 1 else None,
                                axis_names=axis_names, coords=coords, topology_config=self.topology_config,
                                **drivers)

    @property
    def n_steps(self) -> int:
        return self.metrics['axial_force'].shape[-1]

    @property
    def replicate_axis(self) -> Optional[int]:
        names = self._axis_names
        return names.index('replicates') if 'replicates' in names else None

    @property
    def time(self) -> np.ndarray:
        """Step times in ms."""
        return self.dt * np.arange(self.n_steps)

    @property
    def axial_force(self) -> np.ndarray:
        """M-line force in pN (``metrics['axial_force']``)."""
        return self.metrics['axial_force']

    @property
    def mean_force(self) -> float:
        return float(self.axial_force.mean())

    @property
    def steady_state_force(self) -> float:
        """Mean force over the last fifth of the run (at least one step)."""
        tail = max(self.n_steps // 5, 1)
        return float(self.axial_force[..., self.n_steps - tail:].mean())

    def _over_replicates(self, reduce, suffix: str) -> 'SimulationResult':
        if self.replicate_axis is None:
            raise ValueError("No replicate axis to reduce.")
        names = [a for a in self._axis_names if a != 'replicates']
        coords = {a: c for a, c in self.coords.items() if a != 'replicates'}
        return self._derive(lambda v: reduce(v, axis=-2), lambda v: np.mean(v, axis=-2), names, coords,
                            name=self.name + suffix)

    def mean(self) -> 'SimulationResult':
        """Mean over replicates."""
        return self._over_replicates(np.mean, "_mean")

    def std(self) -> 'SimulationResult':
        """Population standard deviation over replicates (drivers: their mean)."""
        return self._over_replicates(np.std, "_std")

    def __getitem__(self, key) -> 'SimulationResult':
        names, coords = axes_after_index(self._axis_names, self.coords, key)
        return self._derive(lambda v: v[key], lambda v: v[key], names, coords)

    def sel(self, **picks) -> 'SimulationResult':
        """Select by coordinate value, e.g. ``result.sel(pCa=5.0)``; the
        selected axes are dropped."""
        index: List = [slice(None)] * self.axial_force.ndim
        for axis, value in picks.items():
            if axis not in self.coords:
                raise ValueError(f"Unknown axis '{axis}'. Available: {list(self.coords)}")
            pos = _coord_position(list(self.coords[axis]), value)
            if pos is None:
                raise ValueError(f"Value {value} not in {axis} coords: {self.coords[axis]}")
            index[self._axis_names.index(axis)] = pos
        out = self[tuple(index)]
        out._axis_names = [a for a in self._axis_names if a not in picks]
        out.coords = {a: c for a, c in self.coords.items() if a not in picks}
        return out

    @classmethod
    def stack(cls, results: List['SimulationResult'], axis_name: str = 'structural',
              axis_values: Optional[List] = None) -> 'SimulationResult':
        """Results of equal shape side by side on a new leading axis (e.g. one
        result per lattice size, which one run() cannot batch)."""
        if not results:
            raise ValueError("Cannot stack empty list of results")
        head = results[0]
        metrics = MetricsDict((k, np.stack([r.metrics[k] for r in results])) for k in head.metrics)
        drivers = {f: np.stack([getattr(r, f) for r in results]) for f in DRIVER_FIELDS}
        coords = dict(head.coords)
        coords[axis_name] = list(range(len(results))) if axis_values is None else axis_values
        return cls(metrics=metrics, rng_key=results[-1].rng_key, final_state=None, metadata=head.metadata,
                   dt=head.dt, name=f"{head.name}_stacked", grid_shape=metrics['axial_force'].shape[:-1],
                   axis_names=[axis_name, *head._axis_names], coords=coords, **drivers)

    def summary(self) -> str:
        """A few lines describing the cube and its force."""
        res = self.metrics.get('solver_residual')
        axes = ' x '.join(self._axis_names) if self._axis_names else 'unnamed axes'
        text = [f"SimulationResult '{self.name}': {self.axial_force.shape} over {axes}",
                f"  {self.n_steps} steps of {self.dt} ms ({self.n_steps * self.dt:.1f} ms)",
                f"  Mean force {self.mean_force:.2f} pN; last fifth of the run {self.steady_state_force:.2f} pN",
                f"  Largest solver residual {float(np.max(res)) if res is not None and res.size else 0.0:.4f} pN",
                f"  {len(self.metrics)} metrics"
                + (f"; coordinates for {', '.join(self.coords)}" if self.coords else "")]
        return '\n'.join(text)

    def __repr__(self) -> str:
        force = self.metrics.get('axial_force')
        return f"SimulationResult(name='{self.name}', shape={getattr(force, 'shape', '?')}, dt={self.dt})"


__all__ = ['SimulationResult', 'MetricsDict', 'axes_after_index', 'DRIVER_FIELDS']
