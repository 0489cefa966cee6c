"""Continuous-batching simulation server (the serving form of the engine).

Requests -- each one condition with its own lattice, parameters, constant
drivers, duration and key -- are admitted into resident device slots as soon
as the memory budget allows, advanced together by chunked launches of the
fused step kernel, and retired individually as they finish; a request that
arrives while others run joins at the next chunk boundary.  The scheduler is
native (``mf_server_*`` in ``csrc/mf_server.inc``); this module is its Python
face.  Each served result equals the same condition run alone through
``run()`` (the per-condition arithmetic does not depend on its neighbours).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

from .engine import (EngineError, MF_ERR_BUSY, N_METRICS, N_PARAMS, get_engine, mf_request)
from .params import DynamicParams
from .simulation import METRIC_KEYS


@dataclass
class ServedResult:
    req_id: int
    metrics: Dict[str, np.ndarray]     # 52 keys -> [n_steps]
    status: int
    t_submit: float
    t_done: float

    @property
    def latency_s(self) -> float:
        return self.t_done - self.t_submit


class SimulationServer:
    """Admit / run / retire simulation requests on one GPU.

    ``precision`` is the arithmetic of every request: ``'mixed'`` (default,
    as ``run(..., precision='mixed')``) or ``'float32'`` (the reference's).
    ``mem_budget`` bounds the device bytes of resident slots (state, tables,
    metric buffers); ``chunk_steps`` is the scheduling tick in timesteps.
    """

    def __init__(self, mem_budget: int = 2 << 30, chunk_steps: int = 50, max_slots: int = 4096,
                 device: Optional[int] = None, precision: str = 'mixed'):
        if precision not in ('float32', 'mixed'):
            raise ValueError("precision must be 'float32' or 'mixed'")
        self.eng = get_engine(device)
        self.lib = self.eng.lib
        self.precision = precision
        self._check(self.lib.mf_server_start_mode(self.eng.h, int(mem_budget), int(chunk_steps), int(max_slots),
                                                  int(precision == 'mixed')), 'mf_server_start_mode')
        self._steps: Dict[int, int] = {}
        self._open = True

    def _check(self, rc, what):
        if rc != 0:
            msg = self.lib.mf_last_error(self.eng.h)
            raise EngineError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def submit(self, topology, params: DynamicParams, pCa: float, z_line: float, duration_ms: float,
               key, dt: float = 1.0, lattice_spacing: float = 14.0) -> int:
        """Queue one condition; returns its request id."""
        up = self.eng.upload(topology)
        n_steps = int(duration_ms / dt)
        r = mf_request()
        r.topo_id = up.topo_id
        r.n_steps = n_steps
        r.dt = float(dt)
        r.key[0], r.key[1] = int(key[0]), int(key[1])
        row = params.param_row()
        for i in range(N_PARAMS):
            r.params[i] = float(row[i])
        r.pCa, r.z_line, r.lattice_spacing = float(pCa), float(z_line), float(lattice_spacing)
        rid = ctypes.c_uint64()
        self._check(self.lib.mf_server_submit(self.eng.h, ctypes.byref(r), ctypes.byref(rid)), 'mf_server_submit')
        self._steps[rid.value] = n_steps
        return rid.value

    def step(self, max_ticks: int = 1):
        """Run scheduling ticks; returns (n_active, n_queued)."""
        a, q = ctypes.c_int32(), ctypes.c_int32()
        self._check(self.lib.mf_server_step(self.eng.h, int(max_ticks), ctypes.byref(a), ctypes.byref(q)),
                    'mf_server_step')
        return a.value, q.value

    def poll(self, req_id: int) -> Optional[ServedResult]:
        """The finished result of a request (and forget it), or None while it runs."""
        n = self._steps[req_id]
        buf = np.zeros((N_METRICS, n), np.float32)
        st = ctypes.c_int32()
        ts, td = ctypes.c_double(), ctypes.c_double()
        rc = self.lib.mf_server_poll(self.eng.h, ctypes.c_uint64(req_id), buf.ctypes.data, ctypes.byref(st),
                                     ctypes.byref(ts), ctypes.byref(td))
        if rc == MF_ERR_BUSY:
            return None
        self._check(rc, 'mf_server_poll')
        del self._steps[req_id]
        m = {k: (buf[i].astype(np.int32) if k == 'newton_iters' else buf[i]) for i, k in enumerate(METRIC_KEYS)}
        return ServedResult(req_id, m, st.value, ts.value, td.value)

    def cancel(self, req_id: int):
        self._check(self.lib.mf_server_cancel(self.eng.h, ctypes.c_uint64(req_id)), 'mf_server_cancel')
        self._steps.pop(req_id, None)

    def drain(self, max_ticks: int = 1 << 30):
        """Tick until nothing is active or queued."""
        while True:
            a, q = self.step(64)
            if a == 0 and q == 0:
                return
            max_ticks -= 64
            if max_ticks <= 0:
                return

    def close(self):
        if self._open:
            self.lib.mf_server_stop(self.eng.h)
            self._open = False

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
