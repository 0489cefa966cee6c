"""ctypes binding of ``libmultifil_b200.so`` and the device-side batch runner.

PyTorch provides device memory and streams; the timestep itself runs in the
hand-written sm_100a kernels behind the C ABI declared in
``include/multifil_b200.h``.  There is no CPU fallback: when the shared library
or a CUDA device is missing every entry point raises :class:`EngineError`.
"""
from __future__ import annotations

import ctypes
import os
import threading
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get('MULTIFIL_B200_LIB', os.path.join(_HERE, 'libmultifil_b200.so'))

MF_FLAG_DYNAMIC_LS = 1
MF_FLAG_PRECISE = 2
MF_FLAG_ORIGINAL_PRNG = 4
MF_FLAG_PLAIN = 8
MF_FLAG_NO_GRAPH = 16
MF_FLAG_CONST_DRIVERS = 32

MF_POP_EXPLICIT = 1
MF_POP_XB = 2
MF_POP_TM = 4

MF_STATUS_NONFINITE = 1
MF_STATUS_NOT_CONVERGED = 2
MF_STATUS_MULTIBIND = 8

MF_ERR_INVALID = -1
MF_ERR_BUSY = -6
MF_ERR_NOMEM = -3

N_METRICS = 52
N_PARAMS = 44


class EngineError(RuntimeError):
    """The CUDA engine is unavailable or a call through the C ABI failed."""


class mf_topo_desc(ctypes.Structure):
    _fields_ = [
        ('n_thick', ctypes.c_int32), ('n_crowns', ctypes.c_int32), ('n_thin', ctypes.c_int32),
        ('n_sites', ctypes.c_int32), ('n_xb_per_crown', ctypes.c_int32),
        ('max_sites_per_face', ctypes.c_int32), ('n_xb_bins', ctypes.c_int32),
        ('xb_to_thin_id', ctypes.c_void_p), ('xb_to_thin_face', ctypes.c_void_p),
        ('xb_valid', ctypes.c_void_p), ('face_to_sites', ctypes.c_void_p),
        ('n_sites_per_face', ctypes.c_void_p), ('tm_prev_neighbor', ctypes.c_void_p),
        ('tm_next_neighbor', ctypes.c_void_p), ('crown_offsets', ctypes.c_void_p),
        ('crown_rests', ctypes.c_void_p), ('binding_offsets', ctypes.c_void_p),
        ('binding_rests', ctypes.c_void_p), ('thin_rest_cumsum', ctypes.c_void_p),
        ('xb_bin_edges', ctypes.c_void_p), ('xb_bin_centers', ctypes.c_void_p),
    ]


class mf_batch(ctypes.Structure):
    _fields_ = [
        ('B', ctypes.c_int32), ('T_max', ctypes.c_int32), ('topo_id', ctypes.c_void_p),
        ('params', ctypes.c_void_p), ('z', ctypes.c_void_p), ('pCa', ctypes.c_void_p),
        ('ls', ctypes.c_void_p), ('n_steps', ctypes.c_void_p), ('keys', ctypes.c_void_p),
        ('K_lat', ctypes.c_void_p), ('nu', ctypes.c_void_p), ('dt', ctypes.c_void_p),
        ('n_newton', ctypes.c_int32), ('n_cg', ctypes.c_int32), ('flags', ctypes.c_int32),
        ('chunk_steps', ctypes.c_int32), ('residual_warn', ctypes.c_float),
        ('metrics_out', ctypes.c_void_p), ('status_out', ctypes.c_void_p),
        ('keys_out', ctypes.c_void_p), ('u_thin', ctypes.c_void_p), ('u_xb', ctypes.c_void_p),
        ('x_trace', ctypes.c_void_p), ('state_trace', ctypes.c_void_p),
        ('bound_trace', ctypes.c_void_p),
        ('n_pops', ctypes.c_int32), ('pop_flags', ctypes.c_int32), ('label_stride', ctypes.c_int32),
        ('pop_params', ctypes.c_void_p), ('pop_frac', ctypes.c_void_p), ('xb_label', ctypes.c_void_p),
        ('tm_label', ctypes.c_void_p),
    ]


class mf_request(ctypes.Structure):
    _fields_ = [
        ('topo_id', ctypes.c_int32), ('n_steps', ctypes.c_int32), ('dt', ctypes.c_float),
        ('key', ctypes.c_uint32 * 2), ('params', ctypes.c_float * N_PARAMS),
        ('pCa', ctypes.c_float), ('z_line', ctypes.c_float), ('lattice_spacing', ctypes.c_float),
    ]


# exported symbol -> (restype, argtypes)
_SIGNATURES = {
    'mf_abi_version': (ctypes.c_int, []),
    'mf_create': (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    'mf_destroy': (ctypes.c_int, [ctypes.c_void_p]),
    'mf_last_error': (ctypes.c_char_p, [ctypes.c_void_p]),
    'mf_upload_topology': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(mf_topo_desc),
                                          ctypes.POINTER(ctypes.c_int32)]),
    'mf_tune_threads': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    'mf_tune_threads_mode': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    'mf_run_batch': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(mf_batch), ctypes.c_void_p]),
    'mf_run_batch_static': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(mf_batch), ctypes.c_void_p]),
    'mf_workspace_bytes': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(mf_batch),
                                          ctypes.POINTER(ctypes.c_uint64)]),
    'mf_transition_tables': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_float,
                                            ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p]),
    'mf_prng_split': (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_void_p]),
    'mf_prng_uniform': (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_void_p]),
    'mf_server_start': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32]),
    'mf_server_start_mode': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32]),
    'mf_server_submit': (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(mf_request),
                                        ctypes.POINTER(ctypes.c_uint64)]),
    'mf_server_step': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_int32)]),
    'mf_server_poll': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double)]),
    'mf_server_cancel': (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    'mf_server_stop': (ctypes.c_int, [ctypes.c_void_p]),
}

_lib = None
_lib_lock = threading.Lock()


def load_library(path: str = LIB_PATH):
    """Load the shared library (no GPU needed) and bind every exported symbol."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise EngineError(f"CUDA engine library not found at {path}; run __graft_entry__.build()")
        lib = ctypes.CDLL(path)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def prng_split(key, n: int, partitionable: bool = True) -> np.ndarray:
    """``jax.random.split(key, n)`` computed by the library's host Threefry."""
    lib = load_library()
    out = np.zeros((n, 2), dtype=np.uint32)
    rc = lib.mf_prng_split(int(key[0]), int(key[1]), n, 1 if partitionable else 0, out.ctypes.data)
    if rc:
        raise EngineError(f"mf_prng_split failed ({rc})")
    return out


def prng_uniform(key, n: int, partitionable: bool = True) -> np.ndarray:
    """``jax.random.uniform(key, (n,))`` (float32) computed by the library's host Threefry."""
    lib = load_library()
    out = np.zeros(n, dtype=np.float32)
    rc = lib.mf_prng_uniform(int(key[0]), int(key[1]), n, 1 if partitionable else 0, out.ctypes.data)
    if rc:
        raise EngineError(f"mf_prng_uniform failed ({rc})")
    return out


def prng_key(seed: int) -> np.ndarray:
    """``jax.random.PRNGKey(seed)`` for 32-bit seeds: ``[0, seed]``."""
    s = int(seed)
    return np.array([(s >> 32) & 0xFFFFFFFF if s >= 0 else 0, s & 0xFFFFFFFF], dtype=np.uint32)


def _torch():
    import torch
    return torch


@dataclass
class _UploadedTopo:
    topo_id: int
    n_dof: int
    total_xbs: int
    n_sites_total: int


def topo_desc_arrays(topo) -> Dict[str, np.ndarray]:
    """Host arrays of a SarcTopology in the layout ``mf_topo_desc`` expects."""
    from .topology import thin_rest_cumsum
    c = np.ascontiguousarray
    # the device lattice has three faces per thin filament; a two-face
    # (invertebrate) lattice gets an empty third face that no head targets
    f2s = np.asarray(topo.face_to_sites, np.int32)
    npf = np.asarray(topo.n_sites_per_face, np.int32)
    if f2s.shape[1] < 3:
        pad = 3 - f2s.shape[1]
        f2s = np.concatenate([f2s, np.full((f2s.shape[0], pad, f2s.shape[2]), -1, np.int32)], axis=1)
        npf = np.concatenate([npf, np.zeros((npf.shape[0], pad), np.int32)], axis=1)
    return dict(
        xb_to_thin_id=c(topo.xb_to_thin_id, dtype=np.int32),
        xb_to_thin_face=c(topo.xb_to_thin_face, dtype=np.int32),
        xb_valid=c(topo.xb_valid, dtype=np.uint8),
        face_to_sites=c(f2s, dtype=np.int32),
        n_sites_per_face=c(npf, dtype=np.int32),
        tm_prev_neighbor=c(topo.tm_prev_neighbor, dtype=np.int32),
        tm_next_neighbor=c(topo.tm_next_neighbor, dtype=np.int32),
        crown_offsets=c(topo.crown_offsets, dtype=np.float32),
        crown_rests=c(topo.crown_rests, dtype=np.float32),
        binding_offsets=c(topo.binding_offsets, dtype=np.float32),
        binding_rests=c(topo.binding_rests, dtype=np.float32),
        thin_rest_cumsum=c(thin_rest_cumsum(topo), dtype=np.float32),
        xb_bin_edges=c(topo.xb_bin_edges, dtype=np.float32),
        xb_bin_centers=c(topo.xb_bin_centers, dtype=np.float32),
    )


class Engine:
    """One device context of the CUDA engine (``mf_create`` ... ``mf_destroy``)."""

    def __init__(self, device: int = 0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise EngineError("multifil_jax_b200 needs a CUDA device; none is available")
        self.lib = load_library()
        self.device = device
        torch.cuda.set_device(device)
        torch.cuda.init()
        h = ctypes.c_void_p()
        rc = self.lib.mf_create(device, ctypes.byref(h))
        if rc:
            raise EngineError(f"mf_create failed ({rc})")
        self.h = h
        self._topos: Dict[tuple, _UploadedTopo] = {}

    def close(self):
        if getattr(self, 'h', None):
            self.lib.mf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.mf_last_error(self.h)
            raise EngineError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def upload(self, topo) -> _UploadedTopo:
        key = topo.size_key()
        if key in self._topos:
            return self._topos[key]
        arrs = topo_desc_arrays(topo)
        d = mf_topo_desc(topo.n_thick, topo.n_crowns, topo.n_thin, topo.n_sites, topo.n_xb_per_crown,
                         topo.max_sites_per_face, topo.n_xb_bins,
                         *[arrs[f].ctypes.data for f in (
                             'xb_to_thin_id', 'xb_to_thin_face', 'xb_valid', 'face_to_sites',
                             'n_sites_per_face', 'tm_prev_neighbor', 'tm_next_neighbor', 'crown_offsets',
                             'crown_rests', 'binding_offsets', 'binding_rests', 'thin_rest_cumsum',
                             'xb_bin_edges', 'xb_bin_centers')])
        tid = ctypes.c_int32()
        self._check(self.lib.mf_upload_topology(self.h, ctypes.byref(d), ctypes.byref(tid)), 'mf_upload_topology')
        up = _UploadedTopo(tid.value, topo.n_dof, topo.total_xbs, topo.n_sites_total)
        self._topos[key] = up
        return up

    def tune_threads(self, topo, threads: int, precision: Optional[str] = None):
        """Set the CTA size of a lattice for one precision mode, or both when None
        (0: back to the library's default)."""
        up = self.upload(topo)
        if precision is None:
            self._check(self.lib.mf_tune_threads(self.h, up.topo_id, int(threads)), 'mf_tune_threads')
        else:
            self._check(self.lib.mf_tune_threads_mode(self.h, up.topo_id, int(precision == 'mixed'), int(threads)),
                        'mf_tune_threads_mode')

    def transition_tables(self, topo, params, pCa: float, d: float, dt: float = 1.0, precision: str = 'float32'):
        """The kernel's transition tables at (pCa, d): cumulative tropomyosin rows
        [27, 4, 4], cumulative crossbridge rows [2, n_bins, 6, 6] (permissiveness,
        bin) and the absorbing-chain entries [2, n_bins, 3] (test hook)."""
        up = self.upload(topo)
        nb = topo.n_xb_bins
        row = np.ascontiguousarray(params, dtype=np.float32).reshape(N_PARAMS)
        tm = np.zeros((27, 4, 4), np.float32)
        xb = np.zeros((2, nb, 6, 6), np.float32)
        pa = np.zeros((2, nb, 3), np.float32)
        self._check(self.lib.mf_transition_tables(self.h, up.topo_id, row.ctypes.data, float(pCa), float(d),
                                                  float(dt), MF_FLAG_PRECISE if precision == 'mixed' else 0,
                                                  tm.ctypes.data, xb.ctypes.data, pa.ctypes.data),
                    'mf_transition_tables')
        return tm, xb, pa

    # ------------------------------------------------------------------
    def run_batch(self, topos, params, z, pCa, ls, n_steps, keys, K_lat=None, nu=None, dt=None,
                  n_newton=4, n_cg=6, flags=0, chunk_steps=0, residual_warn=1.5, stream=None,
                  u_thin=None, u_xb=None, want_x_trace=False, want_state_trace=False, keys_out=None,
                  pops=None, metrics_out=None, n_time=None):
        """Run B conditions through the fused kernel; every array is a torch CUDA tensor.

        ``topos`` is a list of B SarcTopology objects (or one shared).  Returns
        a dict with ``metrics`` [B, 52, T], ``status`` [B] and optional traces.
        ``z``, ``pCa``, ``ls`` are [B, T] traces, or [B] values held for every
        step (then ``n_time`` gives T; MF_FLAG_CONST_DRIVERS).
        ``pops``: subpopulations as a dict ``K``, ``flags`` (MF_POP_*),
        ``rows`` [B, K, 44] float32, ``fractions`` [B, K] float32 and, for
        explicit populations, ``xb_label`` / ``tm_label`` [B, stride] int8
        device tensors.
        """
        torch = _torch()
        dev = torch.device('cuda', self.device)
        if z.dim() == 1:
            if pCa.dim() != 1 or ls.dim() != 1 or n_time is None:
                raise EngineError("drivers held for every step: z, pCa and ls must all be [B] and n_time given")
            B, T = z.shape[0], int(n_time)
            flags = int(flags) | MF_FLAG_CONST_DRIVERS
        else:
            B, T = z.shape
        if not isinstance(topos, (list, tuple)):
            topos = [topos] * B
        by_obj = {}  # one lookup per distinct lattice object, not per condition
        ups = [by_obj[id(t)] if id(t) in by_obj else by_obj.setdefault(id(t), self.upload(t)) for t in topos]
        tid = np.array([u.topo_id for u in ups], dtype=np.int32)
        max_dof = max(u.n_dof for u in ups)
        max_x = max(u.total_xbs for u in ups)
        max_s = max(u.n_sites_total for u in ups)

        def f32(a):
            assert a.is_cuda and a.dtype == torch.float32 and a.is_contiguous()
            return a

        if metrics_out is None:
            metrics = torch.empty((B, N_METRICS, T), dtype=torch.float32, device=dev)
        else:  # device memory, or page-locked host memory the kernel writes over the bus
            assert metrics_out.dtype == torch.float32 and metrics_out.is_contiguous()
            assert tuple(metrics_out.shape) == (B, N_METRICS, T)
            assert metrics_out.is_cuda or metrics_out.is_pinned()
            metrics = metrics_out
        status = torch.zeros(B, dtype=torch.int32, device=dev)
        out = dict(metrics=metrics, status=status)
        xt = st = bt = None
        if want_x_trace:
            xt = torch.zeros((B, T, max_dof), dtype=torch.float32, device=dev)
            out['x_trace'] = xt
        if want_state_trace:
            st = torch.zeros((B, T, max_x + max_s), dtype=torch.int8, device=dev)
            bt = torch.zeros((B, T, max_x + max_s), dtype=torch.int32, device=dev)
            out['state_trace'] = st
            out['bound_trace'] = bt
        bat = mf_batch()
        bat.B, bat.T_max = B, T
        bat.topo_id = tid.ctypes.data
        bat.params = f32(params).data_ptr()
        bat.z = f32(z).data_ptr()
        bat.pCa = f32(pCa).data_ptr()
        bat.ls = f32(ls).data_ptr()
        assert n_steps.dtype == torch.int32
        bat.n_steps = n_steps.data_ptr()
        bat.keys = keys.data_ptr()
        bat.K_lat = f32(K_lat).data_ptr() if K_lat is not None else None
        bat.nu = f32(nu).data_ptr() if nu is not None else None
        bat.dt = f32(dt).data_ptr() if dt is not None else None
        bat.n_newton, bat.n_cg, bat.flags = int(n_newton), int(n_cg), int(flags)
        bat.chunk_steps = int(chunk_steps)
        bat.residual_warn = float(residual_warn)
        bat.metrics_out = metrics.data_ptr()
        bat.status_out = status.data_ptr()
        bat.keys_out = keys_out.data_ptr() if keys_out is not None else None
        bat.u_thin = f32(u_thin).data_ptr() if u_thin is not None else None
        bat.u_xb = f32(u_xb).data_ptr() if u_xb is not None else None
        bat.x_trace = xt.data_ptr() if xt is not None else None
        bat.state_trace = st.data_ptr() if st is not None else None
        bat.bound_trace = bt.data_ptr() if bt is not None else None
        if pops is not None and int(pops['K']) > 1:
            bat.n_pops, bat.pop_flags = int(pops['K']), int(pops['flags'])
            bat.pop_params = f32(pops['rows']).data_ptr()
            bat.pop_frac = f32(pops['fractions']).data_ptr()
            stride = 0
            for name in ('xb_label', 'tm_label'):
                lab = pops.get(name)
                if lab is not None:
                    assert lab.is_cuda and lab.dtype == torch.int8 and lab.is_contiguous() and lab.shape[0] == B
                    stride = lab.shape[1] if stride == 0 else stride
                    assert lab.shape[1] == stride
                    setattr(bat, name, lab.data_ptr())
            bat.label_stride = int(stride)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        rc = self.lib.mf_run_batch(self.h, ctypes.byref(bat), ctypes.c_void_p(s.cuda_stream))
        if rc == MF_ERR_INVALID and not metrics.is_cuda and b'not mapped' in (self.lib.mf_last_error(self.h) or b''):
            # page-locked memory the device cannot address at the same pointer
            # (a host allocator that registers pages without mapping them):
            # run into device memory and copy, as for any other caller
            dm = torch.empty((B, N_METRICS, T), dtype=torch.float32, device=dev)
            bat.metrics_out = dm.data_ptr()
            rc = self.lib.mf_run_batch(self.h, ctypes.byref(bat), ctypes.c_void_p(s.cuda_stream))
            if rc == 0:
                with torch.cuda.stream(s):
                    metrics.copy_(dm, non_blocking=True)
        self._check(rc, 'mf_run_batch')
        return out


_engines: Dict[int, Engine] = {}


def get_engine(device: Optional[int] = None) -> Engine:
    torch = _torch()
    if not torch.cuda.is_available():
        raise EngineError("multifil_jax_b200 needs a CUDA device; none is available")
    d = torch.cuda.current_device() if device is None else device
    if d not in _engines:
        _engines[d] = Engine(d)
    return _engines[d]


def _flags_for(plan, precision: str) -> int:
    f = 0
    if plan.dynamic_ls:
        f |= MF_FLAG_DYNAMIC_LS
    if precision == 'mixed':
        f |= MF_FLAG_PRECISE
    return f


def upload(dev, *arrays):
    """Host arrays -> device tensors of the same dtype and shape, staged in
    one page-locked buffer and moved by one copy (instead of one pageable,
    synchronous copy per array)."""
    torch = _torch()
    tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.int32): torch.int32}
    arrays = [np.ascontiguousarray(a) for a in arrays]
    offs, total = [], 0
    for a in arrays:
        offs.append(total)
        total += (a.nbytes + 15) & ~15
    host = torch.empty(max(total, 16), dtype=torch.uint8, pin_memory=True)
    hn = host.numpy()
    for a, o in zip(arrays, offs):
        hn[o:o + a.nbytes] = a.reshape(-1).view(np.uint8)
    d = host.to(dev, non_blocking=True)
    return [d[o:o + a.nbytes].view(tdt[a.dtype]).view(a.shape) for a, o in zip(arrays, offs)]


def device_pops(sp, dev):
    """A :class:`~multifil_jax_b200.subpopulation.ResolvedSubpop` as the device
    tensors ``Engine.run_batch(pops=...)`` takes."""
    torch = _torch()
    flags = (MF_POP_EXPLICIT if sp.explicit else 0) | (MF_POP_XB if sp.xb else 0) | (MF_POP_TM if sp.tm else 0)
    rows, frac = upload(dev, np.ascontiguousarray(sp.rows, np.float32), np.ascontiguousarray(sp.fractions, np.float32))
    out = dict(K=sp.K, flags=flags, rows=rows, fractions=frac)
    if sp.explicit:
        B = sp.rows.shape[0]
        stride = max(sp.xb_label.shape[1], sp.tm_label.shape[1])
        for name in ('xb_label', 'tm_label'):
            lab = np.zeros((B, stride), np.int8)
            src = getattr(sp, name)
            lab[:, :src.shape[1]] = src
            out[name] = torch.as_tensor(lab).to(dev)
    return out


def host_metrics(B: int, T: int):
    """A page-locked host block for [B, 52, T] metrics that the kernels write
    over the bus (``Engine.run_batch(metrics_out=...)``): the launch leaves
    the result on the host, with no device buffer and no copy after it.
    Blocks come from torch's caching host allocator, so a loop of calls that
    drops each result before the next reuses the same pages."""
    torch = _torch()
    return torch.empty((B, N_METRICS, T), dtype=torch.float32, pin_memory=True)


def execute_plan(topology, plan, static_params, precision: str = 'float32', device: Optional[int] = None,
                 minibatch_size="auto", chunk_steps: int = 0, stream=None, key_major: bool = False,
                 status_out: Optional[np.ndarray] = None) -> np.ndarray:
    """Run every condition of a BatchPlan on the GPU; returns host metrics [B, 52, T]
    (``key_major``: a [52, B, T] view of the same block, one metric per leading
    index).  The kernels write the metrics straight into page-locked host
    memory.  ``status_out`` (int32 [B]) receives every condition's MF_STATUS_*
    bits."""
    torch = _torch()
    eng = get_engine(device)
    dev = torch.device('cuda', eng.device)
    B, T = plan.total, plan.n_steps
    if B == 0 or T == 0:
        return np.zeros((N_METRICS, B, T) if key_major else (B, N_METRICS, T), dtype=np.float32)
    if minibatch_size in (None, "auto"):
        chunk = B
    else:
        chunk = max(1, int(minibatch_size))
    flags = _flags_for(plan, precision)
    out = host_metrics(B, T)
    with torch.cuda.device(dev):
        for s in range(0, B, chunk):
            e = min(B, s + chunk)
            n = e - s

            drv = (plan.z[s:e, 0], plan.pCa[s:e, 0], plan.ls[s:e, 0]) if plan.const_drivers else \
                (plan.z[s:e], plan.pCa[s:e], plan.ls[s:e])
            P, Z, PC, L, K, KL, NU = upload(dev, plan.params[s:e], *drv,
                                            plan.keys[s:e].astype(np.uint32).view(np.int32), plan.K_lat[s:e],
                                            plan.nu[s:e])
            pops = device_pops(plan.subpop.take(s, e), dev) if plan.subpop is not None else None
            res = eng.run_batch([topology] * n, P, Z, PC, L,
                                torch.full((n,), T, dtype=torch.int32, device=dev), K,
                                K_lat=KL, nu=NU,
                                dt=torch.full((n,), plan.dt, dtype=torch.float32, device=dev),
                                n_newton=static_params.n_newton_steps, n_cg=static_params.n_cg_steps,
                                flags=flags, chunk_steps=chunk_steps,
                                residual_warn=static_params.solver_residual_tol, stream=stream, pops=pops,
                                metrics_out=out[s:e], n_time=T)
            if status_out is not None:
                status_out[s:e] = res['status'].cpu().numpy()
        (stream if stream is not None else torch.cuda.current_stream(dev)).synchronize()
    m = out.numpy()
    return m.transpose(1, 0, 2) if key_major else m
