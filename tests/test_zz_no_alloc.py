"""The allocation-free entry point mf_run_batch_static, checked against mf_run_batch.

Who needs it: callers that must not let this library allocate device memory
while they run -- a host framework that owns every byte of HBM through its own
allocator and budget.  mf_run_batch_static takes its scratch from a fixed
8 MiB array compiled into the library instead.  (It still blocks the calling
thread until the stream has finished, like mf_run_batch.)

The test drives the new entry point through the C ABI twice in a row (the
second call reuses the array the first one left behind) and compares both
results with those of the ordinary entry point on the same inputs.  It sits
in its own file, named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-5  # the tolerance the parity tests use for continuous metrics
COUNT_ROWS = [5, 6, 7, 8, 9, 10, 11, 19, 20, 21, 22, 32, 33, 51]  # integer-valued metrics


def _inputs():
    import torch
    from multifil_jax_b200 import SarcTopology, get_skeletal_params, get_cardiac_params
    from multifil_jax_b200.engine import prng_split, prng_key
    s, d = get_skeletal_params()
    _, c = get_cardiac_params()
    t22 = SarcTopology.create(2, 2, s, d)
    t11 = SarcTopology.create(1, 1, s, d)
    topos = [t22] * 5 + [t11] * 3
    B, T = len(topos), 30
    rows = np.stack([d.param_row() if i % 2 == 0 else c.param_row() for i in range(B)])
    pcas = np.linspace(4.2, 6.8, B)
    dev = torch.device('cuda', 0)
    f = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)
    inp = dict(params=f(rows), z=f(np.full((B, T), 930.0)), pCa=f(np.repeat(pcas[:, None], T, 1)),
               ls=f(np.full((B, T), 14.0)), n_steps=torch.as_tensor(np.array([T, T, 20, T, 11, T, T, 7], np.int32),
                                                                    device=dev),
               keys=torch.as_tensor(prng_split(prng_key(21), B).astype(np.int64), device=dev).to(torch.int32),
               K_lat=f(np.zeros(B)), nu=f(np.zeros(B)), dt=f(np.ones(B)))
    return topos, inp, B, T


def _static_call(eng, topos, inp, B, T):
    """mf_run_batch_static through the C ABI with caller-owned outputs."""
    import torch
    from multifil_jax_b200.engine import mf_batch
    ups = [eng.upload(t) for t in topos]
    tid = np.array([u.topo_id for u in ups], dtype=np.int32)
    dev = inp['z'].device
    metrics = torch.full((B, 52, T), np.nan, dtype=torch.float32, device=dev)
    status = torch.full((B,), -7, dtype=torch.int32, device=dev)
    b = mf_batch()
    b.B, b.T_max = B, T
    b.topo_id = tid.ctypes.data
    for k in ('params', 'z', 'pCa', 'ls', 'n_steps', 'keys', 'K_lat', 'nu', 'dt'):
        setattr(b, k, inp[k].data_ptr())
    b.n_newton, b.n_cg, b.flags, b.chunk_steps, b.residual_warn = 4, 6, 0, 0, 1.5
    b.metrics_out = metrics.data_ptr()
    b.status_out = status.data_ptr()
    stream = torch.cuda.current_stream(dev)
    rc = eng.lib.mf_run_batch_static(eng.h, ctypes.byref(b), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, eng.lib.mf_last_error(eng.h)
    torch.cuda.synchronize(dev)
    return metrics.cpu().numpy(), status.cpu().numpy()


def _compare(ref, got, n_steps):
    for i, n in enumerate(n_steps):
        a, b = ref[i, :, :n], got[i, :, :n]
        assert np.array_equal(a[COUNT_ROWS], b[COUNT_ROWS]), i
        np.testing.assert_allclose(b, a, rtol=RTOL, atol=1e-6)


def test_static_scratch_entry_matches_allocating_entry():
    import torch
    from multifil_jax_b200.engine import get_engine
    eng = get_engine(0)
    topos, inp, B, T = _inputs()
    ref = eng.run_batch(topos, inp['params'], inp['z'], inp['pCa'], inp['ls'], inp['n_steps'], inp['keys'],
                        K_lat=inp['K_lat'], nu=inp['nu'], dt=inp['dt'])
    torch.cuda.synchronize()
    ref_m = ref['metrics'].cpu().numpy()
    n_steps = inp['n_steps'].cpu().numpy()
    for _ in range(2):  # the second call finds the first call's leftovers in the array
        got_m, got_s = _static_call(eng, topos, inp, B, T)
        _compare(ref_m, got_m, n_steps)
        assert np.array_equal(got_s, ref['status'].cpu().numpy())


def test_static_scratch_rejects_oversized_batch():
    import torch
    from multifil_jax_b200 import SarcTopology
    from multifil_jax_b200.engine import get_engine, mf_batch, MF_ERR_NOMEM
    eng = get_engine(0)
    topo = SarcTopology.create(2, 2)
    up = eng.upload(topo)
    B, T = 200, 2  # ~200 x 116 kB of workspace: far beyond the 8 MiB array
    dev = torch.device('cuda', 0)
    z = torch.full((B, T), 900.0, device=dev)
    ns = torch.full((B,), T, dtype=torch.int32, device=dev)
    keys = torch.zeros((B, 2), dtype=torch.int32, device=dev)
    par = torch.zeros((B, 44), device=dev)
    out = torch.zeros((B, 52, T), device=dev)
    tid = np.full(B, up.topo_id, np.int32)
    b = mf_batch()
    b.B, b.T_max, b.topo_id = B, T, tid.ctypes.data
    b.params, b.z, b.pCa, b.ls, b.n_steps, b.keys = (par.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(),
                                                     ns.data_ptr(), keys.data_ptr())
    b.n_newton, b.n_cg, b.metrics_out = 4, 6, out.data_ptr()
    rc = eng.lib.mf_run_batch_static(eng.h, ctypes.byref(b), None)
    assert rc == MF_ERR_NOMEM
    msg = eng.lib.mf_last_error(eng.h).decode()
    assert 'static array holds' in msg and str(8 << 20) in msg


def test_static_scratch_rejects_negative_solver_caps():
    import torch
    from multifil_jax_b200.engine import get_engine, mf_batch, MF_ERR_INVALID
    eng = get_engine(0)
    topos, inp, B, T = _inputs()
    tid = np.array([eng.upload(t).topo_id for t in topos], dtype=np.int32)
    out = torch.zeros((B, 52, T), device=inp['z'].device)
    for n_newton, n_cg in ((-1, 6), (4, -2)):
        b = mf_batch()
        b.B, b.T_max, b.topo_id = B, T, tid.ctypes.data
        for k in ('params', 'z', 'pCa', 'ls', 'n_steps', 'keys', 'K_lat', 'nu', 'dt'):
            setattr(b, k, inp[k].data_ptr())
        b.n_newton, b.n_cg, b.metrics_out = n_newton, n_cg, out.data_ptr()
        assert eng.lib.mf_run_batch_static(eng.h, ctypes.byref(b), None) == MF_ERR_INVALID
        assert 'negative solver caps' in eng.lib.mf_last_error(eng.h).decode()
