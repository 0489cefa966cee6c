"""The metrics buffer may be page-locked host memory (the kernel writes it over
the bus, so no copy follows the launch); pageable host memory is refused
before anything runs on the GPU (needs a B200)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(B=6, T=25):
    import torch
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from multifil_jax_b200.engine import prng_split, prng_key
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    dev = torch.device('cuda', 0)
    f = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)
    inp = dict(params=f(np.tile(d.param_row(), (B, 1))), z=f(np.full((B, T), 910.0)),
               pCa=f(np.repeat(np.linspace(4.3, 6.9, B)[:, None], T, 1)), ls=f(np.full((B, T), 14.0)),
               n_steps=torch.full((B,), T, dtype=torch.int32, device=dev),
               keys=torch.as_tensor(prng_split(prng_key(8), B).astype(np.int64), device=dev).to(torch.int32))
    return topo, inp, B, T


@pytest.mark.parametrize('flags', [0, 'precise'])
def test_metrics_into_page_locked_host_memory(engine, flags):
    import torch
    from multifil_jax_b200.engine import MF_FLAG_PRECISE
    fl = MF_FLAG_PRECISE if flags == 'precise' else 0
    topo, inp, B, T = _inputs()
    args = (topo, inp['params'], inp['z'], inp['pCa'], inp['ls'], inp['n_steps'], inp['keys'])
    ref = engine.run_batch(*args, flags=fl)['metrics'].cpu().numpy()
    host = torch.full((B, 52, T), float('nan'), dtype=torch.float32, pin_memory=True)
    engine.run_batch(*args, flags=fl, metrics_out=host)
    torch.cuda.synchronize()
    assert np.array_equal(host.numpy(), ref)


@pytest.mark.parametrize('entry', ['mf_run_batch', 'mf_run_batch_static'])
def test_pageable_metrics_buffer_is_refused(engine, entry):
    from multifil_jax_b200.engine import mf_batch, MF_ERR_INVALID
    topo, inp, B, T = _inputs()
    tid = np.full(B, engine.upload(topo).topo_id, np.int32)
    pageable = np.zeros((B, 52, T), np.float32)
    b = mf_batch()
    b.B, b.T_max, b.topo_id = B, T, tid.ctypes.data
    for k in ('params', 'z', 'pCa', 'ls', 'n_steps', 'keys'):
        setattr(b, k, inp[k].data_ptr())
    b.n_newton, b.n_cg, b.metrics_out = 4, 6, pageable.ctypes.data
    rc = getattr(engine.lib, entry)(engine.h, ctypes.byref(b), None)
    assert rc == MF_ERR_INVALID
    assert 'pageable' in engine.lib.mf_last_error(engine.h).decode()
    assert not pageable.any()


def test_minibatched_run_equals_one_launch():
    """run(minibatch_size=3) writes each minibatch into its slice of the one
    page-locked block; every metric equals the single-launch run's."""
    from multifil_jax_b200 import SarcTopology, get_skeletal_params, run
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    kw = dict(duration_ms=15, pCa=list(np.linspace(4.2, 6.9, 7)), z_line=[900.0, 940.0],
              dynamic_params=d, static_params=s, rng_seed=3, precision='mixed')
    a = run(topo, **kw)
    b = run(topo, minibatch_size=3, **kw)
    for k in a.metrics:
        assert np.array_equal(a.metrics[k], b.metrics[k]), k
    assert np.array_equal(a.rng_key, b.rng_key)
