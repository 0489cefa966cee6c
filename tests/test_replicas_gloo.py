"""Multi-GPU form on the CPU: the replica plumbing of ``bench.py`` with two gloo ranks.

Conditions are independent, so ``bench.py --gpus N`` runs one replica of the
sweep per rank with no collective on the data path.  What it does need across
ranks is checked here with two processes on the gloo backend:
* the timed region's device time is the maximum over ranks,
* the whole-job value counts every rank's condition-steps over that maximum,
* the reference arm runs on rank 0 only (the other ranks return without work).
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, REPO)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    import argparse
    import bench
    r, w, local = bench._dist()
    assert (r, w, local) == (rank, world, rank)
    dist = bench._init_pg(w, local, 'gloo')
    # each rank's "device time" of its replica; the job takes the slowest
    t_local = 1.0 + rank
    t_max = bench._max_over_ranks(t_local, w, None)
    units = 256 * 500 * 3  # condition-steps of one replica over 3 timed steps
    value = units * w / t_max
    # the reference arm: only rank 0 times the CPU path
    ran = []
    orig = bench.cpu_baseline
    bench.cpu_baseline = lambda *a, **k: ran.append(1) or {'value': 1.0}
    try:
        bench.bench_reference(argparse.Namespace(steps=1, warmup=0))
    finally:
        bench.cpu_baseline = orig
    dist.barrier()
    out[rank] = (t_max, value, len(ran))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_replicas_share_only_the_timing():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0          # max over ranks
    assert res[0][1] == res[1][1] == 256 * 500 * 3 * 2 / 2.0
    assert res[0][2] > 0 and res[1][2] == 0       # reference arm on rank 0 only
