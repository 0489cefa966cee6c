"""Benchmark: condition-timesteps/s on the 256-condition pCa sweep (2x2 skeletal, 500 ms).

One bench step = the whole sweep (256 conditions x 500 timesteps) through the
fused kernel in one launch.  Prints ONE JSON line on rank 0.

  value    device throughput with inputs resident in HBM (CUDA events, L2
           flushed between steps, max over ranks)
  e2e      the same sweep through the public run() with host inputs, host
           metrics out (H2D + kernel + D2H inside the timed region)
  plain    one condition per launch, one launch per timestep (baseline form)
  serving  continuous batching of a Poisson request stream, p50/p99 latency

``--impl reference`` times the CPU restatement of the reference algorithm (the
reference's JAX CPU path cannot be installed here) on all host cores.
Multi-GPU: replicas only -- every rank runs its own copy of the sweep.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

B_SWEEP, T_SWEEP = 256, 500
# DRAM bytes (read + write) of one launch of the mixed-precision sweep, from
# ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum on this workload
TRAFFIC_PER_LAUNCH = 2.69e6 + 45.97e6
METRIC = 'condition-timesteps/s'


def _dist():
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    return rank, world, local


def _init_pg(world, local, backend):
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault('MASTER_ADDR', '127.0.0.1')
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=120))
    return dist


def _max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(REPO, '_build', f'clocks_{os.getpid()}.csv')

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.gpu}', f'--query-gpu={self.Q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [l.split(',') for l in open(self.path).read().strip().splitlines() if l.strip()]
        except Exception:
            rows = []
        if not rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        sm = [float(r[1]) for r in rows if r[1].strip().replace('.', '').isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].strip() == 'Active'})
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(rows)}


E2E_WARMUP = 2


def sweep_inputs():
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from multifil_jax_b200.simulation import plan_batch
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    pcas = list(np.linspace(4.0, 7.0, B_SWEEP))
    plan = plan_batch(topo, duration_ms=T_SWEEP, pCa=pcas, z_line=900.0, dynamic_params=d, static_params=s,
                      rng_seed=0)
    return topo, s, d, pcas, plan


# ---------------------------------------------------------------------------
# algorithmic work of one condition-timestep
# ---------------------------------------------------------------------------
# Floating-point operations of the reference algorithm on the 2x2 lattice,
# per unit of work, from an op-counting run of the oracle (`python -m
# oracle.opcount`, which counts every element operation of the oracle's
# timestep by phase; tests/test_opcount.py checks these values against a
# fresh count).  A step costs per_step + Newton iterations x per_newton; each
# condition of a fixed-spacing, fixed-pCa launch builds its sampling and
# absorbing tables once (per_table_build each, the squarings at each
# matrix's own s).
OPCOUNT_2X2 = {'per_step_flops': 68740.1, 'per_newton_flops': 269191.35294117645, 'per_step_sfu': 1272.0,
               'per_newton_sfu': 8792.0, 'table_build_flops': 2617894, 'absorbing_build_flops': 2521696}


def flops_per_condition_step(iters, steps_per_build):
    """Op-counted flops (and SFU calls) per condition-timestep of the sweep."""
    c = OPCOUNT_2X2
    f = c['per_step_flops'] + iters * c['per_newton_flops'] + \
        (c['table_build_flops'] + c['absorbing_build_flops']) / steps_per_build
    sfu = c['per_step_sfu'] + iters * c['per_newton_sfu']
    return f, sfu


def fp32_peak_tflops(sm_mhz, n_sm=148):
    """FP32 CUDA-core peak: SMs x 128 lanes x 2 (fused multiply-add) x clock."""
    return n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12


# ---------------------------------------------------------------------------
def bench_gpu(args):
    import torch
    rank, world, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    _init_pg(world, local, 'nccl')
    from multifil_jax_b200 import run
    from multifil_jax_b200.engine import get_engine, MF_FLAG_PLAIN, MF_FLAG_PRECISE
    eng = get_engine(local)
    topo, s, d, pcas, plan = sweep_inputs()
    flags = MF_FLAG_PRECISE if args.precision == 'mixed' else 0
    B, T = plan.total, plan.n_steps

    def dv(a, dt=torch.float32):
        return torch.as_tensor(np.ascontiguousarray(a), device=dev).to(dt).contiguous()
    P, Z, PC, L = dv(plan.params), dv(plan.z), dv(plan.pCa), dv(plan.ls)
    NS = torch.full((B,), T, dtype=torch.int32, device=dev)
    K = dv(plan.keys.astype(np.int64), torch.int64).to(torch.int32)
    Kl, NU, DT = dv(plan.K_lat), dv(plan.nu), torch.ones(B, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def one_step():
        return eng.run_batch(topo, P, Z, PC, L, NS, K, K_lat=Kl, nu=NU, dt=DT, flags=flags,
                             n_newton=s.n_newton_steps, n_cg=s.n_cg_steps, stream=stream)
    clk = ClockSampler(local)
    clk.__enter__()  # sampling spans warm-up and the timed region (GPU busy throughout)
    for _ in range(args.warmup):
        out = one_step()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if True:
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            ev[k][0].record(stream)
            out = one_step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    clk.__exit__()
    if world > 1:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    t_dev = sum(ms) / 1e3
    t_dev = _max_over_ranks(t_dev, world, dev)
    value = B * T * args.steps * world / t_dev
    met = out['metrics'].cpu().numpy()
    iters_mean = float(met[:, 51, :].mean())
    nbound_mean = float(met[:, 5, :].mean())
    clocks = clk.summary()

    # e2e: the public API with host buffers (plan, H2D, kernel, D2H inside).  The
    # untimed calls first let the page-locked result blocks reach their steady
    # state (each call's result is dropped after the next one returns).
    e2e_times = []
    for k in range(E2E_WARMUP + max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = run(topo, duration_ms=T_SWEEP, pCa=pcas, z_line=900.0, dynamic_params=d, static_params=s,
                rng_seed=0, precision=args.precision)
        t1 = time.perf_counter()
        if k >= E2E_WARMUP:
            e2e_times.append(t1 - t0)
    t_e2e = _max_over_ranks(float(np.sum(e2e_times)), world, dev)
    e2e_value = B * T * len(e2e_times) * world / t_e2e
    # drivers constant in time go up as one value per condition (MF_FLAG_CONST_DRIVERS)
    drv_bytes = 3 * 4 * B if plan.const_drivers else plan.z.nbytes + plan.pCa.nbytes + plan.ls.nbytes
    h2d = plan.params.nbytes + drv_bytes + plan.keys.nbytes + plan.K_lat.nbytes + plan.nu.nbytes + 2 * 4 * B
    d2h = B * 52 * T * 4

    # plain: one condition per launch, one launch per timestep, on a subset
    nplain = args.plain_conditions
    res_plain = None
    if nplain > 0:
        sl = slice(0, nplain)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.run_batch(topo, P[sl].contiguous(), Z[sl].contiguous(), PC[sl].contiguous(), L[sl].contiguous(),
                      NS[sl].contiguous(), K[sl].contiguous(), K_lat=Kl[sl].contiguous(), nu=NU[sl].contiguous(),
                      dt=DT[sl].contiguous(), flags=flags | MF_FLAG_PLAIN, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t_plain = e0.elapsed_time(e1) / 1e3
        res_plain = nplain * T / t_plain

    # the other precision mode, device-timed the same way (for the record)
    other = 'float32' if args.precision == 'mixed' else 'mixed'
    oflags = MF_FLAG_PRECISE if other == 'mixed' else 0
    eng.run_batch(topo, P, Z, PC, L, NS, K, K_lat=Kl, nu=NU, dt=DT, flags=oflags, stream=stream)
    oe = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        oe[k][0].record(stream)
        eng.run_batch(topo, P, Z, PC, L, NS, K, K_lat=Kl, nu=NU, dt=DT, flags=oflags, stream=stream)
        oe[k][1].record(stream)
    torch.cuda.synchronize()
    other_value = B * T * args.steps / (sum(a.elapsed_time(b) for a, b in oe) / 1e3)

    flops, sfu = flops_per_condition_step(iters_mean, T)
    sm_mhz = clocks.get('sm_mhz') or 1965.0
    fp32_peak = fp32_peak_tflops(sm_mhz)
    launch_s = t_dev / args.steps / world if world == 1 else t_dev / args.steps
    achieved_tf = flops * (B * T) / launch_s / 1e12
    peaks_path = os.path.join(REPO, 'MEASURED_PEAKS.json')
    if os.path.exists(peaks_path):
        peaks, peak_source = json.load(open(peaks_path)), 'measured (copy bandwidth of this pool)'
    else:
        peaks, peak_source = {'hbm_gbs': 6650.0}, 'fallback (earlier measurement on this pool)'
    hbm_bytes_step = B * T * (52 * 4 + 3 * 4)  # metrics written + drivers read (algorithmic)
    hbm_gbs = hbm_bytes_step / launch_s / 1e9
    line = {
        'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': t_dev / args.steps * 1e3, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32' if args.precision == 'float32' else 'f32+f64',
        'data': 'synthetic (pCa sweep inputs, random keys from PRNGKey(0))',
        'config': {'workload': '256-condition pCa sweep, 2x2 skeletal lattice, pCa=linspace(4,7,256), '
                               'z_line=900 nm, 500 ms at dt=1 ms, keys split(PRNGKey(0),256)',
                   'conditions': B, 'timesteps': T, 'precision': args.precision, 'parallelism': f'replicas{world}',
                   'l2': 'flushed between timed steps (256 MB write)', 'launches_per_step': 1,
                   'plain_conditions': nplain, 'plain_condition_timesteps_per_s': res_plain,
                   'batched_over_plain': (value / world / res_plain) if res_plain else None,
                   'mean_newton_iters': iters_mean, 'mean_bound_heads': nbound_mean,
                   f'{other}_value': other_value,
                   'precision_modes': 'mixed = node displacements + float64 residual test + renormalised '
                                      'float64 expm squaring (<=1e-5 force error vs the FP64 oracle); '
                                      'float32 = the reference\'s single-precision arithmetic'},
        'e2e': {'value': e2e_value, 'unit': METRIC, 'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': int(d2h),
                'warmup_calls': E2E_WARMUP,
                'd2h_path': 'the kernel writes the metrics into page-locked host memory over the bus '
                            '(inside the launch, no copy after it)'},
        'gpu_launches': args.steps,
        'roofline': {'bound': 'fp32', 'achieved': achieved_tf, 'peak': fp32_peak, 'unit': 'TFLOP/s',
                     'frac': achieved_tf / fp32_peak,
                     'peak_source': f'148 SMs x 128 FP32 lanes x 2 x median SM clock under load ({sm_mhz:.0f} MHz); '
                                    'no measured FP32 figure exists for this pool',
                     'flops_per_condition_step': flops, 'sfu_calls_per_condition_step': sfu,
                     'flops_source': 'op-counting run of the oracle (python -m oracle.opcount): per step '
                                     f"{OPCOUNT_2X2['per_step_flops']:.0f} + {iters_mean:.3f} Newton iterations x "
                                     f"{OPCOUNT_2X2['per_newton_flops']:.0f} + one sampling and one absorbing "
                                     f'table build per condition over {T} steps',
                     'traffic': args.traffic if args.traffic is not None else (
                         TRAFFIC_PER_LAUNCH if (B, T, args.precision) == (256, 500, 'mixed') else None),
                     'traffic_unit': 'DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum, ncu)',
                     'note': 'not a tensor-core contraction and not HBM-bound: state stays on chip, the step is a '
                             'chain of dependent CUDA-core and shared-memory operations per condition'},
        'roofline_hbm': {'bound': 'hbm', 'achieved': hbm_gbs, 'peak': peaks['hbm_gbs'], 'unit': 'GB/s',
                         'frac': hbm_gbs / peaks['hbm_gbs'], 'peak_source': peak_source,
                         'algorithmic_bytes_per_condition_step': 220},
        'clocks': clocks,
    }
    if rank == 0 and not args.no_workloads:
        line['uneven'] = measure_uneven(args)
        sin, _, _ = measure_sinusoid(args)
        line['sinusoid'] = sin
        if args.serve_requests > 0:
            line['serving'] = measure_serving(args)
    if rank == 0 and not args.no_cpu_baseline:
        line['cpu_baseline'] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def bench_serving(args, device):
    """Poisson arrivals of mixed requests through the continuous-batching server."""
    from multifil_jax_b200 import SarcTopology, get_skeletal_params, get_cardiac_params
    from multifil_jax_b200.serve import SimulationServer
    from multifil_jax_b200.engine import prng_split, prng_key
    rng = np.random.default_rng(1)
    n = args.serve_requests
    topos = {}
    reqs = []
    for i in range(n):
        r, c = (int(v) for v in rng.integers(1, args.serve_max_lattice + 1, 2))
        preset = 'skeletal' if rng.random() < 0.5 else 'cardiac'
        key = (r, c, preset)
        if key not in topos:
            sp = get_skeletal_params() if preset == 'skeletal' else get_cardiac_params()
            topos[key] = (SarcTopology.create(r, c, *sp), sp[1])
        dur = float(rng.uniform(args.serve_min_ms, args.serve_max_ms))
        reqs.append((key, float(rng.uniform(4, 7)), float(rng.uniform(850, 1000)), dur,
                     prng_split(prng_key(1000 + i), 1)[0]))
    total_steps = sum(int(r[3]) for r in reqs)
    srv = SimulationServer(mem_budget=args.serve_budget_gb << 30, chunk_steps=args.serve_chunk, device=device,
                           precision=args.precision)
    # arrival rate: a fraction of the measured batched capacity for this mix
    lam = args.serve_rate
    t_arr = np.cumsum(rng.exponential(1.0 / lam, n))
    ids = {}
    t0 = time.perf_counter()
    i = 0
    while i < n or srv.step(0) != (0, 0):
        now = time.perf_counter() - t0
        while i < n and t_arr[i] <= now:
            k, pCa, z, dur, key = reqs[i]
            ids[srv.submit(topos[k][0], topos[k][1], pCa, z, dur, key)] = i
            i += 1
        a, q = srv.step(1)
        if a == 0 and q == 0 and i < n:
            time.sleep(max(0.0, min(0.002, t_arr[i] - (time.perf_counter() - t0))))
        if i >= n and a == 0 and q == 0:
            break
    t_end = time.perf_counter() - t0
    lat = []
    for rid in list(ids):
        r = srv.poll(rid)
        if r is not None:
            lat.append(r.latency_s)
    srv.close()
    lat = np.array(lat)
    return {'requests': n, 'completed': int(lat.size), 'arrival_rate_per_s': lam,
            'p50_latency_s': float(np.percentile(lat, 50)) if lat.size else None,
            'p99_latency_s': float(np.percentile(lat, 99)) if lat.size else None,
            'condition_timesteps_per_s': total_steps / t_end, 'wall_s': t_end,
            'mix': f'lattice 1..{args.serve_max_lattice} square/rect, duration U[{args.serve_min_ms},{args.serve_max_ms}] ms, '
                   f'skeletal/cardiac 50/50, chunk {args.serve_chunk} steps, {args.precision} precision'}


def _oracle_sample(args_tuple):
    nr, nc, T, pCa, seed = args_tuple
    import numpy as np
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from oracle import step as OS, prng
    s, d = get_skeletal_params()
    topo = SarcTopology.create(nr, nc, s, d)
    key = prng.split(prng.PRNGKey(0), 256)[seed]
    t0 = time.perf_counter()
    OS.run_condition(topo, d.param_row(), np.full(T, 900.0), np.full(T, pCa), np.full(T, 14.0), key)
    return time.perf_counter() - t0


def cpu_baseline(args, cores=1, n_cond=8, T=150, pool=None):
    """The oracle (NumPy restatement of the reference timestep) on host cores:
    n_cond conditions spread over the sweep's pCa range (their keys), T steps
    each.  With ``pool`` (worker processes already started and warmed) the
    conditions run in parallel and only their work is timed."""
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    idx = np.linspace(0, 255, n_cond).round().astype(int)
    jobs = [(2, 2, T, float(np.linspace(4.0, 7.0, 256)[i]), int(i)) for i in idx]
    t0 = time.perf_counter()
    if pool is not None:
        pool.map(_oracle_sample, jobs, chunksize=1)
    else:
        for j in jobs:
            _oracle_sample(j)
    dt = time.perf_counter() - t0
    return {'value': n_cond * T / dt, 'unit': METRIC, 'cores': cores, 'kind': 'port',
            'sample': f'{n_cond} conditions of the 2x2 pCa sweep (pCa spread over 4..7, their sweep keys) x '
                      f'{T} timesteps (oracle, NumPy float32)'}


def bench_reference(args):
    """--impl reference: the reference algorithm on the host CPU (JAX is not installable here).

    One worker process per host core, started and warmed before timing; each
    timed step runs two conditions per core for 60 timesteps."""
    rank, world, local = _dist()
    if rank != 0:
        return
    import multiprocessing as mp
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    cores = len(os.sched_getaffinity(0))
    n_cond, T = 2 * cores, 60
    vals = []
    with mp.get_context('spawn').Pool(cores) as pool:
        pool.map(_oracle_sample, [(2, 2, 2, 4.5, 0)] * cores, chunksize=1)  # start and import in every worker
        for _ in range(args.warmup):
            cpu_baseline(args, cores=cores, n_cond=cores, T=5, pool=pool)
        for _ in range(args.steps):
            vals.append(cpu_baseline(args, cores=cores, n_cond=n_cond, T=T, pool=pool)['value'])
    v = float(np.mean(vals))
    print(json.dumps({
        'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': METRIC, 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': '256-condition pCa sweep, 2x2 skeletal lattice, 500 ms (sampled)',
                   'note': 'reference JAX path not installable (no jax wheel offline); its NumPy restatement '
                           '(oracle) runs instead, one worker process per host core'},
        'cpu_baseline': {'value': v, 'unit': METRIC, 'cores': cores, 'kind': 'port',
                         'sample': f'{n_cond} conditions x {T} timesteps per step (each from its initial '
                                   f'equilibrium), 2x2 lattice, pool started before timing'},
        'e2e': {'value': v, 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)


def profile_case(args):
    """One warm-up and one measured launch of the fused kernel (profiling target)."""
    import torch
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from multifil_jax_b200.simulation import plan_batch
    from multifil_jax_b200.engine import get_engine, MF_FLAG_PRECISE, MF_FLAG_DYNAMIC_LS
    parts = [int(v) for v in args.profile_case.split(',')]
    B, T = parts[0], parts[1]
    n = parts[2] if len(parts) > 2 else 2
    dyn = len(parts) > 3 and parts[3] != 0  # lattice spacing solved as an unknown (K_lat 5, nu 0.5)
    s, d = get_skeletal_params()
    topo = SarcTopology.create(n, n, s, d)
    plan = plan_batch(topo, duration_ms=T, pCa=list(np.linspace(4.0, 7.0, B)), dynamic_params=d, static_params=s)
    dev = torch.device('cuda', 0)
    dv = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev).to(torch.float32).contiguous()
    eng = get_engine(0)
    keys = torch.as_tensor(plan.keys.astype(np.int64), device=dev).to(torch.int32)
    NS = torch.full((B,), T, dtype=torch.int32, device=dev)
    flags = MF_FLAG_PRECISE if args.precision == 'mixed' else 0
    kw = {}
    if dyn:
        flags |= MF_FLAG_DYNAMIC_LS
        kw = dict(K_lat=torch.full((B,), 5.0 * topo.n_thick, device=dev), nu=torch.full((B,), 0.5, device=dev))
    for _ in range(2):
        out = eng.run_batch(topo, dv(plan.params), dv(plan.z), dv(plan.pCa), dv(plan.ls), NS, keys, flags=flags,
                            **kw)
    torch.cuda.synchronize()
    print(json.dumps({'profile_case': [B, T, n, int(dyn)],
                      'force_last_mean': float(out['metrics'][:, 0, -1].mean())}))


# ---------------------------------------------------------------------------
# workload studies (one JSON line each, separate from the benchmark line)
# ---------------------------------------------------------------------------
def uneven_conditions(n=512, seed=0):
    """512 conditions: lattices nrows, ncols ~ U{1..4}, z ~ U[850, 1000] nm,
    pCa ~ U[4, 7], duration ~ U[200, 1000] ms, lattice spacing solved as an
    unknown with K_lat = 5, nu = 0.5, skeletal parameters, keys
    split(PRNGKey(0), 512)[i]."""
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from multifil_jax_b200.engine import prng_split, prng_key
    rng = np.random.default_rng(seed)
    s, d = get_skeletal_params()
    topos, conds = {}, []
    keys = prng_split(prng_key(0), n)
    for i in range(n):
        r, c = (int(v) for v in rng.integers(1, 5, 2))
        if (r, c) not in topos:
            topos[(r, c)] = SarcTopology.create(r, c, s, d)
        conds.append(dict(topology=topos[(r, c)], z_line=float(rng.uniform(850, 1000)),
                          pCa=float(rng.uniform(4, 7)), duration_ms=float(int(rng.uniform(200, 1000))),
                          K_lat=5.0, nu=0.5, dynamic_params=d, key=keys[i]))
    return conds, topos


def measure_uneven(args):
    """Uneven-batch workload (one run_conditions call, host arrays in and
    host metrics out): 512 conditions of lattices 1-4 x 1-4, lattice spacing
    solved as an unknown, default CTA sizes."""
    import torch
    from multifil_jax_b200 import run_conditions
    conds, topos = uneven_conditions()
    total = sum(int(c['duration_ms']) for c in conds)
    run_conditions(conds, precision=args.precision)  # warm-up: every kernel variant loaded
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run_conditions(conds, precision=args.precision)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return {'workload': '512 conditions, nrows/ncols ~ U{1..4}, z ~ U[850,1000] nm, pCa ~ U[4,7], '
                        '200-1000 ms at dt 1 ms, dynamic lattice spacing (K_lat 5, nu 0.5), skeletal, '
                        'keys split(PRNGKey(0),512), one launch through run_conditions',
            'conditions': len(conds), 'condition_timesteps': total, 'value': total / wall, 'unit': METRIC,
            'wall_s': wall, 'precision': args.precision}


def measure_sinusoid(args, modes=('mixed',)):
    """Sinusoid workload: 512 conditions of uneven length and dt in one launch
    per precision mode (device-timed); returns throughput and the forces."""
    import torch
    from multifil_jax_b200 import SarcTopology, get_skeletal_params
    from multifil_jax_b200.engine import get_engine, upload, MF_FLAG_PRECISE
    s, d = get_skeletal_params()
    topo = SarcTopology.create(2, 2, s, d)
    eng = get_engine(0)
    dev = torch.device('cuda', 0)
    conds = sinusoid_conditions()
    B, T = len(conds), max(c[2] for c in conds)
    Z = np.zeros((B, T), np.float32)
    NS = np.zeros(B, np.int32)
    DT = np.zeros(B, np.float32)
    KEYS = np.zeros((B, 2), np.uint32)
    for i, (f, dt, n, z, key) in enumerate(conds):
        Z[i, :n], Z[i, n:] = z, z[-1]
        NS[i], DT[i], KEYS[i] = n, dt, key
    P = np.tile(d.param_row(), (B, 1)).astype(np.float32)
    PC = np.full((B, T), 4.5, np.float32)
    L = np.full((B, T), 14.0, np.float32)
    total = int(NS.sum())
    out = {'workload': '2x2 skeletal, pCa 4.5, z = 900 + 2 sin(2 pi f t) nm, f = logspace(0, 2.7, 64) Hz x 8 '
                       'seeds, dt = min(1, 1000/(20 f)) ms, 5 cycles (>= 200 ms), one launch per mode',
           'conditions': B, 'condition_timesteps': total, 'unit': METRIC}
    forces = {}
    for name in modes:
        flags = MF_FLAG_PRECISE if name == 'mixed' else 0
        a = upload(dev, P, Z, PC, L, NS, KEYS.view(np.int32), np.zeros(B, np.float32), np.zeros(B, np.float32), DT)
        kw = dict(K_lat=a[6], nu=a[7], dt=a[8], n_newton=s.n_newton_steps, n_cg=s.n_cg_steps, flags=flags)
        eng.run_batch(topo, *a[:6], **kw)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = eng.run_batch(topo, *a[:6], **kw)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        forces[name] = res['metrics'][:, 0, :].cpu().numpy()
        out[f'{name}_value'] = total / (ms / 1e3)
        out[f'{name}_ms'] = ms
    return out, conds, forces


def measure_serving(args):
    """Serving workload: capacity of the request mix (every request at t = 0),
    then a Poisson stream at a fraction of that capacity, and the plain path on
    a sample of the same mix for the served-over-plain ratio."""
    cap_args = argparse.Namespace(**vars(args))
    cap_args.serve_requests = args.serve_capacity_requests
    cap_args.serve_rate = 1e9
    cap = bench_serving(cap_args, 0)
    cap_req = cap['requests'] / cap['wall_s']
    run_args = argparse.Namespace(**vars(args))
    run_args.serve_rate = args.serve_load * cap_req
    res = bench_serving(run_args, 0)
    plain = plain_on_request_mix(args)
    res.update({'capacity_requests_per_s': cap_req,
                'capacity_condition_timesteps_per_s': cap['condition_timesteps_per_s'],
                'load_fraction_of_capacity': args.serve_load,
                'plain_condition_timesteps_per_s': plain['value'],
                'served_over_plain': res['condition_timesteps_per_s'] / plain['value'],
                'capacity_over_plain': cap['condition_timesteps_per_s'] / plain['value'],
                'plain_sample': plain['sample']})
    return res


def plain_on_request_mix(args, n=32, steps=40):
    """The plain form (one condition per launch, one launch per timestep) on
    the first n requests of the serving mix, each cut to `steps` steps."""
    import torch
    from multifil_jax_b200 import SarcTopology, get_skeletal_params, get_cardiac_params
    from multifil_jax_b200.engine import get_engine, upload, prng_split, prng_key, MF_FLAG_PLAIN, MF_FLAG_PRECISE
    rng = np.random.default_rng(1)
    eng = get_engine(0)
    dev = torch.device('cuda', 0)
    flags = MF_FLAG_PLAIN | (MF_FLAG_PRECISE if args.precision == 'mixed' else 0)
    total_t = 0.0
    for i in range(n):
        r, c = (int(v) for v in rng.integers(1, args.serve_max_lattice + 1, 2))
        sp = get_skeletal_params() if rng.random() < 0.5 else get_cardiac_params()
        rng.uniform(args.serve_min_ms, args.serve_max_ms)
        pca, z = float(rng.uniform(4, 7)), float(rng.uniform(850, 1000))
        topo = SarcTopology.create(r, c, *sp)
        key = prng_split(prng_key(1000 + i), 1)[0]
        a = upload(dev, sp[1].param_row()[None].astype(np.float32), np.full((1, steps), z, np.float32),
                   np.full((1, steps), pca, np.float32), np.full((1, steps), 14.0, np.float32),
                   np.array([steps], np.int32), key[None].view(np.int32), np.zeros(1, np.float32),
                   np.zeros(1, np.float32), np.ones(1, np.float32))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.run_batch(topo, *a[:6], K_lat=a[6], nu=a[7], dt=a[8], flags=flags)
        e1.record()
        torch.cuda.synchronize()
        total_t += e0.elapsed_time(e1) / 1e3
    return {'value': n * steps / total_t,
            'sample': f'the first {n} requests of the mix, {steps} steps each, one launch per step'}


def study_uneven(args):
    """Uneven batch in one launch: default CTA sizes vs the autotuner's."""
    import torch
    from multifil_jax_b200 import run_conditions
    from multifil_jax_b200.autotune import autotune_many, choose_batch_sizes
    conds, topos = uneven_conditions()
    total = sum(int(c['duration_ms']) for c in conds)
    out = {'study': 'uneven', 'metric': METRIC, 'conditions': len(conds), 'condition_timesteps': total,
           'precision': args.precision, 'lattices': sorted(f'{r}x{c}' for r, c in topos)}

    def timed():
        run_conditions(conds, precision=args.precision)  # warm-up: every kernel variant loaded
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run_conditions(conds, precision=args.precision)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    out['default_threads'] = ('library default with the spacing solved as an unknown: 512 threads up to '
                              '4000 nodes, else 1024')
    t_def = timed()
    tuned = autotune_many(list(topos.values()), precision=args.precision, dynamic_ls=True)
    # the per-lattice sizes checked on the batch itself (20 steps of it)
    short = [dict(c, duration_ms=min(float(c['duration_ms']), 20.0)) for c in conds]

    def run_short():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run_conditions(short, precision=args.precision)
        torch.cuda.synchronize()
        return time.perf_counter() - t0
    kept = choose_batch_sizes(list(topos.values()), tuned, run_short, precision=args.precision)
    t_tuned = timed()
    out['tuned_threads'] = {f'{r}x{c}': v for (r, c), v in sorted(tuned.items())}
    out['kept_threads'] = {f'{r}x{c}': v for (r, c), v in sorted(kept.items())}
    out['default_value'] = total / t_def
    out['tuned_value'] = total / t_tuned
    out['wall_s'] = {'default': t_def, 'tuned': t_tuned}
    out['note'] = 'wall time of run_conditions (host arrays in, host metrics out) for the whole batch'
    print(json.dumps(out), flush=True)


def sinusoid_conditions(n_freq=64, n_seeds=8):
    """Sinusoidal length perturbation on the 2x2 skeletal lattice at pCa 4.5:
    z(t) = 900 + 2 sin(2 pi f t) nm for f = logspace(0, 2.7, 64) Hz x 8 seeds
    (keys split(PRNGKey(seed), 1)[0]), dt = min(1, 1000 / (20 f)) ms, five full
    cycles and at least 200 ms."""
    from multifil_jax_b200.engine import prng_split, prng_key
    out = []
    for k in range(n_freq):
        f = 10.0 ** (2.7 * k / (n_freq - 1))
        dt = min(1.0, 1000.0 / (20.0 * f))
        n = int(max(5000.0 / f, 200.0) / dt)
        z = (900.0 + 2.0 * np.sin(2.0 * np.pi * f * np.arange(n) * dt / 1000.0)).astype(np.float32)
        for seed in range(n_seeds):
            out.append((f, dt, n, z, prng_split(prng_key(seed), 1)[0]))
    return out


def stiffness(force, z, f, dt):
    """Complex stiffness DFT(F)/DFT(z) at f over the whole cycles after one settling cycle."""
    period = 1000.0 / f / dt
    n0 = int(round(period))
    n1 = n0 + int(round(int((len(force) - n0) // period) * period))
    ph = np.exp(-2j * np.pi * f * np.arange(n0, n1) * dt / 1000.0)
    F = np.asarray(force[n0:n1], np.float64)
    Z = np.asarray(z[n0:n1], np.float64)
    return np.sum((F - F.mean()) * ph) / np.sum((Z - Z.mean()) * ph)


def study_sinusoid(args):
    """The precision-study workload (512 conditions of uneven length and dt)
    in one launch per precision mode: throughput, and how far the float32
    mode's complex stiffness sits from the mixed mode's per frequency.  The
    FP64-oracle comparison of this workload is tests/test_gpu_precision_study.py."""
    out, conds, forces = measure_sinusoid(args, modes=('mixed', 'float32'))
    out['study'] = 'sinusoid'
    out['metric'] = METRIC
    Y = {name: np.array([stiffness(f[i, :c[2]], c[3], c[0], c[1]) for i, c in enumerate(conds)])
         for name, f in forces.items()}
    rel = np.abs(Y['float32'] - Y['mixed']) / np.abs(Y['mixed'])
    fr = np.array([c[0] for c in conds])
    out['float32_vs_mixed_stiffness'] = {
        'median_rel': float(np.median(rel)), 'max_rel': float(rel.max()),
        'median_rel_by_decade': {f'{lo:g}-{hi:g} Hz': float(np.median(rel[(fr >= lo) & (fr < hi)]))
                                 for lo, hi in ((1, 10), (10, 100), (100, 600))}}
    out['mean_abs_stiffness_pN_per_nm'] = {f'{fr[i]:.1f} Hz': float(np.mean(np.abs(Y['mixed'][i:i + 8])))
                                           for i in (0, 8 * 31, 8 * 63)}
    print(json.dumps(out), flush=True)


def study_serving(args):
    """Serving at 50 / 80 / 95 % of the measured capacity of the request mix."""
    import torch
    res = []
    cap_args = argparse.Namespace(**vars(args))
    cap_args.serve_requests = args.study_capacity_requests
    cap_args.serve_rate = 1e9  # every request arrives at t = 0: the server's capacity
    cap = bench_serving(cap_args, 0)
    mean_steps = cap['condition_timesteps_per_s'] * cap['wall_s'] / max(cap['requests'], 1)
    cap_req = cap['requests'] / cap['wall_s']
    res.append(dict(cap, load='capacity'))
    for frac in (0.5, 0.8, 0.95):
        a = argparse.Namespace(**vars(args))
        a.serve_rate = frac * cap_req
        r = bench_serving(a, 0)
        res.append(dict(r, load=f'{int(frac * 100)}% of capacity'))
    print(json.dumps({'study': 'serving', 'capacity_requests_per_s': cap_req, 'mean_steps_per_request': mean_steps,
                      'runs': res}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--precision', default='mixed', choices=['float32', 'mixed'])
    ap.add_argument('--plain-conditions', type=int, default=256)
    ap.add_argument('--serve-requests', type=int, default=10000)
    ap.add_argument('--serve-rate', type=float, default=200.0)
    ap.add_argument('--serve-load', type=float, default=0.5,
                    help='arrival rate of the bench line\'s serving run, as a fraction of the measured capacity')
    ap.add_argument('--serve-capacity-requests', type=int, default=2000)
    ap.add_argument('--serve-max-lattice', type=int, default=6)
    ap.add_argument('--serve-min-ms', type=float, default=100.0)
    ap.add_argument('--serve-max-ms', type=float, default=2000.0)
    ap.add_argument('--serve-chunk', type=int, default=25)
    ap.add_argument('--serve-budget-gb', type=int, default=8)
    ap.add_argument('--traffic', type=float, default=None)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-workloads', action='store_true',
                    help='leave the uneven, sinusoid and serving workloads out of the bench line')
    ap.add_argument('--study', default=None, choices=['uneven', 'serving', 'sinusoid'],
                    help='run one workload study instead of the bench line')
    ap.add_argument('--study-capacity-requests', type=int, default=2000)
    ap.add_argument('--profile-case', default=None,
                    help='B,T[,lattice[,dyn]]: run the fused kernel once on B conditions x T steps (for ncu); '
                         'dyn=1 solves the lattice spacing (K_lat 5 per thick filament, nu 0.5)')
    args = ap.parse_args()
    if args.study == 'uneven':
        study_uneven(args)
    elif args.study == 'serving':
        study_serving(args)
    elif args.study == 'sinusoid':
        study_sinusoid(args)
    elif args.profile_case:
        profile_case(args)
    elif args.impl == 'reference':
        bench_reference(args)
    else:
        bench_gpu(args)


if __name__ == '__main__':
    main()
