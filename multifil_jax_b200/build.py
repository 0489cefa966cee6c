"""Compile the CUDA engine in-tree for sm_100a: ``python -m multifil_jax_b200.build``.

The twenty instances of the step kernel (CTA size x precision mode x
dynamic spacing) are separate translation units of ``csrc/mf_kernels.cu`` and
compile in parallel with the host/ABI unit ``csrc/mf_api.cu``; the objects are
linked into ``libmultifil_b200.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, 'libmultifil_b200.so')
DEPS = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
    os.path.join(os.path.dirname(HERE), 'include', 'multifil_b200.h')]
INSTANCES = [(nt, p, d) for nt in (128, 256, 384, 512, 1024) for p in (0, 1) for d in (0, 1)]

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC']


def nvcc() -> str:
    for cand in (shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def up_to_date(out: str = OUT) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}): {' '.join(cmd)}\n{r.stderr[-4000:]}")
    return r.stderr


def build(force: bool = False, verbose: bool = False, out: str = OUT, extra_flags=()) -> str:
    """Build the library (``extra_flags``: more nvcc flags, e.g. a -D for a
    diagnostic build written to another ``out``)."""
    if not force and up_to_date(out):
        return out
    flags = NVCC_FLAGS + list(extra_flags) + (['-Xptxas=-v'] if verbose else [])
    with tempfile.TemporaryDirectory(prefix='mf_build_') as tmp:
        jobs = [[nvcc(), *flags, '-c', os.path.join(CSRC, 'mf_api.cu'), '-o', os.path.join(tmp, 'mf_api.o')]]
        for nt, p, d in INSTANCES:
            jobs.append([nvcc(), *flags, f'-DMF_NT={nt}', f'-DMF_P={p}', f'-DMF_D={d}', '-c',
                         os.path.join(CSRC, 'mf_kernels.cu'), '-o', os.path.join(tmp, f'mf_k_{nt}_{p}_{d}.o')])
        with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            logs = list(ex.map(_run, jobs))
        objs = [j[-1] for j in jobs]
        _run([nvcc(), *ARCH, '-shared', *objs, '-o', out + '.tmp'])
    os.replace(out + '.tmp', out)
    if verbose:
        print('\n'.join(logs))
    return out


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
