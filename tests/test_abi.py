"""The C ABI library loads on a CPU-only host and exports every declared symbol."""
import os
import re
import subprocess
import ctypes

import numpy as np
import pytest

from multifil_jax_b200 import engine

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, 'include', 'multifil_b200.h')


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(mf_[a-z0-9_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    lib = engine.load_library()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert lib.mf_abi_version() == 2


def test_ctypes_struct_layout_matches_c():
    # compile a tiny C program against the header and compare sizeof/offsetof
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "multifil_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(mf_topo_desc), sizeof(mf_batch), sizeof(mf_request),
         offsetof(mf_batch, metrics_out), offsetof(mf_batch, bound_trace), offsetof(mf_request, pCa),
         offsetof(mf_batch, n_pops), offsetof(mf_batch, tm_label));
  printf("%zu %zu %zu %zu\n", sizeof(mf_state_batch), offsetof(mf_state_batch, thick_axial),
         offsetof(mf_state_batch, status_out), offsetof(mf_state_batch, u_xb));
  return 0;
}'''
    tmp = os.path.join(REPO, '_build')
    os.makedirs(tmp, exist_ok=True)
    c = os.path.join(tmp, 'abi_layout.c')
    exe = os.path.join(tmp, 'abi_layout')
    open(c, 'w').write(src)
    subprocess.run(['gcc', '-I', os.path.join(REPO, 'include'), c, '-o', exe], check=True)
    out = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    from multifil_jax_b200.timestep import mf_state_batch
    sb = [ctypes.sizeof(mf_state_batch), mf_state_batch.thick_axial.offset, mf_state_batch.status_out.offset,
          mf_state_batch.u_xb.offset]
    assert out[-4:] == sb
    out = out[:-4]
    py = [ctypes.sizeof(engine.mf_topo_desc), ctypes.sizeof(engine.mf_batch), ctypes.sizeof(engine.mf_request),
          engine.mf_batch.metrics_out.offset, engine.mf_batch.bound_trace.offset, engine.mf_request.pCa.offset,
          engine.mf_batch.n_pops.offset, engine.mf_batch.tm_label.offset]
    assert out == py


def test_no_cuda_raises_cleanly(monkeypatch):
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    with pytest.raises(engine.EngineError):
        engine.get_engine(0)


def test_invalid_arguments_are_rejected_without_a_device():
    lib = engine.load_library()
    assert lib.mf_prng_split(0, 0, -1, 1, None) < 0
    assert lib.mf_create(0, None) < 0
    assert lib.mf_destroy(None) < 0
    from multifil_jax_b200.timestep import _bind
    assert _bind(lib)(None, None, None) < 0
