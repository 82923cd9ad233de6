"""solar_gpu_norm_noalloc: the reference's per-step norm for callers that cannot allocate.

Hosts whose device memory belongs to another runtime's budget, and per-step diagnostic
hooks that must not cause the device-wide synchronisation of cudaMalloc / cudaFree, call
this entry point with device pointers they already own; its only scratch is a fixed array
inside the library.  The test checks it against the context-based solar_gpu_norm (same
FP64 formula, auxiliary.f90:100-125) on two calls in a row -- the second call on a
different field, so stale scratch from the first call would show -- and that grids larger
than the fixed scratch are rejected before any launch.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from solar_b200 import _lib, configs
from solar_b200.solver import Solver

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12   # the FP64 reduction tolerance used by the other norm tests


def _smooth_state(shape, seed):
    rng = np.random.default_rng(seed)
    q = rng.standard_normal(shape)
    return q


def test_norm_noalloc_matches_context_norm_twice():
    import torch

    cfg = configs.c1(nx=32, nr=32)
    q = _smooth_state((6, 5, cfg.nr, cfg.nx, cfg.nx), 11)
    with Solver(cfg) as s:
        s.set_state(q)
        want = {4: s.norm(4), 5: s.norm(5)}        # v_r, then p
    lib = _lib.load()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for field in (4, 5):                           # two calls in a row, different inputs
        d_field = torch.from_numpy(np.ascontiguousarray(q[:, field - 1])).to("cuda")
        out.fill_(-1.0)
        rc = lib.solar_gpu_norm_noalloc(ctypes.c_void_p(d_field.data_ptr()), cfg.nx, cfg.nr,
                                        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, _lib.last_error()
        stream.synchronize()
        got = out.item()
        assert abs(got - want[field]) <= REL_TOL * want[field], (field, got, want[field])


def test_norm_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _lib.load().solar_gpu_norm_noalloc(ctypes.c_void_p(small.data_ptr()), 16, 4096,
                                            ctypes.c_void_p(out.data_ptr()), None)
    assert rc == -1
    assert "exceeds" in _lib.last_error()
