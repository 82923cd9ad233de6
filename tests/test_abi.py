"""The C-ABI library loads and exports every entry point declared in include/solar_gpu.h,
and rejects bad descriptors before touching a device (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from solar_b200 import _lib, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "solar_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(solar_(?:gpu|desc)_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    return _lib.load(build_if_missing=True)


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.EXPORTS, name


def test_abi_version(lib):
    assert lib.solar_gpu_abi_version() == 1


def _desc(cfg, **kw):
    d = _lib.SolarDesc()
    _lib.load().solar_desc_defaults(ctypes.byref(d))
    model = np.ascontiguousarray(cfg.model)
    d.nx, d.nr, d.dt = cfg.nx, cfg.nr, cfg.dt
    d.model = model.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for k, v in kw.items():
        setattr(d, k, v)
    return d, model


def test_defaults_match_reference(lib):
    d = _lib.SolarDesc()
    lib.solar_desc_defaults(ctypes.byref(d))
    assert (d.sponge_amp, d.sponge_exp, d.sponge_len) == (0.1, 3.0, 30)   # sponge.f90:20-27
    assert d.sponge_lower == 1 and d.sponge_upper == 1
    assert d.nfields == 5 and d.nruns == 1 and d.precision == _lib.SOLAR_FP64


@pytest.mark.parametrize("field,value", [("nx", 24), ("nx", 8), ("nr", 10), ("nfields", 3),
                                         ("precision", 7), ("nruns", 0), ("dt", -1.0)])
def test_init_rejects_bad_descriptors(lib, field, value):
    d, keep = _desc(configs.c1(nx=16, nr=16), **{field: value})
    h = ctypes.c_void_p()
    rc = lib.solar_gpu_init(ctypes.byref(d), ctypes.byref(h))
    assert rc == -1, _lib.last_error()
    assert not h.value
    assert len(_lib.last_error()) > 0


def test_init_rejects_dropping_rho_with_gravity(lib):
    cfg = configs.c1(nx=16, nr=16)
    cfg.model[:, 5] = 1e-9   # g != 0 makes rho feed v_r (compute_rhs_acoustic.f90:83)
    d, keep = _desc(cfg, nfields=4)
    h = ctypes.c_void_p()
    assert lib.solar_gpu_init(ctypes.byref(d), ctypes.byref(h)) == -1
    assert "g0" in _lib.last_error()


def test_null_context_is_an_error_not_a_crash(lib):
    q = np.zeros(10)
    assert lib.solar_gpu_rk4(None, 1) == -5
    assert lib.solar_gpu_get_state(None, 0, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == -5
    assert lib.solar_gpu_finalize(None) == 0


def test_new_entry_points_reject_a_null_context(lib):
    out = np.zeros(4)
    p = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.solar_gpu_rk4_norms(None, 0, 4, 2, p) == -5
    assert lib.solar_gpu_set_watchdog(None, 1) == -5
    assert lib.solar_gpu_inject_wait_timeout(None, 1, 100) == -5
    assert lib.solar_gpu_step_phase_part(None, 0, 0) == -5


def test_norm_noalloc_rejects_planes_beyond_int_range_before_any_launch(lib):
    # nx * nx > INT_MAX would overflow the kernel's plane size: refused on the host, before
    # the device is touched (the pointers are never dereferenced).
    fake = ctypes.c_void_p(4096)
    assert lib.solar_gpu_norm_noalloc(fake, 46341, 4, fake, None) == -1
    assert "INT_MAX" in _lib.last_error()
    assert lib.solar_gpu_norm_noalloc(fake, 16, 4096, fake, None) == -1
    assert "exceeds" in _lib.last_error()
    assert lib.solar_gpu_norm_noalloc(None, 16, 16, fake, None) == -1
