"""ctypes binding of ``libsolar_gpu.so`` (the C-ABI of ``include/solar_gpu.h``).

There is no CPU fallback: if the library is missing or cannot be loaded, every entry
point raises.  The library is built in-tree by ``solar_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)

SOLAR_OK = 0
SOLAR_ERR_ARG = -1
SOLAR_ERR_CUDA = -2
SOLAR_ERR_NAN = -3
SOLAR_ERR_TIMEOUT = -4
SOLAR_ERR_STATE = -5
SOLAR_ERR_NOMEM = -6
SOLAR_FORCING_OFF = 0
SOLAR_FORCING_ANALYTIC = 1
SOLAR_FORCING_SAMPLES = 2
SOLAR_FP64 = 0
SOLAR_FP32 = 1
SOLAR_KERNEL_EDGE = 1
SOLAR_KERNEL_STAGE = 2
SOLAR_KERNEL_FILTER = 4
SOLAR_KERNEL_ADJ_STAGE = 8


class SolarError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"solar_gpu status {status}: {msg}")
        self.status = status


class SolarDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("nr", ctypes.c_int), ("precision", ctypes.c_int),
        ("nfields", ctypes.c_int), ("nruns", ctypes.c_int), ("device", ctypes.c_int),
        ("dt", ctypes.c_double), ("model", _D), ("c2_3d", _D),
        ("sponge_amp", ctypes.c_double), ("sponge_exp", ctypes.c_double),
        ("sponge_len", ctypes.c_int), ("sponge_lower", ctypes.c_int), ("sponge_upper", ctypes.c_int),
        ("fix_reversed_rotation", ctypes.c_int),
        ("tile_x", ctypes.c_int), ("tile_y", ctypes.c_int), ("kchunk", ctypes.c_int),
    ]


# (name, argtypes) of every exported entry point declared in include/solar_gpu.h
_P = ctypes.c_void_p
EXPORTS = {
    "solar_desc_defaults": [ctypes.POINTER(SolarDesc)],
    "solar_gpu_init": [ctypes.POINTER(SolarDesc), ctypes.POINTER(ctypes.c_void_p)],
    "solar_gpu_finalize": [_P],
    "solar_gpu_set_state": [_P, ctypes.c_int, _D],
    "solar_gpu_get_state": [_P, ctypes.c_int, _D],
    "solar_gpu_add_gaussian": [_P, ctypes.c_int] + [ctypes.c_double] * 5,
    "solar_gpu_rk4": [_P, ctypes.c_int],
    "solar_gpu_rk4_runs": [_P, _I],
    "solar_gpu_time_rk4_runs": [_P, _I, _D],
    "solar_gpu_compute_rhs": [_P, _D, _D],
    "solar_gpu_bc_rhs": [_P, _D],
    "solar_gpu_sponge": [_P, _D, _D],
    "solar_gpu_filter_exp": [_P, _D, _D],
    "solar_gpu_gradient": [_P, _D, _D, _D, _D],
    "solar_gpu_divergence": [_P, _D, _D, _D, _D],
    "solar_gpu_curl": [_P, _D, _D, _D, _D, _D, _D],
    "solar_gpu_norm": [_P, ctypes.c_int, ctypes.c_int, _D],
    "solar_gpu_norm_noalloc": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "solar_gpu_rk4_norms": [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D],
    "solar_gpu_set_watchdog": [_P, ctypes.c_int],
    "solar_gpu_inject_wait_timeout": [_P, ctypes.c_int, ctypes.c_int],
    "solar_gpu_diag": [_P, ctypes.c_int, _D],
    "solar_gpu_time_rk4": [_P, ctypes.c_int, ctypes.c_int, _D],
    "solar_gpu_synchronize": [_P],
    "solar_gpu_last_error": [ctypes.c_char_p, ctypes.c_int],
    "solar_gpu_abi_version": [],
    "solar_gpu_device_name": [ctypes.c_int, ctypes.c_char_p, ctypes.c_int],
    "solar_gpu_set_receivers": [_P, ctypes.c_int, _D],
    "solar_gpu_record": [_P, ctypes.c_int, _D],
    "solar_gpu_misfit_gradient": [_P, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D],
    "solar_gpu_misfit_gradient_nested": [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D],
    "solar_gpu_rhs_adjoint": [_P, _D, _D],
    "solar_gpu_filter_adjoint": [_P, _D, _D],
    "solar_gpu_rk4_adjoint": [_P, ctypes.c_int, _D, _D],
    "solar_gpu_set_owned_zones": [_P, ctypes.c_int, ctypes.c_int],
    "solar_gpu_edge_routes": [_I],
    "solar_gpu_step_phase": [_P, ctypes.c_int],
    "solar_gpu_step_phase_part": [_P, ctypes.c_int, ctypes.c_int],
    "solar_gpu_set_owned_planes": [_P, ctypes.c_int, ctypes.c_int],
    "solar_gpu_planes_size": [_P, ctypes.c_int],
    "solar_gpu_pack_planes": [_P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
    "solar_gpu_unpack_planes": [_P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
    "solar_gpu_lines_size": [_P, ctypes.c_int],
    "solar_gpu_pack_lines": [_P, ctypes.c_int, _I, ctypes.c_int, ctypes.c_void_p],
    "solar_gpu_unpack_lines": [_P, ctypes.c_int, _I, ctypes.c_int, ctypes.c_void_p],
    "solar_gpu_stream": [_P],
    "solar_gpu_reduce_owned": [_P, ctypes.c_int, ctypes.c_int, _D],
    "solar_gpu_set_forcing": [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "solar_gpu_set_forcing_samples": [_P, ctypes.c_int, _D, ctypes.c_int],
    "solar_gpu_load_forcing": [_P, ctypes.c_char_p, ctypes.c_int],
    "solar_io_read_forcing": [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D],
    "solar_gpu_set_clock": [_P, ctypes.c_double, ctypes.c_int],
    "solar_gpu_get_clock": [_P, _D, _I],
    "solar_gpu_write_restart": [_P, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_int],
    "solar_gpu_read_restart": [_P, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, _D, _I],
    "solar_gpu_write_visual": [_P, ctypes.c_int, ctypes.c_char_p, ctypes.c_int],
    "solar_gpu_write_grid": [_P, ctypes.c_char_p],
    "solar_gpu_write_radial_trace": [_P, ctypes.c_int, ctypes.c_char_p],
    "solar_gpu_output_plane": [_P, _I],
    "solar_io_cue_name": [ctypes.c_int, ctypes.c_char_p, ctypes.c_int],
    "solar_io_format_es": [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_char_p],
    "solar_io_write_restart": [ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int],
    "solar_io_read_restart": [ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _I],
    "solar_io_write_visual": [ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_int],
    "solar_io_write_grid": [ctypes.c_char_p, _I],
    "solar_io_append_trace": [ctypes.c_char_p, _D, ctypes.c_int],
}

# entry points whose return type is not int
RESTYPES = {"solar_desc_defaults": None, "solar_gpu_lines_size": ctypes.c_longlong,
            "solar_gpu_planes_size": ctypes.c_longlong,
            "solar_gpu_stream": ctypes.c_void_p}

_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = False):
    """Load the CUDA library (raises OSError if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        if build_if_missing:
            _build.build()
        else:
            raise OSError(f"CUDA library {path} is not built; run python -m solar_b200.build")
    lib = ctypes.CDLL(path)
    for name, args in EXPORTS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def device_name(device: int = 0) -> str:
    buf = ctypes.create_string_buffer(256)
    if load().solar_gpu_device_name(device, buf, 256) != SOLAR_OK:
        return "unknown"
    return buf.value.decode(errors="replace")


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    load().solar_gpu_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != SOLAR_OK:
        raise SolarError(status, last_error())
