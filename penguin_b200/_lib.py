"""ctypes loader of libpenguin_b200.so (the C ABI of include/penguin_b200.h).

There is no fallback: without the compiled CUDA library every entry point
raises.  Build it with ``python -m penguin_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

from .params import PGParams

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpenguin_b200.so")

PG_OK, PG_ERR_CONFIG, PG_ERR_CUDA, PG_ERR_NAN, PG_ERR_TIMEOUT, PG_ERR_ARG = range(6)
STATUS_NAMES = {0: "PG_OK", 1: "PG_ERR_CONFIG", 2: "PG_ERR_CUDA", 3: "PG_ERR_NAN", 4: "PG_ERR_TIMEOUT",
                5: "PG_ERR_ARG"}

# every symbol declared in include/penguin_b200.h
EXPORTS = [
    "pg_version", "pg_last_error", "pg_check_params", "pg_make_grid",
    "pg_configure", "pg_grid_init_orbadv", "pg_grid_global_dt", "pg_grid_solve", "pg_grid_release",
    "pg_global_dt_noalloc",
    "pg_disk_create", "pg_disk_destroy", "pg_disk_dims", "pg_disk_set_state", "pg_disk_get_state",
    "pg_disk_set_dust", "pg_disk_get_dust", "pg_disk_autotune", "pg_disk_set_tuning", "pg_sweep_variant",
    "pg_recon_weights",
    "pg_disk_write_snapshot", "pg_disk_read_snapshot", "pg_disk_set_average", "pg_disk_reset_average",
    "pg_disk_get_average",
    "pg_disk_state_ptr", "pg_disk_global_dt", "pg_disk_solve", "pg_disk_step_host", "pg_disk_run", "pg_disk_sync", "pg_disk_clock",
    "pg_disk_planet", "pg_disk_check", "pg_disk_torque", "pg_kernels_per_step", "pg_disk_profile",
    "pg_ens_check_params", "pg_ens_create", "pg_ens_destroy", "pg_ens_size", "pg_ens_dims", "pg_ens_set_state",
    "pg_ens_get_state", "pg_ens_run", "pg_ens_sync", "pg_ens_clock", "pg_ens_planet", "pg_ens_check",
    "pg_ens_totals", "pg_ens_torque", "pg_ens_kernels_per_step", "pg_ens_profile", "pg_ens_set_dust",
    "pg_ens_get_dust", "pg_ens_autotune", "pg_ens_set_tuning",
    "pg_adj_check_params", "pg_adj_create", "pg_adj_destroy", "pg_adj_set_params", "pg_adj_forward",
    "pg_adj_backward", "pg_adj_model_error", "pg_adj_dot_test", "pg_adj_pass_check", "pg_adj_replay_diff", "pg_adj_pass_fields", "pg_adj_schedule", "pg_adj_steps", "pg_adj_device_bytes", "pg_adj_set_sweep_reverse",
    "pg_disk3_create", "pg_disk3_destroy", "pg_disk3_set_state", "pg_disk3_get_state", "pg_disk3_global_dt",
    "pg_disk3_solve", "pg_disk3_run", "pg_disk3_clock", "pg_disk3_check", "pg_disk3_pass_times", "pg_disk3_stages", "pg_disk3_write_snapshot", "pg_disk3_read_snapshot", "pg_make_axis",
    "pg_test_div_1p5", "pg_test_bounded_wait",
]


class PGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class PGBody(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("m", "a", "e", "x", "y", "z", "vx", "vy", "vz", "rs")]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m penguin_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_int
    d = ctypes.c_double
    PP = ctypes.POINTER(PGParams)
    sig = {
        "pg_version": (ctypes.c_char_p, []),
        "pg_last_error": (ctypes.c_char_p, []),
        "pg_check_params": (i, [PP]),
        "pg_make_grid": (i, [PP, dp, dp, dp, dp]),
        "pg_configure": (i, [PP]),
        "pg_grid_init_orbadv": (i, [vp]),
        "pg_grid_global_dt": (i, [vp, vp, d, dp]),
        "pg_grid_solve": (i, [vp, d, d]),
        "pg_grid_release": (i, []),
        "pg_global_dt_noalloc": (i, [PP, vp, vp, vp, vp, vp, d, dp, vp]),
        "pg_disk_create": (i, [PP, i, vp, ctypes.POINTER(vp)]),
        "pg_disk_destroy": (i, [vp]),
        "pg_disk_dims": (i, [vp, ip, ip, ip]),
        "pg_disk_set_state": (i, [vp, d, dp, dp, dp, dp]),
        "pg_disk_get_state": (i, [vp, dp, dp, dp, dp, dp]),
        "pg_disk_set_dust": (i, [vp, dp, dp, dp]),
        "pg_disk_autotune": (i, [vp, i, ip]),
        "pg_disk_set_tuning": (i, [vp, ip]),
        "pg_sweep_variant": (i, [i, ip]),
        "pg_recon_weights": (i, [PP, i, dp]),
        "pg_disk_write_snapshot": (i, [vp, ctypes.c_char_p, i]),
        "pg_disk_read_snapshot": (i, [vp, ctypes.c_char_p, dp]),
        "pg_disk_set_average": (i, [vp, d]),
        "pg_disk_reset_average": (i, [vp]),
        "pg_disk_get_average": (i, [vp, dp, dp, dp, dp]),
        "pg_disk_get_dust": (i, [vp, dp, dp, dp]),
        "pg_disk_state_ptr": (i, [vp, ctypes.POINTER(vp)]),
        "pg_disk_global_dt": (i, [vp, d, dp]),
        "pg_disk_solve": (i, [vp, d, d]),
        "pg_disk_step_host": (i, [vp, i, d, dp, dp, ip]),
        "pg_disk_run": (i, [vp, i, d]),
        "pg_disk_sync": (i, [vp]),
        "pg_disk_clock": (i, [vp, dp, dp, ctypes.POINTER(ctypes.c_longlong)]),
        "pg_disk_planet": (i, [vp, ctypes.POINTER(PGBody)]),
        "pg_disk_check": (i, [vp]),
        "pg_disk_torque": (i, [vp, dp]),
        "pg_kernels_per_step": (i, [vp]),
        "pg_disk_profile": (i, [vp, i, d, ctypes.POINTER(ctypes.c_float), i]),
        "pg_ens_check_params": (i, [PP, i]),
        "pg_ens_create": (i, [PP, i, i, vp, ctypes.POINTER(vp)]),
        "pg_ens_destroy": (i, [vp]),
        "pg_ens_size": (i, [vp]),
        "pg_ens_dims": (i, [vp, i, ip, ip]),
        "pg_ens_set_state": (i, [vp, i, d, dp, dp, dp]),
        "pg_ens_get_state": (i, [vp, i, dp, dp, dp, dp, dp]),
        "pg_ens_run": (i, [vp, i, d]),
        "pg_ens_sync": (i, [vp]),
        "pg_ens_clock": (i, [vp, i, dp, dp, ctypes.POINTER(ctypes.c_longlong)]),
        "pg_ens_planet": (i, [vp, i, ctypes.POINTER(PGBody)]),
        "pg_ens_check": (i, [vp]),
        "pg_ens_totals": (i, [vp, i, dp, dp]),
        "pg_ens_torque": (i, [vp, i, dp]),
        "pg_ens_set_dust": (i, [vp, i, dp, dp, dp]),
        "pg_ens_get_dust": (i, [vp, i, dp, dp, dp]),
        "pg_adj_check_params": (i, [PP]),
        "pg_adj_create": (i, [PP, i, vp, i, ctypes.POINTER(vp)]),
        "pg_adj_destroy": (i, [vp]),
        "pg_adj_set_params": (i, [vp, d, d, d]),
        "pg_adj_forward": (i, [vp, vp, d, i, i, vp]),
        "pg_adj_backward": (i, [vp, vp, vp, dp]),
        "pg_adj_model_error": (i, [vp, d, dp]),
        "pg_adj_dot_test": (i, [vp, d, vp, vp, dp]),
        "pg_adj_pass_check": (i, [vp, d, d, vp, dp]),
        "pg_adj_replay_diff": (i, [vp, d, dp]),
        "pg_adj_pass_fields": (i, [vp, i, d, d, vp, vp, vp]),
        "pg_adj_schedule": (i, [vp, dp, i]),
        "pg_adj_steps": (i, [vp]),
        "pg_adj_device_bytes": (ctypes.c_longlong, [vp]),
        "pg_adj_set_sweep_reverse": (i, [vp, i]),
        "pg_ens_kernels_per_step": (i, [vp]),
        "pg_ens_profile": (i, [vp, i, d, ctypes.POINTER(ctypes.c_float), i]),
        "pg_ens_autotune": (i, [vp, i, ip]),
        "pg_ens_set_tuning": (i, [vp, ip]),
        "pg_disk3_create": (i, [PP, i, vp, ctypes.POINTER(vp)]),
        "pg_disk3_destroy": (i, [vp]),
        "pg_disk3_set_state": (i, [vp, d, dp, dp, dp, dp, dp]),
        "pg_disk3_get_state": (i, [vp, dp, dp, dp, dp, dp, dp]),
        "pg_disk3_global_dt": (i, [vp, d, dp]),
        "pg_disk3_solve": (i, [vp, d, d]),
        "pg_disk3_run": (i, [vp, i, d]),
        "pg_disk3_clock": (i, [vp, dp, dp, ctypes.POINTER(ctypes.c_longlong)]),
        "pg_disk3_check": (i, [vp]),
        "pg_disk3_pass_times": (i, [vp, i, dp]),
        "pg_disk3_stages": (i, [vp, d, d, dp]),
        "pg_disk3_write_snapshot": (i, [vp, ctypes.c_char_p]),
        "pg_test_div_1p5": (i, [dp, ctypes.c_longlong, dp]),
        "pg_test_bounded_wait": (i, [ip, ip, ctypes.POINTER(ctypes.c_float)]),
        "pg_disk3_read_snapshot": (i, [vp, ctypes.c_char_p, dp]),
        "pg_make_axis": (i, [PP, i, dp, dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != PG_OK:
        raise PGError(status, lib().pg_last_error().decode())
