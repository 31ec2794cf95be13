"""ctypes binding of librmhd2d.so (include/rmhd2d.h).

The library is loaded from this package directory only; there is no
fallback.  If it is missing, ``load()`` raises with the command that builds it.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "librmhd2d.so"
HEADER = PKG.parent / "include" / "rmhd2d.h"

OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "no sm_100 device", 4: "invalid solver state",
          5: "I/O error", 6: "kernel error"}

BC = {"periodic": 0, "symmetric": 1, "zero_gradient": 2, "wall": 3, "flare": 4}
CT = {"stage1": 0, "contact": 1}
PRECISION = {"fp64_exact": 0, "exact": 0, "fp64_fast": 1, "fast": 1, "fp32_bulk": 2, "bulk32": 2}


class Config(ctypes.Structure):
    """Mirror of rmhd2d_config."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("gamma_mhd", ctypes.c_double), ("cfl", ctypes.c_double), ("eps", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("bc", ctypes.c_int), ("bc_y", ctypes.c_int), ("precision", ctypes.c_int), ("device", ctypes.c_int),
        ("stream", ctypes.c_void_p), ("ct_scheme", ctypes.c_int),
    ]


# (name, restype, argtypes) of every exported function.
_D = ctypes.POINTER(ctypes.c_double)
_S = ctypes.c_void_p
SIGNATURES = [
    ("rmhd2d_config_default", None, [ctypes.POINTER(Config)]),
    ("rmhd2d_create", ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    ("rmhd2d_destroy", ctypes.c_int, [_S]),
    ("rmhd2d_set_state", ctypes.c_int, [_S, _D, ctypes.c_int]),
    ("rmhd2d_set_state_device", ctypes.c_int, [_S, ctypes.c_void_p, ctypes.c_int]),
    ("rmhd2d_get_state", ctypes.c_int, [_S, _D]),
    ("rmhd2d_set_eta_table", ctypes.c_int, [_S, _D]),
    ("rmhd2d_apply_boundary", ctypes.c_int, [_S]),
    ("rmhd2d_calculate_dt", ctypes.c_int, [_S, _D]),
    ("rmhd2d_step_rk2", ctypes.c_int, [_S]),
    ("rmhd2d_run", ctypes.c_int, [_S, ctypes.c_int]),
    ("rmhd2d_run_timed", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("rmhd2d_profile_step", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_float)]),
    ("rmhd2d_get_dt", ctypes.c_int, [_S, _D]),
    ("rmhd2d_get_total_time", ctypes.c_int, [_S, _D]),
    ("rmhd2d_check_crashed", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_save", ctypes.c_int, [_S, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
    ("rmhd2d_load", ctypes.c_int, [_S, ctypes.c_char_p]),
    ("rmhd2d_write_snapshot", ctypes.c_int, [ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_int]),
    ("rmhd2d_set_tile_shape", ctypes.c_int, [_S, ctypes.c_int]),
    ("rmhd2d_get_tile_shape", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_autotune", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_get_tuning", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    ("rmhd2d_set_stage_shapes", ctypes.c_int, [_S, ctypes.c_int, ctypes.c_int]),
    ("rmhd2d_get_stage_shapes", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_batch_create", ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("rmhd2d_batch_destroy", ctypes.c_int, [_S]),
    ("rmhd2d_batch_size", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_batch_member", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("rmhd2d_batch_run", ctypes.c_int, [_S, ctypes.c_int]),
    ("rmhd2d_batch_run_timed", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("rmhd2d_batch_set_launch", ctypes.c_int, [_S, ctypes.c_int, ctypes.c_int]),
    ("rmhd2d_batch_get_launch", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_batch_autotune", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
    ("rmhd2d_batch_get_tuning", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_float)]),
    ("rmhd2d_batch_last_error", ctypes.c_char_p, [_S]),
    ("rmhd2d_run_fixed_dt", ctypes.c_int, [_S, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    ("rmhd2d_adjoint_forward", ctypes.c_int, [_S, ctypes.c_int, ctypes.c_int]),
    ("rmhd2d_adjoint_dts", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_double)]),
    ("rmhd2d_adjoint_backward", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_double)]),
    ("rmhd2d_adjoint_release", ctypes.c_int, [_S]),
    ("rmhd2d_calculate_dt_noalloc", ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_void_p,
                                                    ctypes.POINTER(ctypes.c_double)]),
    ("rmhd2d_create_slab", ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("rmhd2d_slab_halo_doubles", ctypes.c_int, [_S, ctypes.POINTER(ctypes.c_longlong)]),
    ("rmhd2d_slab_pack", ctypes.c_int, [_S, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    ("rmhd2d_slab_unpack", ctypes.c_int, [_S, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    ("rmhd2d_slab_stage", ctypes.c_int, [_S, ctypes.c_int]),
    ("rmhd2d_slab_fill", ctypes.c_int, [_S, ctypes.c_int]),
    ("rmhd2d_slab_refresh_rate", ctypes.c_int, [_S]),
    ("rmhd2d_slab_get_words", ctypes.c_int, [_S, ctypes.c_void_p]),
    ("rmhd2d_slab_set_words", ctypes.c_int, [_S, ctypes.c_void_p]),
    ("rmhd2d_last_error", ctypes.c_char_p, [_S]),
    ("rmhd2d_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("rmhd2d_abi_version", ctypes.c_int, []),
]

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load librmhd2d.so from the package directory (no fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m resistivemhd_gpu_b200.build` "
                               "(the CUDA path has no CPU fallback)")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


class RMHDError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def check(status: int, handle=None) -> None:
    if status != OK:
        msg = load().rmhd2d_last_error(handle)
        raise RMHDError(status, msg.decode() if msg else "")


def check_batch(status: int, handle=None) -> None:
    if status != OK:
        msg = load().rmhd2d_batch_last_error(handle)
        raise RMHDError(status, msg.decode() if msg else "")
