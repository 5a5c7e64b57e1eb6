"""Loader of the engine's C ABI (include/dsmc.h) from lib/libdsmc_b200.so.

The library is built in-tree by dsmc_erlend_b200.build.  Loading fails loudly
when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .abi import Counters, Derived, Drag, Params

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libdsmc_b200.so"

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_U32 = C.POINTER(C.c_uint32)
_P = C.POINTER(Params)
_DV = C.POINTER(Derived)

# name -> (restype, argtypes); every symbol declared in include/dsmc.h.
SIGNATURES = {
    "dsmc_default_params": (None, [_P]),
    "dsmc_setup": (C.c_int, [_P, _DV]),
    "dsmc_wall_model_name": (C.c_char_p, [C.c_int]),
    "dsmc_status_string": (C.c_char_p, [C.c_int]),
    "dsmc_write_field": (C.c_int, [_P, _DV, C.c_int64, C.c_void_p, C.c_char_p]),
    "dsmc_ctx_create": (C.c_int, [_P, _DV, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dsmc_ctx_destroy": (C.c_int, [C.c_void_p]),
    "dsmc_init_cold": (C.c_int, [C.c_void_p]),
    "dsmc_init_warm": (C.c_int, [C.c_void_p, _D]),
    "dsmc_init_warm_tensor": (C.c_int, [C.c_void_p, _D]),
    "dsmc_init_warm_mixture": (C.c_int, [C.c_void_p, _D]),
    "dsmc_step": (C.c_int, [C.c_void_p, C.c_int]),
    "dsmc_step_read": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dsmc_stage_move": (C.c_int, [C.c_void_p]),
    "dsmc_stage_boundary": (C.c_int, [C.c_void_p]),
    "dsmc_stage_index": (C.c_int, [C.c_void_p]),
    "dsmc_stage_collide": (C.c_int, [C.c_void_p]),
    "dsmc_stage_sample": (C.c_int, [C.c_void_p]),
    "dsmc_stage_end_step": (C.c_int, [C.c_void_p]),
    "dsmc_synchronize": (C.c_int, [C.c_void_p]),
    "dsmc_get_counters": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Counters)]),
    "dsmc_get_fields": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dsmc_get_fields_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dsmc_get_fields_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dsmc_set_fields_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]),
    "dsmc_download_particles": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, C.c_int64,
                                          _I64]),
    "dsmc_upload_particles": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, C.c_int64]),
    "dsmc_get_cell_starts": (C.c_int, [C.c_void_p, C.c_int, _I32]),
    "dsmc_checkpoint_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "dsmc_checkpoint_load": (C.c_int, [C.c_void_p, C.c_char_p]),
    "dsmc_drag_report": (C.c_int, [_P, _DV, C.POINTER(Counters), C.POINTER(Drag)]),
    "dsmc_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "dsmc_get_launch_config": (C.c_int, [C.c_void_p, _I32, _I32, C.c_int, C.POINTER(C.c_int),
                                         C.POINTER(C.c_char_p)]),
    "dsmc_set_launch_config": (C.c_int, [C.c_void_p, _I32, C.c_int]),
    "dsmc_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "dsmc_set_step_mode": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dsmc_get_step_mode": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "dsmc_grid_sync_probe": (C.c_int, [C.c_void_p, C.c_int64]),
    "dsmc_get_phase_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int,
                                       C.POINTER(C.c_int), C.POINTER(C.c_char_p), C.c_int]),
    "dsmc_get_kernel_times": (C.c_int, [C.c_void_p, _D, _I64, C.c_int, C.POINTER(C.c_int),
                                        C.POINTER(C.c_char_p)]),
    "dsmc_k_intersect": (C.c_int, [_P, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "dsmc_k_inside_box": (C.c_int, [_P, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
    "dsmc_k_scatter": (C.c_int, [_P, _DV, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    "dsmc_k_inject": (C.c_int, [_P, _DV, _D, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int64,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                _I64, C.c_void_p]),
    "dsmc_k_collide": (C.c_int, [_P, _DV, C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                 C.c_void_p, C.c_void_p, C.c_void_p]),
    "dsmc_k_elastic": (C.c_int, [_P, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                 C.c_uint32, C.c_void_p, C.c_void_p]),
    "dsmc_append_particles_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "dsmc_remove_inside_box": (C.c_int, [C.c_void_p, C.c_int]),
    "dsmc_collide_list": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int32, _I32, C.c_uint32,
                                    C.c_uint32, C.c_uint32, _I32]),
}

_lib = None


class DsmcError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = load().dsmc_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: status {status} ({msg})" if what else
                         f"status {status} ({msg})")


def load(path: str | os.PathLike | None = None):
    """Loads the engine library (once) and declares every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `python -m dsmc_erlend_b200.build` "
            "(the engine has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = ""):
    if status != 0:
        raise DsmcError(status, what)
