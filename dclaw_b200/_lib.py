"""ctypes binding of the CUDA library (dclaw_b200/lib/libdclaw_b200.so).

The library is the only compute path: importing this module on a machine
where the shared object is missing raises, and so does calling any entry
point without a CUDA device. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

from .params import CAdjBatch, CAdjMember, CBatch, CClock, CMember, CParams

LIB_DIR = Path(__file__).resolve().parent / "lib"
LIB_PATH = LIB_DIR / "libdclaw_b200.so"

_vp = ctypes.c_void_p
_int = ctypes.c_int
_dbl = ctypes.c_double
_sz = ctypes.c_size_t
_pp = ctypes.POINTER(CParams)

# name -> (restype, argtypes); mirrors include/dclaw_b200.h
SIGNATURES = {
    "dclaw_abi_version": (_int, []),
    "dclaw_error_string": (ctypes.c_char_p, [_int]),
    "dclaw_params_default": (None, [_pp]),
    "dclaw_params_check": (_int, [_pp]),
    "dclaw_params_check_5": (_int, [_pp]),
    "dclaw_workspace_bytes": (_sz, [_int, _int]),
    "dclaw_bc2amr": (_int, [_vp, _int, _int, _int, _pp, _vp]),
    "dclaw_setaux": (_int, [_vp, _int, _int, _int, _pp, _vp]),
    "dclaw_b4step2": (_int, [_vp, _vp, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _pp, _vp, _vp]),
    "dclaw_step2": (_int, [_vp, _vp, _int, _int, _int, _dbl, _dbl, _dbl, _pp, _vp, _vp, _vp, _sz, _vp]),
    "dclaw_src2": (_int, [_vp, _vp, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _pp, _vp]),
    "dclaw_step": (_int, [_vp, _vp, _vp, _int, _int, _dbl, _dbl, _pp, _vp, _vp, _sz, _vp, _vp]),
    "dclaw_clock_init": (_int, [_vp, _dbl, _dbl, _dbl, _int, _vp]),
    "dclaw_clock_set_obs": (_int, [_vp, _dbl, _vp]),
    "dclaw_obs_record": (_int, [_vp, _int, _vp, _vp, _vp, ctypes.c_int64, _int, _int, _vp, _vp, _vp]),
    "dclaw_peak_update": (_int, [_vp, _vp, _vp, ctypes.c_int64, _int, _vp]),
    "dclaw_peak_adjoint": (_int, [_vp, _vp, ctypes.c_int64, _int, _vp, _vp]),
    "dclaw_fields_from_fortran": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _vp]),
    "dclaw_fields_to_fortran": (_int, [_vp, _int, _int, _int, _int, _int, _vp, _vp]),
    "dclaw_max_wave_speed": (_int, [_vp, _int, _int, _pp, _vp, _vp]),
    "dclaw_step_full": (_int, [_vp, _vp, _vp, _vp, _int, _int, _dbl, _dbl, _pp, _vp, _vp, _sz, _vp, _vp]),
    "dclaw_step_full_workspace_bytes": (_sz, [_int, _int]),
    "dclaw_step_noalloc": (_int, [_vp, _vp, _vp, _int, _int, _dbl, _dbl, _pp, _vp, _vp]),
    "dclaw_step_noalloc_max_cells": (_sz, []),
    "dclaw_step_host": (_int, [_vp, _vp, _vp, _int, _int, _dbl, _dbl, _pp, _vp, _vp, _sz, _int, _vp]),
    "dclaw_step_host_workspace_bytes": (_sz, [_int, _int]),
    "dclaw_step_host_bands": (_int, [_int, _int, _int, _vp, _int]),
    "dclaw_rows_granule": (_int, []),
    "dclaw_step_rows": (_int, [_vp, _vp, _vp, _int, _int, _dbl, _dbl, _pp, _vp, _vp, _sz, _int, _int, _vp]),
    "dclaw_clock_tick": (_int, [_vp, _pp, _vp]),
    "dclaw_batch_tile_shapes": (_int, [_vp, _vp, _int]),
    "dclaw_batch_layout": (_int, [_int, _vp, _vp, _vp, _vp, _int, ctypes.POINTER(CMember), ctypes.POINTER(CBatch)]),
    "dclaw_step_batched": (_int, [ctypes.POINTER(CBatch), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dclaw_batch_reset": (_int, [ctypes.POINTER(CBatch), _vp, _vp]),
    "dclaw_adjoint_workspace_bytes": (_sz, [_int, _int]),
    "dclaw_adjoint_supported": (_int, [_pp]),
    "dclaw_step_adjoint_prepare": (_int, [_vp, _vp, _int, _int, _dbl, _dbl, _vp, _pp, _vp, _sz, _vp, _vp]),
    "dclaw_step_adjoint_reverse": (_int, [_vp, _vp, _int, _int, _dbl, _dbl, _vp, _pp, _vp, _vp, _vp, _vp, _vp,
                                          _sz, _vp, _vp]),
    "dclaw_step_adjoint_batched_prepare": (_int, [ctypes.POINTER(CAdjBatch), _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                  _vp]),
    "dclaw_step_adjoint_batched_reverse": (_int, [ctypes.POINTER(CAdjBatch), _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                  _vp, _vp, _vp, _vp, _vp]),
    "dclaw_step_adjoint": (_int, [_vp, _vp, _int, _int, _dbl, _dbl, _vp, _pp, _vp, _vp, _vp, _vp, _vp, _sz, _vp,
                                  _vp]),
    "dclaw_adjoint_batch_layout": (_int, [_int, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(CAdjMember),
                                          ctypes.POINTER(CAdjBatch)]),
    "dclaw_step_adjoint_batched": (_int, [ctypes.POINTER(CAdjBatch), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                          _vp, _vp, _vp]),
}

_lib = None


class DClawError(RuntimeError):
    pass


def load() -> ctypes.CDLL:
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise DClawError(f"CUDA library not built: {LIB_PATH} is missing (run dclaw_b200.build.build())")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str = "dclaw call") -> None:
    if rc != 0:
        msg = load().dclaw_error_string(rc).decode()
        raise DClawError(f"{what} failed: {msg} (code {rc})")


def ptr(t) -> ctypes.c_void_p:
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return ctypes.c_void_p(0)
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None) -> ctypes.c_void_p:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


__all__ = ["load", "check", "ptr", "stream_ptr", "DClawError", "CParams", "CClock", "LIB_PATH", "SIGNATURES"]
