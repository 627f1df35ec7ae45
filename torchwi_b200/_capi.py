"""ctypes binding of the C ABI in include/twi_b200.h.

The CUDA library is mandatory: every entry point raises if it is missing or
if no CUDA device is present.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
import threading

from .build import LIB

_lock = threading.Lock()
_lib = None

TWI_OK, TWI_ERR_INVALID, TWI_ERR_CUDA, TWI_ERR_STATE, TWI_ERR_DEVICE, TWI_ERR_NOMEM = range(6)


class TwiError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[twi status {status}] {message}")
        self.status = status


class TwiInvalid(TwiError, ValueError):
    pass


class Problem(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int), ("nx", ctypes.c_int), ("nz", ctypes.c_int),
                ("nt", ctypes.c_int), ("h", ctypes.c_float), ("dt", ctypes.c_float),
                ("nshots", ctypes.c_int), ("ckpt_interval", ctypes.c_int),
                ("exact", ctypes.c_int), ("accumulate", ctypes.c_int),
                ("shots_per_cta", ctypes.c_int), ("rows_per_warp", ctypes.c_int),
                ("use_graphs", ctypes.c_int), ("wavelet_per_shot", ctypes.c_int),
                ("forward_only", ctypes.c_int), ("exa", ctypes.c_int),
                ("time_block", ctypes.c_int), ("reconstruct", ctypes.c_int),
                ("persistent", ctypes.c_int),
                ("unchained", ctypes.c_int)]


class Layout(ctypes.Structure):
    _fields_ = [("workspace_bytes", ctypes.c_size_t), ("vel", ctypes.c_size_t),
                ("wavelet", ctypes.c_size_t), ("gathers", ctypes.c_size_t),
                ("resid", ctypes.c_size_t), ("grad", ctypes.c_size_t),
                ("dimx", ctypes.c_int), ("dimz", ctypes.c_int), ("pitch", ctypes.c_int),
                ("ckpt_interval", ctypes.c_int), ("nsegments", ctypes.c_int),
                ("shots_per_cta", ctypes.c_int), ("rows_per_warp", ctypes.c_int),
                ("time_block", ctypes.c_int), ("adjoint_rows_per_warp", ctypes.c_int),
                ("adjoint_shots_per_cta", ctypes.c_int)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "twi_version": [],
    "twi_last_error": [],
    "twi_fdm_forward": [_vp] * 7 + [_i] * 4 + [_f] * 5 + [_vp],
    "twi_fdm_backward": [_vp] * 7 + [_i] * 4 + [_f] * 3 + [_vp],
    "twi_fdm_forward_only": [_vp] * 6 + [_i] * 4 + [_f] * 5 + [_vp],
    "twi_fdm_forward_only_noalloc": [_vp] * 3 + [_i] * 4 + [_f] * 5 + [_vp],
    "twi_fdm_exa_forward": [_vp] * 8 + [_i] * 4 + [_f] * 5 + [_vp],
    "twi_fdm_exa_backward": [_vp] * 8 + [_i] * 4 + [_f] * 3 + [_vp],
    "twi_plan_create": [ctypes.POINTER(Problem), ctypes.POINTER(_vp)],
    "twi_plan_layout": [_vp, ctypes.POINTER(Layout)],
    "twi_plan_bind": [_vp, _vp, ctypes.c_size_t],
    "twi_plan_set_shots": [_vp, _vp, _vp, _vp, _vp],
    "twi_plan_set_model": [_vp, _vp],
    "twi_forward": [_vp, _i, _vp],
    "twi_forward_residual": [_vp, _vp, _vp, _vp],
    "twi_residual": [_vp, _vp, _vp, _vp],
    "twi_gradient": [_vp, _vp],
    "twi_plan_check": [_vp, _vp],
    "twi_plan_profile": [_vp, _i, _i, ctypes.POINTER(ctypes.c_float), _vp],
    "twi_plan_destroy": [_vp],
    "twi_plan_footprint_bytes": [_vp, ctypes.POINTER(ctypes.c_size_t)],
    "twi_check_wait_timeout": [_i, ctypes.POINTER(ctypes.c_float), _vp],
    "twi_check_counter_wait": [_i, _i, ctypes.POINTER(ctypes.c_float), _vp],
    "twi_autotune_scratch_bytes": [_vp, ctypes.POINTER(ctypes.c_size_t)],
    "twi_autotune": [_vp, _vp, ctypes.c_size_t, _vp, _vp, ctypes.POINTER(ctypes.c_float)],
    "twi_batch_create": [ctypes.POINTER(_vp), _i, ctypes.POINTER(_vp)],
    "twi_batch_workspace_size": [_vp, ctypes.POINTER(ctypes.c_size_t)],
    "twi_batch_bind": [_vp, _vp, ctypes.c_size_t],
    "twi_batch_forward": [_vp, _i, _vp],
    "twi_batch_gradient": [_vp, _vp],
    "twi_batch_destroy": [_vp],
    "twi_engine_create": [_i, _i, _i, _i, ctypes.POINTER(_vp)],
    "twi_engine_workspace_size": [_vp, ctypes.POINTER(ctypes.c_size_t)],
    "twi_engine_bind": [_vp, _vp, ctypes.c_size_t],
    "twi_engine_submit": [_vp, _vp, _i, _vp, ctypes.c_longlong],
    "twi_engine_run": [_vp, _i, _vp, ctypes.POINTER(ctypes.c_longlong), _i, ctypes.POINTER(_i)],
    "twi_engine_pending": [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)],
    "twi_engine_destroy": [_vp],
}
_RESTYPES = {"twi_last_error": ctypes.c_char_p}


def lib() -> ctypes.CDLL:
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB):
                raise TwiError(TWI_ERR_CUDA,
                               f"CUDA library {LIB} is missing; run `python -m torchwi_b200.build` "
                               "(there is no CPU fallback)")
            L = ctypes.CDLL(LIB)
            for name, args in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, ctypes.c_int)
            _lib = L
        return _lib


def last_error() -> str:
    msg = lib().twi_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status != TWI_OK:
        msg = last_error()
        if status == TWI_ERR_INVALID:
            raise TwiInvalid(status, msg)
        raise TwiError(status, msg)
