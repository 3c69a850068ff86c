"""ctypes binding of libmset_b200.so (the C ABI declared in include/mset_b200.h).

The shared library is built in-tree by ``mset_b200/csrc/Makefile``
(``python -c "import __graft_entry__ as g; g.build()"``).  There is no
fallback: if the library is missing or a CUDA device is absent, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmset_b200.so")
CSRC = os.path.join(_HERE, "csrc")

MSET_MODE_MSET = 1
MSET_MODE_SSET = 2
MSET_ADJOINT_REF = 0
MSET_ADJOINT_EXACT = 1
# status codes (include/mset_b200.h)
MSET_E_ARG = -1
MSET_E_UNSUPPORTED = -2
MSET_E_CUDA = -3
MSET_E_STATE = -4
MSET_E_NOMEM = -5

_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)

# every symbol the header declares, with (restype, argtypes)
SIGNATURES = {
    "mset_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "mset_destroy": (C.c_int, [C.c_void_p]),
    "mset_last_error": (C.c_char_p, []),
    "mset_version": (C.c_char_p, []),
    "mset_upload": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mset_run": (C.c_int, [C.c_void_p, C.c_int, _F, _F, _F, _F, _F]),
    "mset_run_ex": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _F, _F, _F, _F, _F]),
    "mset_error": (C.c_int, [C.c_void_p, C.c_int, _F]),
    "mset_forward_position": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, _F, _F, _F, _F, _F]),
    "mset_adjoint_position": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _F, C.c_int, _F, _F, _F]),
    "mset_upload_cells": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(_F)]),
    "mset_mex_upload_cells": (C.c_int, [C.c_void_p, C.POINTER(_F)]),
    "mset_read_state": (C.c_int, [C.c_void_p, _F, _F]),
    "mset_set_sequential_split": (C.c_int, [C.c_void_p, C.c_int]),
    "mset_sequential_split": (C.c_int, [C.c_void_p]),
    "mset_batch_time_plain": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "mset_mex_upload": (C.c_int, [C.c_void_p]),
    "mset_mex_run": (C.c_int, [C.c_int, _F, _F, _F, _F, _F]),
    "mset_mex_error": (C.c_int, [C.c_int, _F]),
    "mset_mex_clear": (C.c_int, []),
    "mset_mex_session": (C.c_void_p, []),
    "mset_batch_setup": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mset_batch_set_tilt": (C.c_int, [C.c_void_p, C.c_int, _F, _F, _F, _F, _F]),
    "mset_batch_set_volume": (C.c_int, [C.c_void_p, C.c_int, _F]),
    "mset_batch_gradient": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "mset_batch_error": (C.c_int, [C.c_void_p, _D]),
    "mset_batch_simulate": (C.c_int, [C.c_void_p, _F]),
    "mset_batch_apply": (C.c_int, [C.c_void_p]),
    "mset_batch_get_tilt": (C.c_int, [C.c_void_p, C.c_int, _F, _F, _F, _F]),
    "mset_batch_time": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "mset_batch_launch_count": (C.c_int, [C.c_void_p]),
    "mset_rotate_volume": (C.c_int, [C.c_void_p, _F, _F, C.c_int, _F, _F, _F, C.c_double, C.c_double, C.c_double,
                                     C.c_int]),
    "mset_batch_set_amplitude_bf16": (C.c_int, [C.c_void_p, C.c_int]),
    "mset_batch_set_checkpoint": (C.c_int, [C.c_void_p, C.c_int]),
    "mset_batch_iteration_setup": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mset_batch_iteration_setup_nd": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "mset_rotate_volume_nd": (C.c_int, [C.c_void_p, _F, _F, C.c_int, C.c_int, C.c_int, _F, _F, _F, C.c_double,
                                        C.c_double, C.c_double, C.c_int]),
    "mset_batch_set_rec": (C.c_int, [C.c_void_p, _F]),
    "mset_batch_get_rec": (C.c_int, [C.c_void_p, _F]),
    "mset_batch_iterate": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D]),
    "mset_batch_iterate_bls": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _D, _F, C.POINTER(C.c_int)]),
    "mset_batch_iterate_time": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "mset_batch_iterate_phase": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "mset_batch_device_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                                         C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "mset_tv": (C.c_int, [C.c_void_p, _F, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, _D]),
    "mset_batch_read_gradient": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "mset_batch_tune": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "mset_batch_get_tune": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mset_batch_variants": (C.c_int, [C.c_int]),
    "mset_batch_set_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "mset_group_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "mset_group_destroy": (C.c_int, [C.c_void_p]),
    "mset_group_add": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mset_group_set_schedule": (C.c_int, [C.c_void_p, C.c_int]),
    "mset_group_tune": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
    "mset_group_gradient": (C.c_int, [C.c_void_p, C.c_int]),
    "mset_group_time": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D]),
    "mset_split_ctas": (C.c_int, [C.c_int, _D, _I, C.c_int, _I]),
    "mset_batch_gradient_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                              C.c_float, C.c_float, C.c_int] + [C.c_void_p] * 10),
}


class UploadArgs(C.Structure):
    """mset_upload_args (include/mset_b200.h)."""

    _fields_ = [
        ("n", C.c_int32),
        ("nz", C.c_int32),
        ("num_scan_pos", C.c_int32),
        ("N_scan_x", C.c_int32),
        ("N_scan_y", C.c_int32),
        ("sigma", C.c_float),
        ("potential_pixelsize", C.c_float),
        ("alpha", C.c_float),
        ("E0", C.c_float),
        ("step_size", C.c_float * 3),
        ("slice_binning", C.c_int32),
        ("RVol", _F),
        ("init_wave2D", _F),
        ("prop2D", _F),
        ("scan_xlist", _F),
        ("scan_ylist", _F),
        ("measured", _F),
    ]


class BatchArgs(C.Structure):
    """mset_batch_args (include/mset_b200.h)."""

    _fields_ = [
        ("n", C.c_int32),
        ("nz", C.c_int32),
        ("slice_binning", C.c_int32),
        ("method", C.c_int32),
        ("adjoint", C.c_int32),
        ("sigma", C.c_float),
        ("potential_pixelsize", C.c_float),
        ("step_size", C.c_float * 3),
        ("ntilts", C.c_int32),
        ("npos", _I),
        ("prop2D", _F),
    ]


class IterArgs(C.Structure):
    """mset_iter_args (include/mset_b200.h)."""

    _fields_ = [
        ("nv", C.c_int32),
        ("angles", _F),
        ("vec1", _F),
        ("vec2", _F),
        ("vec3", _F),
        ("use_positivity", C.c_int32),
        ("use_tv", C.c_int32),
        ("tv_lambda", C.c_double),
        ("tv_iter", C.c_int32),
        ("tv_fista", C.c_int32),
    ]


class TuneResult(C.Structure):
    """mset_tune_result (include/mset_b200.h)."""

    _fields_ = [
        ("grid", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("checkpoint", C.c_int32),
        ("candidates", C.c_int32),
        ("us_per_position", C.c_double),
        ("save_bytes", C.c_double),
        ("threads", C.c_int32),
        ("staged", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


MSET_GROUP_SERIAL = 0
MSET_GROUP_CONCURRENT = 1


class MsetError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, func: str, code: int, msg: str):
        super().__init__(f"{func} failed ({code}): {msg}")
        self.code = code


_lock = threading.Lock()
_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load libmset_b200.so once; raise if it is missing (no fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise FileNotFoundError(
                f"{p} is missing: build it with `make -C {CSRC} -j8` "
                "(or __graft_entry__.build()); mset_b200 has no CPU fallback")
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        return lib


def check(func: str, rc: int) -> None:
    if rc != 0:
        msg = load().mset_last_error().decode(errors="replace")
        raise MsetError(func, rc, msg)


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_F)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)
