"""ctypes driver of oracle/_ref/libmset_ref.so: the reference's own CUDA MEX
code (src/CUDA/mex_main.cu, mset.cu, utility.cu, mex_tools.cpp, compiled
unchanged with `make -C oracle ref`) behind the project's mex shim.

TEST INFRASTRUCTURE ONLY: a checker and a timed baseline; it needs a GPU
and cuFFT.  Inputs use the MEX layouts (C order [nz][n][n] volume, [n][n]
complex probe and centred propagator, [P][n][n] centred measured patterns).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libmset_ref.so")
# this library's MEX gateway (mset_b200/mex/mset_cuda_kernel.cpp) behind the
# same shim and driver (make -C oracle gw)
GATEWAY = os.path.join(HERE, "_gw", "libmset_gateway.so")
_F = C.POINTER(C.c_float)
_libs = {}


def available(path: str = LIB) -> bool:
    return os.path.exists(path)


def lib(path: str = LIB) -> C.CDLL:
    if path not in _libs:
        L = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_upload.argtypes = [C.c_int, C.c_int, _F, _F, _F, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                 _F, _F, _F, C.c_int, _F]
        L.ref_run.argtypes = [C.c_int, _F, _F, _F, _F, _F]
        L.ref_error.argtypes = [C.c_int, _F]
        L.ref_mode.argtypes = [C.c_char_p]
        _libs[path] = L
    return _libs[path]


def _f(a):
    return a.ctypes.data_as(_F)


class RefSession:
    """upload / run / error through a MEX gateway and the shim: the
    reference's own (default) or this library's (path=GATEWAY)"""

    def __init__(self, path: str = LIB):
        self.path = path

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"MEX call failed ({rc}): {lib(self.path).ref_last_error().decode()}")

    def upload(self, rvol, probe, prop, *, sigma, dz, scan_x, scan_y, measured, step=(0, 0, 0), binning=1,
               nsx=None, nsy=None):
        self.rvol = np.ascontiguousarray(rvol, dtype=np.float32)
        self.nz, self.n, _ = self.rvol.shape
        self.probe = np.ascontiguousarray(probe, dtype=np.complex64)
        self.prop = np.ascontiguousarray(prop, dtype=np.complex64)
        self.sx = np.ascontiguousarray(scan_x, dtype=np.float32)
        self.sy = np.ascontiguousarray(scan_y, dtype=np.float32)
        self.meas = np.ascontiguousarray(measured, dtype=np.float32)
        self.step = np.asarray(step, dtype=np.float32)
        self.npos = self.sx.size
        nsx = self.npos if nsx is None else nsx
        nsy = 1 if nsy is None else nsy
        self._check(lib(self.path).ref_upload(self.n, self.nz, _f(self.rvol), _f(self.probe.view(np.float32)),
                                _f(self.prop.view(np.float32)), float(sigma), float(dz), int(nsx), int(nsy),
                                self.npos, _f(self.sx), _f(self.sy), _f(self.step), int(binning), _f(self.meas)))

    def run(self, mode=1):
        rv = np.empty((self.nz, self.n, self.n), np.float32)
        pr = np.empty((self.n, self.n), np.complex64)
        sx = np.empty(self.npos, np.float32)
        sy = np.empty(self.npos, np.float32)
        err = np.zeros(1, np.float32)
        self._check(lib(self.path).ref_run(int(mode), _f(rv), _f(pr.view(np.float32)), _f(sx), _f(sy), _f(err)))
        return rv, pr, sx, sy, float(err[0])

    def error(self, mode=1) -> float:
        err = np.zeros(1, np.float32)
        self._check(lib(self.path).ref_error(int(mode), _f(err)))
        return float(err[0])
