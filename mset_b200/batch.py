"""Batched method: every position of every tilt in one persistent launch.

All positions of all tilts see the same beam-frame volume, probe and scan
positions; the gradients are accumulated in FP64 on the device
(include/mset_b200.h, ``mset_batch_*``).  This changes the reference's
sequential per-position update (src/CUDA/mset.cu:107-333) into a gradient
step over the whole tilt series.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import MSET_ADJOINT_REF, MSET_MODE_MSET, check, dptr, fptr
from .session import _c32, _cplx_f32


class BatchSession:
    def __init__(self, *, n: int, nz: int, npos: Sequence[int], prop, sigma: float,
                 potential_pixelsize: float, slice_binning: int = 1, method: int = MSET_MODE_MSET,
                 adjoint: int = MSET_ADJOINT_REF, step_size=(0.0, 0.0, 0.0), device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        check("mset_create", self._lib.mset_create(int(device), C.byref(h)))
        self._h = h
        self.n, self.nz = int(n), int(nz)
        self.b = min(int(slice_binning), self.nz)
        self.method = int(method)
        self.ns = 1 if self.method == 2 else -(-self.nz // self.b)
        self.npos = np.ascontiguousarray(np.asarray(npos, dtype=np.int32))
        self.ntilts = int(self.npos.size)
        self._prop = _cplx_f32(prop)
        a = _lib.BatchArgs()
        a.n, a.nz, a.slice_binning = self.n, self.nz, int(slice_binning)
        a.method, a.adjoint = self.method, int(adjoint)
        a.sigma, a.potential_pixelsize = float(sigma), float(potential_pixelsize)
        a.step_size[:] = [float(v) for v in step_size]
        a.ntilts = self.ntilts
        a.npos = self.npos.ctypes.data_as(C.POINTER(C.c_int32))
        a.prop2D = fptr(self._prop)
        check("mset_batch_setup", self._lib.mset_batch_setup(self._h, C.byref(a)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mset_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tilt(self, j: int, *, probe=None, scan_x=None, scan_y=None, measured=None, volume=None):
        pr = _cplx_f32(probe) if probe is not None else None
        sx = _c32(scan_x).reshape(-1) if scan_x is not None else None
        sy = _c32(scan_y).reshape(-1) if scan_y is not None else None
        me = _c32(measured) if measured is not None else None
        vo = _c32(volume) if volume is not None else None
        check("mset_batch_set_tilt", self._lib.mset_batch_set_tilt(
            self._h, int(j), fptr(pr), fptr(sx), fptr(sy), fptr(me), fptr(vo)))

    def gradient(self, want=("grad", "probe", "posdir", "err")):
        return self._fetch(self._lib.mset_batch_gradient, "mset_batch_gradient", want)

    def _fetch(self, fn, name, want):
        g = np.zeros((self.ntilts, self.ns, self.n, self.n)) if "grad" in want else None
        p = np.zeros((self.ntilts, self.n, self.n, 2)) if "probe" in want else None
        d = np.zeros((int(self.npos.sum()), 2)) if "posdir" in want else None
        e = np.zeros(self.ntilts) if "err" in want else None
        check(name, fn(self._h, dptr(g), dptr(p), dptr(d), dptr(e)))
        out = {}
        if g is not None:
            out["grad"] = g
        if p is not None:
            out["probe"] = p[..., 0] + 1j * p[..., 1]
        if d is not None:
            out["posdir"] = d
        if e is not None:
            out["err"] = e
        return out

    def read_gradient(self, want=("grad", "probe", "posdir", "err")):
        """results of the last pass (e.g. one run through a SeriesGroup)"""
        return self._fetch(self._lib.mset_batch_read_gradient, "mset_batch_read_gradient", want)

    def tune(self, mem_budget_bytes: float = 0.0) -> dict:
        """pick persistent CTAs and checkpoint interval by timing (include/mset_b200.h)"""
        r = _lib.TuneResult()
        check("mset_batch_tune", self._lib.mset_batch_tune(self._h, float(mem_budget_bytes), C.byref(r)))
        return r.as_dict()

    def set_variant(self, variant: int):
        """use compiled kernel shape `variant` of this window (mset_batch_set_variant)"""
        check("mset_batch_set_variant", self._lib.mset_batch_set_variant(self._h, int(variant)))

    def variants(self) -> int:
        return int(self._lib.mset_batch_variants(self.n))

    def shape(self) -> dict:
        """the batch shape the next pass uses (mset_batch_get_tune)"""
        r = _lib.TuneResult()
        check("mset_batch_get_tune", self._lib.mset_batch_get_tune(self._h, C.byref(r)))
        return r.as_dict()

    def error(self) -> np.ndarray:
        e = np.zeros(self.ntilts)
        check("mset_batch_error", self._lib.mset_batch_error(self._h, dptr(e)))
        return e

    def simulate(self) -> np.ndarray:
        out = np.empty((int(self.npos.sum()), self.n, self.n), np.float32)
        check("mset_batch_simulate", self._lib.mset_batch_simulate(self._h, fptr(out)))
        return out

    def apply(self):
        check("mset_batch_apply", self._lib.mset_batch_apply(self._h))

    def get_tilt(self, j: int):
        v = np.empty((self.nz, self.n, self.n), np.float32)
        p = np.empty((self.n, self.n, 2), np.float32)
        k = max(int(self.npos[j]), 1)
        sx = np.empty(k, np.float32)
        sy = np.empty(k, np.float32)
        check("mset_batch_get_tilt", self._lib.mset_batch_get_tilt(self._h, int(j), fptr(v), fptr(p), fptr(sx), fptr(sy)))
        return v, p.view(np.complex64).reshape(self.n, self.n), sx[: self.npos[j]], sy[: self.npos[j]]

    def time_gradient(self, reps: int) -> float:
        ms = np.zeros(1)
        check("mset_batch_time", self._lib.mset_batch_time(self._h, int(reps), dptr(ms)))
        return float(ms[0])

    def time_plain(self, reps: int) -> float:
        """device ms per pass of the plain form (one launch per tilt, one CTA
        per position, no graph, no checkpointing)"""
        ms = np.zeros(1)
        check("mset_batch_time_plain", self._lib.mset_batch_time_plain(self._h, int(reps), dptr(ms)))
        return float(ms[0])

    def set_amplitude_bf16(self, on: bool = True):
        """keep measured counts as BF16 (set before the measured patterns)"""
        check("mset_batch_set_amplitude_bf16", self._lib.mset_batch_set_amplitude_bf16(self._h, int(bool(on))))

    def set_checkpoint(self, k: int):
        """keep the wave entering every k-th slab and recompute the rest in the
        adjoint (0: keep all)"""
        check("mset_batch_set_checkpoint", self._lib.mset_batch_set_checkpoint(self._h, int(k)))

    # ---- full batched iteration -------------------------------------------
    def iteration_setup(self, nv, angles, *, vec1=(0, 0, 1), vec2=(0, 1, 0), vec3=(1, 0, 0),
                        positivity=True, tv_lambda=0.0, tv_iter=300, tv_fista=True):
        """nv: the cubic reconstruction's edge, or its shape (nv3, nv2, nv1)
        (C order [nv3][nv2][nv1], nv3 = the session depth)"""
        self._angles = np.ascontiguousarray(np.asarray(angles, dtype=np.float32).reshape(-1, 3))
        self._vecs = [np.ascontiguousarray(np.asarray(v, dtype=np.float32)) for v in (vec1, vec2, vec3)]
        shape = (int(nv),) * 3 if np.isscalar(nv) else tuple(int(x) for x in nv)
        a = _lib.IterArgs()
        a.nv = shape[0]
        a.angles = fptr(self._angles)
        a.vec1, a.vec2, a.vec3 = (fptr(v) for v in self._vecs)
        a.use_positivity = int(bool(positivity))
        a.use_tv = int(tv_lambda > 0)
        a.tv_lambda = float(tv_lambda) if tv_lambda > 0 else 1.0
        a.tv_iter = int(tv_iter)
        a.tv_fista = int(bool(tv_fista))
        self.rec_shape = shape
        self.nv = shape[0]
        nv3, nv2, nv1 = shape
        check("mset_batch_iteration_setup_nd",
              self._lib.mset_batch_iteration_setup_nd(self._h, C.byref(a), nv1, nv2, nv3))

    def set_rec(self, rec):
        r = _c32(rec)
        check("mset_batch_set_rec", self._lib.mset_batch_set_rec(self._h, fptr(r)))

    def get_rec(self):
        r = np.empty(self.rec_shape, np.float32)
        check("mset_batch_get_rec", self._lib.mset_batch_get_rec(self._h, fptr(r)))
        return r

    def iterate(self, niter: int, use_graph: bool = True):
        e = np.zeros((max(niter, 1), self.ntilts))
        t = np.zeros(max(niter, 1))
        check("mset_batch_iterate", self._lib.mset_batch_iterate(self._h, int(niter), int(use_graph), dptr(e), dptr(t)))
        return e[:niter], t[:niter]

    def iterate_bls(self, niter: int, bls_parameter: float = 0.5):
        """iterations with the reference's backtracking line search
        (mset_batch_iterate_bls); returns (mean errors, step sizes) of the
        accepted iterations"""
        e = np.zeros(max(niter, 1))
        st = np.zeros((max(niter, 1), 3), np.float32)
        k = C.c_int()
        check("mset_batch_iterate_bls", self._lib.mset_batch_iterate_bls(
            self._h, int(niter), float(bls_parameter), dptr(e), fptr(st), C.byref(k)))
        return e[:k.value], st[:k.value]

    def time_iteration(self, niter: int) -> float:
        ms = np.zeros(1)
        check("mset_batch_iterate_time", self._lib.mset_batch_iterate_time(self._h, int(niter), dptr(ms)))
        return float(ms[0])


class SeriesGroup:
    """Several batched sessions (tilt series of any window, slab, scan and
    tilt counts) run as one pass (``mset_group_*`` in include/mset_b200.h)."""

    def __init__(self, sessions: Sequence[BatchSession], device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        check("mset_group_create", self._lib.mset_group_create(int(device), C.byref(h)))
        self._h = h
        self.sessions = list(sessions)  # kept alive: the group borrows them
        for s in self.sessions:
            check("mset_group_add", self._lib.mset_group_add(self._h, s._h))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mset_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_schedule(self, schedule: int):
        check("mset_group_set_schedule", self._lib.mset_group_set_schedule(self._h, int(schedule)))

    def tune(self, mem_budget_bytes: float = 0.0) -> int:
        sched = C.c_int()
        check("mset_group_tune", self._lib.mset_group_tune(self._h, float(mem_budget_bytes), C.byref(sched)))
        return int(sched.value)

    def run(self, use_graph: bool = True):
        check("mset_group_gradient", self._lib.mset_group_gradient(self._h, int(bool(use_graph))))

    def time(self, reps: int, use_graph: bool = True) -> float:
        ms = np.zeros(1)
        check("mset_group_time", self._lib.mset_group_time(self._h, int(reps), int(bool(use_graph)), dptr(ms)))
        return float(ms[0])


def split_ctas(work, ctas_per_sm, sms: int) -> np.ndarray:
    """mset_split_ctas: CTAs per member of a concurrent group pass"""
    lib = _lib.load()
    w = np.ascontiguousarray(np.asarray(work, dtype=np.float64))
    o = np.ascontiguousarray(np.asarray(ctas_per_sm, dtype=np.int32))
    out = np.zeros(w.size, np.int32)
    check("mset_split_ctas", lib.mset_split_ctas(int(w.size), dptr(w), o.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 int(sms), out.ctypes.data_as(C.POINTER(C.c_int32))))
    return out
