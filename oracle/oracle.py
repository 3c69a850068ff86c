"""ctypes wrapper of oracle/libmset_oracle.so (FP64 restatement of the
reference's per-position model and tilt passes, mset_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared against.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmset_oracle.so")
_lib = None

_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)


def build() -> None:
    subprocess.run(["make", "-C", HERE, "libmset_oracle.so"], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "mset_oracle.c")):
            build()
        L = C.CDLL(LIB)
        L.orc_fft2.argtypes = [_D, C.c_int, C.c_int, C.c_int]
        L.orc_run_tilt.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D, C.c_int, C.c_int,
                                   C.c_int, C.c_int, _F, _F, _F, _F, _F, _F, _D]
        L.orc_position.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _D, _D,
                                   _D, C.c_double, C.c_double, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        L.orc_position_loss.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _D, _D, _D,
                                        C.c_double, C.c_double, _D]
        L.orc_position_loss.restype = C.c_double
        L.orc_batched_tilt.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                       C.c_int, _F, _F, _F, _F, _F, _F, _D, _D, _D, _D, C.c_int]
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _f(a):
    return None if a is None else a.ctypes.data_as(_F)


def _d(a):
    return None if a is None else a.ctypes.data_as(_D)


def fft2(a: np.ndarray, sign: int = -1) -> np.ndarray:
    z = np.ascontiguousarray(a, dtype=np.complex128).copy()
    lib().orc_fft2(z.view(np.float64).ctypes.data_as(_D), z.shape[0], z.shape[1], sign)
    return z


def run_tilt(rvol, probe, prop, scan_x, scan_y, measured, *, sigma, dz, step=(0, 0, 0), binning=1,
             method=1, adjoint=0, update=True):
    """Sequential tilt pass (mset.cu run_main_* / run_error_*).  Returns
    (rvol, probe, scan_x, scan_y, err_sum) with err_sum = sum over positions and
    pixels of (A-M)^2 (not normalised)."""
    rv = np.ascontiguousarray(rvol, dtype=np.float32).copy()
    nz, n, _ = rv.shape
    pr = np.ascontiguousarray(probe, dtype=np.complex64).copy()
    pp = np.ascontiguousarray(prop, dtype=np.complex64)
    sx = np.ascontiguousarray(scan_x, dtype=np.float32).copy()
    sy = np.ascontiguousarray(scan_y, dtype=np.float32).copy()
    me = np.ascontiguousarray(measured, dtype=np.float32)
    st = np.asarray(step, dtype=np.float64)
    err = np.zeros(1)
    rc = lib().orc_run_tilt(n, nz, binning, sigma, dz, _d(st), method, adjoint, int(update), sx.size,
                            _f(rv), pr.view(np.float32).ctypes.data_as(_F), pp.view(np.float32).ctypes.data_as(_F),
                            _f(sx), _f(sy), _f(me), _d(err))
    assert rc == 0
    return rv, pr, sx, sy, float(err[0])


def amp_std(measured_one: np.ndarray) -> np.ndarray:
    """sqrt(ifftshift(I)) in standard FFT order (mset.cu:206-210)."""
    return np.ascontiguousarray(np.sqrt(np.fft.ifftshift(np.asarray(measured_one, dtype=np.float64))))


def position(V, probe, prop, scan_x, scan_y, amp, *, sigma, dz, binning=1, method=1, adjoint=0):
    """One position in FP64: dict with psi0, far, err, grad (ns slabs, complex),
    chi0, probe_dir, pos_dir, waves (ns+1: psi0, then the wave after each slab)."""
    V = np.ascontiguousarray(V, dtype=np.float64)
    nz, n, _ = V.shape
    ns = 1 if method == 2 else -(-nz // binning)
    pr = np.ascontiguousarray(probe, dtype=np.complex128)
    pp = np.ascontiguousarray(prop, dtype=np.complex128)
    am = np.ascontiguousarray(amp, dtype=np.float64)
    out = dict(psi0=np.zeros((n, n), np.complex128), far=np.zeros((n, n), np.complex128),
               grad=np.zeros((ns, n, n), np.complex128), chi0=np.zeros((n, n), np.complex128),
               probe_dir=np.zeros((n, n), np.complex128), waves=np.zeros((ns + 1, n, n), np.complex128))
    err = np.zeros(1)
    pd = np.zeros(2)
    c = lambda a: a.view(np.float64).ctypes.data_as(_D)
    rc = lib().orc_position(n, nz, binning, sigma, dz, method, adjoint, _d(V), c(pr), c(pp), float(scan_x),
                            float(scan_y), _d(am), c(out["psi0"]), c(out["far"]), _d(err), c(out["grad"]),
                            c(out["chi0"]), c(out["probe_dir"]), _d(pd), c(out["waves"]))
    assert rc == 0
    out["err"] = float(err[0])
    out["pos_dir"] = pd
    return out


def position_loss(V, probe, prop, scan_x, scan_y, amp, *, sigma, dz, binning=1, method=1) -> float:
    V = np.ascontiguousarray(V, dtype=np.float64)
    nz, n, _ = V.shape
    pr = np.ascontiguousarray(probe, dtype=np.complex128)
    pp = np.ascontiguousarray(prop, dtype=np.complex128)
    am = np.ascontiguousarray(amp, dtype=np.float64)
    c = lambda a: a.view(np.float64).ctypes.data_as(_D)
    return lib().orc_position_loss(n, nz, binning, sigma, dz, method, _d(V), c(pr), c(pp), float(scan_x),
                                   float(scan_y), _d(am))


def batched_tilt(rvol, probe, prop, scan_x, scan_y, measured, *, sigma, dz, binning=1, method=1, adjoint=0,
                 nthreads=0):
    """Batched pass over one tilt: (grad_slab [ns][n][n], probe_acc [n][n]
    complex, pos_dir [P][2], err_sum)."""
    rv = np.ascontiguousarray(rvol, dtype=np.float32)
    nz, n, _ = rv.shape
    ns = 1 if method == 2 else -(-nz // binning)
    pr = np.ascontiguousarray(probe, dtype=np.complex64)
    pp = np.ascontiguousarray(prop, dtype=np.complex64)
    sx = np.ascontiguousarray(scan_x, dtype=np.float32)
    sy = np.ascontiguousarray(scan_y, dtype=np.float32)
    me = np.ascontiguousarray(measured, dtype=np.float32)
    g = np.zeros((ns, n, n))
    pa = np.zeros((n, n, 2))
    pd = np.zeros((sx.size, 2))
    err = np.zeros(1)
    rc = lib().orc_batched_tilt(n, nz, binning, sigma, dz, method, adjoint, sx.size, _f(rv),
                                pr.view(np.float32).ctypes.data_as(_F), pp.view(np.float32).ctypes.data_as(_F),
                                _f(sx), _f(sy), _f(me), _d(g), _d(pa), _d(pd), _d(err), int(nthreads))
    assert rc == 0
    return g, pa[..., 0] + 1j * pa[..., 1], pd, float(err[0])


def max_threads() -> int:
    return lib().orc_max_threads()


_lib32 = None


def lib32() -> C.CDLL:
    """oracle/libcpu_fp32.so: the single-precision CPU port (cpu_fp32.c)"""
    global _lib32
    if _lib32 is None:
        p = os.path.join(HERE, "libcpu_fp32.so")
        if not os.path.exists(p) or os.path.getmtime(p) < os.path.getmtime(os.path.join(HERE, "cpu_fp32.c")):
            subprocess.run(["make", "-C", HERE, "libcpu_fp32.so"], check=True, capture_output=True)
        L = C.CDLL(p)
        L.cpu32_batched_tilt.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _F, _F, _F,
                                         _F, _F, _F, _D, _D, _D, _D, C.c_int]
        L.cpu32_simulate.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _F, _F, _F, _F,
                                     _F, _F, C.c_int]
        L.cpu32_sequential_tilt.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D, C.c_int, _F,
                                            _F, _F, _F, _F, _F, _D]
        _lib32 = L
    return _lib32


def batched_tilt_fp32(rvol, probe, prop, scan_x, scan_y, measured, *, sigma, dz, binning=1, nthreads=0):
    """The batched pass over one tilt in single precision (cpu_fp32.c; window
    a power of two, reference adjoint formula): the same outputs as
    batched_tilt."""
    rv = np.ascontiguousarray(rvol, dtype=np.float32)
    nz, n, _ = rv.shape
    ns = -(-nz // binning)
    pr = np.ascontiguousarray(probe, dtype=np.complex64)
    pp = np.ascontiguousarray(prop, dtype=np.complex64)
    sx = np.ascontiguousarray(scan_x, dtype=np.float32)
    sy = np.ascontiguousarray(scan_y, dtype=np.float32)
    me = np.ascontiguousarray(measured, dtype=np.float32)
    g = np.zeros((ns, n, n))
    pa = np.zeros((n, n, 2))
    pd = np.zeros((sx.size, 2))
    err = np.zeros(1)
    rc = lib32().cpu32_batched_tilt(n, nz, binning, sigma, dz, sx.size, _f(rv),
                                    pr.view(np.float32).ctypes.data_as(_F), pp.view(np.float32).ctypes.data_as(_F),
                                    _f(sx), _f(sy), _f(me), _d(g), _d(pa), _d(pd), _d(err), int(nthreads))
    if rc != 0:
        raise ValueError("cpu_fp32: the window must be a power of two")
    return g, pa[..., 0] + 1j * pa[..., 1], pd, float(err[0])


def sequential_tilt_fp32(rvol, probe, prop, scan_x, scan_y, measured, *, sigma, dz, step, binning=1):
    """The reference-semantics tilt pass (run_main_mset) in single precision on
    one thread (cpu_fp32.c): returns the updated (rvol, probe, scan_x,
    scan_y) and the error sum, as run_tilt does in FP64."""
    rv = np.array(rvol, dtype=np.float32, order="C")
    nz, n, _ = rv.shape
    pr = np.array(probe, dtype=np.complex64, order="C")
    pp = np.ascontiguousarray(prop, dtype=np.complex64)
    sx = np.array(scan_x, dtype=np.float32)
    sy = np.array(scan_y, dtype=np.float32)
    me = np.ascontiguousarray(measured, dtype=np.float32)
    st = np.asarray(step, dtype=np.float64)
    err = np.zeros(1)
    rc = lib32().cpu32_sequential_tilt(n, nz, binning, sigma, dz, _d(st), sx.size, _f(rv),
                                       pr.view(np.float32).ctypes.data_as(_F), pp.view(np.float32).ctypes.data_as(_F),
                                       _f(sx), _f(sy), _f(me), _d(err))
    if rc != 0:
        raise ValueError("cpu_fp32: the window must be a power of two")
    return rv, pr, sx, sy, float(err[0])


def _rot_setup():
    L = lib()
    L.orc_rot3d.argtypes = [_D, C.c_int, C.c_int, C.c_int, _D, _D, _D, C.c_double, C.c_double, C.c_double, C.c_int]
    L.orc_rotation_matrix.argtypes = [_D, _D, _D, C.c_double, C.c_double, C.c_double, C.c_int, _D]
    L.orc_rotation_plan.argtypes = [_D, C.c_double, _D]
    return L


VEC1, VEC2, VEC3 = (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), (1.0, 0.0, 0.0)  # main.m:25-27


def rot3d(vol, angles, inverse=False, vecs=(VEC1, VEC2, VEC3)):
    """Func_rot_3Dvol_FourierShear (inverse=False) / Func_inv_rot_3Dvol_FourierShear
    (inverse=True) of a C-order [n3][n2][n1] volume (MATLAB size n1 x n2 x n3),
    FP64.  angles = (phi, theta, psi) in degrees."""
    L = _rot_setup()
    v = np.ascontiguousarray(vol, dtype=np.float64).copy()
    n3, n2, n1 = v.shape
    vv = [np.asarray(x, dtype=np.float64) for x in vecs]
    L.orc_rot3d(_d(v), n1, n2, n3, _d(vv[0]), _d(vv[1]), _d(vv[2]), float(angles[0]), float(angles[1]),
                float(angles[2]), int(inverse))
    return v


def rotation_matrix(angles, inverse=False, vecs=(VEC1, VEC2, VEC3)):
    L = _rot_setup()
    vv = [np.asarray(x, dtype=np.float64) for x in vecs]
    M = np.zeros(9)
    active = L.orc_rotation_matrix(_d(vv[0]), _d(vv[1]), _d(vv[2]), float(angles[0]), float(angles[1]),
                                   float(angles[2]), int(inverse), _d(M))
    return M.reshape(3, 3), bool(active)


def rotation_plan(M, step=11.0):
    L = _rot_setup()
    M = np.ascontiguousarray(M, dtype=np.float64)
    out = np.zeros(11)
    L.orc_rotation_plan(_d(M), float(step), _d(out))
    return dict(num_step=int(out[0]), forward=bool(out[1]), mI=int(out[2]), coeffs=out[3:].copy())


def simulate_fp32(rvol, probe, prop, scan_x, scan_y, *, sigma, dz, binning=1, nthreads=0):
    """|Psi|^2 in the centred layout [P][n][n] of every position (single
    precision, cpu_fp32.c): the forward model for host-side test data."""
    rv = np.ascontiguousarray(rvol, dtype=np.float32)
    nz, n, _ = rv.shape
    pr = np.ascontiguousarray(probe, dtype=np.complex64)
    pp = np.ascontiguousarray(prop, dtype=np.complex64)
    sx = np.ascontiguousarray(scan_x, dtype=np.float32)
    sy = np.ascontiguousarray(scan_y, dtype=np.float32)
    out = np.zeros((sx.size, n, n), np.float32)
    rc = lib32().cpu32_simulate(n, nz, binning, sigma, dz, sx.size, _f(rv), pr.view(np.float32).ctypes.data_as(_F),
                                pp.view(np.float32).ctypes.data_as(_F), _f(sx), _f(sy), _f(out), int(nthreads))
    if rc != 0:
        raise ValueError("cpu_fp32: the window must be a power of two")
    return out
