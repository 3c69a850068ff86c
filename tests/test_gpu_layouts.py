"""One session handle used first by the sequential entry points, then by the
batched method, then by the sequential ones again, at the 128 x 128 window.
The two kinds of session take kernel shapes with different scrambled
Fourier layouts there (the two-pass shape shared with the 8-CTA sequential
cluster geometry, the three-phase batched shape), so each setup must rebuild
the session's twiddle, propagator and probe tables for its own shape: the
results equal those of fresh sessions of each kind."""
import ctypes as C

import numpy as np

from mset_b200 import _lib
from mset_b200._lib import check, dptr, fptr
from mset_b200.batch import BatchSession
from mset_b200.session import Session
from tests.helpers import rel_l2, small_case

import pytest

pytestmark = pytest.mark.gpu


def _batch_on_handle(lib, h, c, npos):
    """mset_batch_setup / set_tilt / gradient through the C ABI on handle h"""
    prop = np.ascontiguousarray(c["prop"], dtype=np.complex64)
    n, nz = c["V"].shape[1], c["V"].shape[0]
    a = _lib.BatchArgs()
    a.n, a.nz, a.slice_binning = n, nz, c["b"]
    a.method, a.adjoint = 1, 0
    a.sigma, a.potential_pixelsize = float(c["sigma"]), float(c["dz"])
    a.step_size[:] = [0.0, 0.0, 0.0]
    a.ntilts = 1
    counts = np.array([npos], np.int32)
    a.npos = counts.ctypes.data_as(C.POINTER(C.c_int32))
    a.prop2D = fptr(prop.view(np.float32))
    check("mset_batch_setup", lib.mset_batch_setup(h, C.byref(a)))
    pr = np.ascontiguousarray(c["probe"], dtype=np.complex64).view(np.float32)
    sx = np.ascontiguousarray(c["sx"], np.float32)
    sy = np.ascontiguousarray(c["sy"], np.float32)
    me = np.ascontiguousarray(c["meas"], np.float32)
    vo = np.ascontiguousarray(c["V"], np.float32)
    check("mset_batch_set_tilt", lib.mset_batch_set_tilt(h, 0, fptr(pr), fptr(sx), fptr(sy), fptr(me), fptr(vo)))
    ns = -(-nz // c["b"])
    g = np.zeros((1, ns, n, n))
    p = np.zeros((1, n, n, 2))
    d = np.zeros((npos, 2))
    e = np.zeros(1)
    check("mset_batch_gradient", lib.mset_batch_gradient(h, dptr(g), dptr(p), dptr(d), dptr(e)))
    return g, p, d, e


def _upload_run(s, c, npos):
    s.upload(c["V"], c["probe"], c["prop"], sigma=c["sigma"], potential_pixelsize=c["dz"], scan_x=c["sx"],
             scan_y=c["sy"], measured=c["meas"], step_size=(1e-3, 1e-6, 1e-3), slice_binning=c["b"],
             n_scan_x=npos, n_scan_y=1)
    return s.run(1)


def test_one_handle_switches_between_sequential_and_batched_layouts(gpu_available):
    npos = 4
    c = small_case(n=128, nz=6, npos=npos, b=2, seed=31, defocus=15.0, jitter=5.0, strength=20.0)
    with Session() as fresh:
        seq_ref = _upload_run(fresh, c, npos)
    bs = BatchSession(n=128, nz=6, npos=[npos], prop=c["prop"], sigma=c["sigma"], potential_pixelsize=c["dz"],
                      slice_binning=c["b"])
    bs.set_tilt(0, probe=c["probe"], scan_x=c["sx"], scan_y=c["sy"], measured=c["meas"], volume=c["V"])
    bat_ref = bs.gradient()
    bs.close()
    with Session() as s:
        seq1 = _upload_run(s, c, npos)
        g, p, d, e = _batch_on_handle(s._lib, s._h, c, npos)
        seq2 = _upload_run(s, c, npos)
    for a, b in zip(seq1, seq_ref):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    for a, b in zip(seq2, seq_ref):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    assert rel_l2(g, bat_ref["grad"]) < 1e-9
    assert rel_l2(p[..., 0] + 1j * p[..., 1], bat_ref["probe"]) < 1e-9
    assert rel_l2(d, bat_ref["posdir"]) < 1e-9
    assert abs(e[0] - bat_ref["err"][0]) <= 1e-9 * bat_ref["err"][0]
