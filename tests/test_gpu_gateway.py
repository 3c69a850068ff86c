"""The MEX gateway a MATLAB user builds (mset_b200/mex/mset_cuda_kernel.cpp),
compiled against the project's MEX API shim (make -C oracle gw) and driven
with the call sequence of Run_MSET_recon.m:162-174 / 226-235 ('upload',
'run_mset' / 'run_sset', 'upload', 'error_mset' / 'error_sset'), beside the
reference's own MEX module behind the same shim (oracle/_ref) and this
library's Session API, on the golden cases' inputs.  The gateway hands the
measured cell to the library as a pointer table."""
import glob
import os

import numpy as np
import pytest

from mset_b200 import Session
from oracle import refharness
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))
needs_gw = pytest.mark.skipif(not refharness.available(refharness.GATEWAY), reason="oracle/_gw not built")


def _drive(path, g, mode):
    r = refharness.RefSession(path)
    kw = dict(sigma=float(g["sigma"]), dz=float(g["dz"]), scan_x=g["sx"], scan_y=g["sy"], measured=g["meas"],
              binning=int(g["b"]))
    r.upload(g["V"], g["probe"], g["prop"], step=g["step"], **kw)
    out = r.run(mode)
    r.upload(g["V"], g["probe"], g["prop"], **kw)
    return out, r.error(mode)


@needs_gw
@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
@pytest.mark.parametrize("mode,tag", [(1, "mset"), (2, "sset")])
def test_gateway_matches_session_and_reference_mex(gpu_available, path, mode, tag):
    g = np.load(path)
    V, probe, sx0, sy0 = g["V"], g["probe"], g["sx"], g["sy"]
    (rv, pr, sx, sy, err), e_only = _drive(refharness.GATEWAY, g, mode)
    # the same library through its own API
    with Session() as s:
        kw = dict(sigma=float(g["sigma"]), potential_pixelsize=float(g["dz"]), scan_x=sx0, scan_y=sy0,
                  measured=g["meas"], slice_binning=int(g["b"]))
        s.upload(V, probe, g["prop"], step_size=g["step"], **kw)
        rv_s, pr_s, sx_s, sy_s, err_s = s.run(mode)
        s.upload(V, probe, g["prop"], **kw)
        e_s = s.error(mode)
    assert rel_l2(rv - V, rv_s - V) < 1e-6
    assert rel_l2(pr - probe, pr_s - probe) < 1e-6
    assert rel_l2(np.r_[sx - sx0, sy - sy0], np.r_[sx_s - sx0, sy_s - sy0]) < 1e-6
    assert abs(err - err_s) <= 1e-6 * err_s and abs(e_only - e_s) <= 1e-6 * e_s
    # the reference's stored outputs of the same call sequence (its own MEX module)
    assert rel_l2(rv - V, g[f"{tag}_rvol"] - V) < 1e-4
    assert rel_l2(pr - probe, g[f"{tag}_probe"] - probe) < 1e-4
    assert rel_l2(np.r_[sx - sx0, sy - sy0], np.r_[g[f"{tag}_sx"] - sx0, g[f"{tag}_sy"] - sy0]) < 1e-4
    assert abs(err - float(g[f"{tag}_err"])) <= 1e-4 * float(g[f"{tag}_err"])
    assert abs(e_only - float(g[f"{tag}_error_only"])) <= 1e-4 * float(g[f"{tag}_error_only"])
    if refharness.available():
        (rv_r, pr_r, _, _, err_r), e_r = _drive(refharness.LIB, g, mode)
        assert rel_l2(rv - V, rv_r - V) < 1e-4
        assert abs(e_only - e_r) <= 1e-4 * e_r


@needs_gw
def test_gateway_rejects_an_unknown_mode_as_the_reference_does(gpu_available):
    """mexErrMsgTxt with the reference's message (mex_main.cu:36-37)"""
    L = refharness.lib(refharness.GATEWAY)
    assert L.ref_mode(b"run_xset") == -1
    msg = L.ref_last_error()
    assert msg.startswith(b"The running mode is not correct (choose 'upload' or 'run_mset'")
    if refharness.available():
        R = refharness.lib(refharness.LIB)
        assert R.ref_mode(b"run_xset") == -1
        assert R.ref_last_error() == msg
