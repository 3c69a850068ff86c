"""The library against the reference's own CUDA implementation run on the
same GPU (oracle/_ref/libmset_ref.so, the reference's src/CUDA code compiled
unchanged), on the golden cases' inputs.  Tolerance 1e-4 relative L2 on the
changes a run_mset / run_sset pass makes."""
import glob
import os

import numpy as np
import pytest

from mset_b200 import Session
from oracle import refharness
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
@pytest.mark.parametrize("mode,tag", [(1, "mset"), (2, "sset")])
def test_library_matches_reference_cuda(gpu_available, path, mode, tag):
    g = np.load(path)
    V, probe, sx0, sy0 = g["V"], g["probe"], g["sx"], g["sy"]
    n = V.shape[1]
    if n not in (24, 32, 48, 64, 96, 128, 160):
        pytest.skip("window without a compiled kernel")
    with Session() as s:
        s.upload(V, probe, g["prop"], sigma=float(g["sigma"]), potential_pixelsize=float(g["dz"]), scan_x=sx0,
                 scan_y=sy0, measured=g["meas"], step_size=g["step"], slice_binning=int(g["b"]))
        rv, pr, sx, sy, err = s.run(mode)
        s.upload(V, probe, g["prop"], sigma=float(g["sigma"]), potential_pixelsize=float(g["dz"]), scan_x=sx0,
                 scan_y=sy0, measured=g["meas"], step_size=g["step"], slice_binning=int(g["b"]))
        e_only = s.error(mode)
    assert rel_l2(rv - V, g[f"{tag}_rvol"] - V) < 1e-4
    assert rel_l2(pr - probe, g[f"{tag}_probe"] - probe) < 1e-4
    assert rel_l2(np.r_[sx - sx0, sy - sy0], np.r_[g[f"{tag}_sx"] - sx0, g[f"{tag}_sy"] - sy0]) < 1e-4
    assert abs(err - float(g[f"{tag}_err"])) <= 1e-4 * float(g[f"{tag}_err"])
    assert abs(e_only - float(g[f"{tag}_error_only"])) <= 1e-4 * float(g[f"{tag}_error_only"])


@pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built")
def test_reference_harness_runs_live(gpu_available):
    """the live reference build reproduces its committed golden vectors"""
    g = np.load(GOLD[0])
    r = refharness.RefSession()
    r.upload(g["V"], g["probe"], g["prop"], sigma=float(g["sigma"]), dz=float(g["dz"]), scan_x=g["sx"],
             scan_y=g["sy"], measured=g["meas"], step=g["step"], binning=int(g["b"]))
    rv, pr, sx, sy, err = r.run(1)
    assert rel_l2(rv - g["V"], g["mset_rvol"] - g["V"]) < 1e-5
