"""Pin the FP64 oracle to the reference's own implementation: golden vectors
in tests/golden/ref_*.npz were produced by the reference's CUDA MEX code
(src/CUDA/mset.cu, compiled unchanged, run on a B200 by
tests/golden/make_golden.py).  The oracle must reproduce the reference's
run_mset / run_sset updates and error_mset / error_sset values.

Tolerance: the reference computes in FP32 with cuFFT, the oracle in FP64, so
the changes it makes agree to ~1e-5 relative L2; 1e-4 is asserted.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_*.npz")))


def test_golden_vectors_exist():
    assert GOLD, "tests/golden/ref_*.npz missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
@pytest.mark.parametrize("mode,tag", [(1, "mset"), (2, "sset")])
def test_oracle_reproduces_reference(path, mode, tag):
    g = np.load(path)
    V, probe, sx0, sy0 = g["V"], g["probe"], g["sx"], g["sy"]
    rv, pr, sx, sy, err = O.run_tilt(V, probe, g["prop"], sx0, sy0, g["meas"], sigma=float(g["sigma"]),
                                     dz=float(g["dz"]), step=g["step"].astype(np.float64), binning=int(g["b"]),
                                     method=mode)
    n2 = V.shape[1] ** 2
    npos = sx0.size
    assert rel_l2(rv - V, g[f"{tag}_rvol"] - V) < 1e-4
    assert rel_l2(pr - probe, g[f"{tag}_probe"] - probe) < 1e-4
    assert rel_l2(np.r_[sx - sx0, sy - sy0], np.r_[g[f"{tag}_sx"] - sx0, g[f"{tag}_sy"] - sy0]) < 1e-4
    assert abs(err / npos / n2 - float(g[f"{tag}_err"])) <= 1e-4 * float(g[f"{tag}_err"])
    _, _, _, _, e2 = O.run_tilt(V, probe, g["prop"], sx0, sy0, g["meas"], sigma=float(g["sigma"]),
                                dz=float(g["dz"]), binning=int(g["b"]), method=mode, update=False)
    assert abs(e2 / npos / n2 - float(g[f"{tag}_error_only"])) <= 1e-4 * float(g[f"{tag}_error_only"])
