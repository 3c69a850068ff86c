"""Fixture from the reference's own example dataset and stored reconstruction.

The reference ships examples/CuAu_24size_dataset: eight v7.3 MAT-files of
4D-STEM patterns (24x24 window, 24x24 scan, tilts -70..52.5 deg), and
MSET_recon.mat, the STEM_data state its reconstruction (MATLAB STEP02/STEP03
path) ended with.  That state holds, for the last tilt (52.5 deg):

  rec          the final reconstruction (24^3)
  RVol         single(Func_inv_rot(rec, tilt 8)): STEP01 of the last error pass
  init_wave2D  the probe of tilt 8
  tmp_probe_wfn  the probe shifted to the last scan position (24, 24)
  save_wave_f  the waves after every slice for that position
  error        per-tilt errors of the final state (mean over positions of
               mean((sqrt(I) - |Psi|)^2), STEP02_FORWARD_4D.m:47-48)

This script reads them with mset_b200.matfile and stores tilt 8's inputs and
those outputs as tests/golden/example_tilt8.npz (C views of the MATLAB arrays:
volumes [z][y][x], 2D arrays transposed).

    python tests/golden/make_example_fixture.py <reference-root> [outfile]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mset_b200.matfile import loadmat73  # noqa: E402
from mset_b200.recon import load_example  # noqa: E402


def main(ref_root, out):
    d = os.path.join(ref_root, "examples", "CuAu_24size_dataset")
    S = loadmat73(os.path.join(d, "MSET_recon.mat"), names=["STEM_data"])["STEM_data"]
    ex = load_example(d, probe_from=os.path.join(d, "MSET_recon.mat"))
    t = ex["tilts"][7]
    c = lambda a: np.ascontiguousarray(a)  # noqa: E731
    np.savez_compressed(
        out,
        rec=c(S["rec"].transpose(2, 1, 0).astype(np.float32)),
        RVol=c(S["RVol"].transpose(2, 1, 0).astype(np.float32)),
        probe=c(t.probe),
        scan_x=t.scan_x, scan_y=t.scan_y,
        measured=t.measured,
        prop=c(S["prop2D"].T.astype(np.complex64)),
        angles=ex["angles"][7],
        sigma=float(S["sigma"].ravel()[0]), dz=float(S["potential_pixelsize"].ravel()[0]),
        error=float(S["error"].ravel()[7]),
        tmp_probe=c(S["tmp_probe_wfn"].T.astype(np.complex64)),
        exit_wave=c(S["save_wave_f"][:, :, -1].T.astype(np.complex64)),
    )


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(__file__),
                                                                          "example_tilt8.npz"))
