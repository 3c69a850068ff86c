"""Generate golden vectors from the reference's own CUDA implementation.

Runs oracle/_ref/libmset_ref.so -- the reference's src/CUDA/mex_main.cu,
mset.cu and utility.cu compiled unchanged (`make -C oracle ref`) behind the
project's mex shim -- on seeded inputs and stores inputs and outputs as
tests/golden/ref_<case>.npz.  Needs a CUDA GPU (the reference uses cuFFT).

    python tests/golden/make_golden.py [outdir]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refharness import RefSession  # noqa: E402
from tests.helpers import reasonable_steps, small_case  # noqa: E402

CASES = {
    # the reference example's window (24x24) with MSET slices
    "n24_z6_b1": dict(n=24, nz=6, npos=6, b=1, seed=101, defocus=20.0, jitter=4.0),
    "n24_z7_b2": dict(n=24, nz=7, npos=5, b=2, seed=102, defocus=0.0, jitter=3.0),
    "n64_z4_b1": dict(n=64, nz=4, npos=4, b=1, seed=103, defocus=40.0, jitter=6.0),
}


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, k in CASES.items():
        c = small_case(n=k["n"], nz=k["nz"], npos=k["npos"], b=k["b"], seed=k["seed"], defocus=k["defocus"],
                       jitter=k["jitter"])
        k["steps"] = reasonable_steps(c)
        out = dict(V=c["V"], probe=c["probe"], prop=c["prop"], sx=c["sx"], sy=c["sy"], meas=c["meas"],
                   sigma=c["sigma"], dz=c["dz"], b=k["b"], step=np.array(k["steps"], np.float32))
        for mode, tag in ((1, "mset"), (2, "sset")):
            r = RefSession()
            r.upload(c["V"], c["probe"], c["prop"], sigma=c["sigma"], dz=c["dz"], scan_x=c["sx"], scan_y=c["sy"],
                     measured=c["meas"], step=k["steps"], binning=k["b"])
            rv, pr, sx, sy, err = r.run(mode)
            out.update({f"{tag}_rvol": rv, f"{tag}_probe": pr, f"{tag}_sx": sx, f"{tag}_sy": sy,
                        f"{tag}_err": np.float32(err)})
            r = RefSession()
            r.upload(c["V"], c["probe"], c["prop"], sigma=c["sigma"], dz=c["dz"], scan_x=c["sx"], scan_y=c["sy"],
                     measured=c["meas"], step=k["steps"], binning=k["b"])
            out[f"{tag}_error_only"] = np.float32(r.error(mode))
        np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
