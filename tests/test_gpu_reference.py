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


@pytest.fixture(scope="module")
def small_series(gpu_available):
    """The small configuration (24^3 volume at 0.4 A in a 64^2 window, 24
    slices of 1 voxel, 12x12 scan at 2 px, 5 tilts over +-30 deg): per tilt
    the beam-frame volume at half the true potential and seeded Poisson
    counts of the library's forward model at the truth."""
    from mset_b200 import synth
    from mset_b200.batch import BatchSession
    cfg = synth.CONFIGS["small"]
    spec = synth.make_specimen(cfg)
    n, k = cfg.window, spec.scan_x.size
    tilts = []
    for j, vt in enumerate(spec.volumes):
        bs = BatchSession(n=n, nz=vt.shape[0], npos=[k], prop=spec.prop, sigma=spec.sigma,
                          potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning)
        bs.set_tilt(0, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y,
                    measured=np.zeros((k, n, n), np.float32), volume=vt)
        meas = synth.poisson(bs.simulate(), cfg.seed + 1000 + j)
        bs.close()
        tilts.append(dict(V=(0.5 * vt).astype(np.float32), meas=meas))
    return cfg, spec, tilts


@pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built")
def test_small_config_all_tilts_match_reference_cuda(small_series):
    """run_mset and error_mset of every tilt of the small configuration (144
    positions, 24 slices, sequential per-position updates) through this
    library, through the reference's own CUDA module and through the FP64
    oracle, on the same inputs.  Both FP32 implementations are compared with
    FP64: this library's volume / probe changes and errors to 1e-4, its scan
    position changes to the cancellation bound of 64^2 windows (3e-4).  The
    reference itself deviates from FP64 by ~1.4e-4 on the volume change
    (measured on one B200: 1.4e-4 against this library's 2e-5), so library
    and reference agree to the sum of their deviations, which is asserted
    too: the two implementations differ by no more than the reference's own
    rounding."""
    from oracle import oracle as O
    from tests.helpers import reasonable_steps
    cfg, spec, tilts = small_series
    nsx, nsy = cfg.scan
    n2 = cfg.window ** 2
    for j, t in enumerate(tilts):
        c = dict(V=t["V"], probe=spec.probe, prop=spec.prop, sx=spec.scan_x, sy=spec.scan_y, meas=t["meas"],
                 sigma=spec.sigma, dz=cfg.dx, b=cfg.slice_binning)
        step = reasonable_steps(c, 1, 0, frac=(0.01, 0.002, 0.02))
        kw = dict(sigma=spec.sigma, scan_x=spec.scan_x, scan_y=spec.scan_y, measured=t["meas"])
        with Session() as s:
            s.upload(t["V"], spec.probe, spec.prop, potential_pixelsize=cfg.dx, step_size=step,
                     slice_binning=cfg.slice_binning, n_scan_x=nsx, n_scan_y=nsy, **kw)
            lib = s.run(1)
            s.upload(t["V"], spec.probe, spec.prop, potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning,
                     n_scan_x=nsx, n_scan_y=nsy, **kw)
            lib_e = s.error(1)
        r = refharness.RefSession()
        r.upload(t["V"], spec.probe, spec.prop, dz=cfg.dx, step=step, binning=cfg.slice_binning, nsx=nsx, nsy=nsy,
                 **kw)
        ref = r.run(1)
        r.upload(t["V"], spec.probe, spec.prop, dz=cfg.dx, binning=cfg.slice_binning, nsx=nsx, nsy=nsy, **kw)
        ref_e = r.error(1)
        rv_o, pr_o, sx_o, sy_o, err_o = O.run_tilt(t["V"], spec.probe, spec.prop, spec.scan_x, spec.scan_y,
                                                   t["meas"], sigma=spec.sigma, dz=cfg.dx, step=step,
                                                   binning=cfg.slice_binning)
        _, _, _, _, erro_o = O.run_tilt(t["V"], spec.probe, spec.prop, spec.scan_x, spec.scan_y, t["meas"],
                                        sigma=spec.sigma, dz=cfg.dx, binning=cfg.slice_binning, update=False)
        oracle = (rv_o, pr_o, sx_o, sy_o, err_o / (nsx * nsy) / n2)
        oracle_e = erro_o / (nsx * nsy) / n2

        def dev(a, b, e_a, e_b):
            return {"rvol": rel_l2(a[0] - t["V"], b[0] - t["V"]),
                    "probe": rel_l2(a[1] - spec.probe, b[1] - spec.probe),
                    "pos": rel_l2(np.r_[a[2] - spec.scan_x, a[3] - spec.scan_y],
                                  np.r_[b[2] - spec.scan_x, b[3] - spec.scan_y]),
                    "err": abs(a[4] - b[4]) / b[4], "error_only": abs(e_a - e_b) / e_b}
        lo, ro, lr = dev(lib, oracle, lib_e, oracle_e), dev(ref, oracle, ref_e, oracle_e), dev(lib, ref, lib_e, ref_e)
        print("tilt", j, "library-oracle", {q: f"{v:.1e}" for q, v in lo.items()},
              "reference-oracle", {q: f"{v:.1e}" for q, v in ro.items()})
        for q in ("rvol", "probe", "err", "error_only"):
            assert lo[q] < 1e-4, (j, q, lo[q])
        assert lo["pos"] < 3e-4, (j, lo["pos"])
        for q, v in lr.items():
            # |lib - ref| <= |lib - oracle| + |ref - oracle| (relative to the
            # oracle's change; 5% slack for the change of reference vector)
            assert v <= 1.05 * (lo[q] + ro[q]) + 1e-7, (j, q, v, lo[q], ro[q])
