"""The reference's own example dataset and stored reconstruction
(examples/CuAu_24size_dataset, read with mset_b200.matfile).

tests/golden/example_tilt8.npz (made by tests/golden/make_example_fixture.py)
holds, for the last tilt, the reference's final reconstruction, the rotated
volume its last error pass used, the probe, the 576 measured patterns and
what the reference computed from them: the per-tilt error, the shifted probe
and the exit wave of the last scan position.  The oracle (CPU) and the library
(GPU) must reproduce those numbers, relative error <= 1e-4 (FP32 state; the
reference ran in single precision).

The stored reconstruction trajectory itself (MSET_recon.mat, rec_save and
mean_error per iteration) is not asserted.  It starts from rec = 0, where the
model predicts no intensity outside the probe aperture: the amplitude
residual Psi (1 - M/A) there has magnitude M and the phase of Psi, which is
rounding noise, so the first updates depend on the arithmetic (an FP32
restatement of STEP02/STEP03 differs from FP64 by 64% on the first
position's gradient).  The reference ran in single precision; replaying its
loop (mset_b200.recon.reconstruct) with the FP64 oracle gives mean errors
within 1-4% of the stored ones, and the library (FP32) within 0.5% of the
oracle.
"""
import os

import numpy as np
import pytest

from tests.helpers import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "example_tilt8.npz")
# the reference checkout (for the raw .mat files), named by MSET_REFERENCE_ROOT
_ROOT = os.environ.get("MSET_REFERENCE_ROOT", "")
REF = os.path.join(_ROOT, "examples", "CuAu_24size_dataset") if _ROOT else ""
TOL = 1e-4


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(FIX))


def _error_oracle(V, f):
    from oracle import oracle as O
    _, _, _, _, e = O.run_tilt(V, f["probe"], f["prop"], f["scan_x"], f["scan_y"], f["measured"],
                               sigma=float(f["sigma"]), dz=float(f["dz"]), update=False)
    P, n = f["measured"].shape[0], f["measured"].shape[1]
    return e / P / n / n  # STEP02_FORWARD_4D.m:47-48


# ---- oracle (CPU) --------------------------------------------------------------
def test_oracle_error_pass_reproduces_reference(fx):
    assert abs(_error_oracle(fx["RVol"], fx) - fx["error"]) <= TOL * fx["error"]


def test_oracle_rotation_reproduces_reference(fx):
    from oracle import oracle as O
    assert rel_l2(O.rot3d(fx["rec"], fx["angles"], inverse=True), fx["RVol"]) < 1e-5


def test_oracle_probe_shift_and_exit_wave_reproduce_reference(fx):
    from oracle import oracle as O
    o = O.position(fx["RVol"], fx["probe"], fx["prop"], fx["scan_x"][-1], fx["scan_y"][-1],
                   O.amp_std(fx["measured"][-1]), sigma=float(fx["sigma"]), dz=float(fx["dz"]))
    assert rel_l2(o["psi0"], fx["tmp_probe"]) < 1e-5
    assert rel_l2(np.fft.ifft2(o["far"]), fx["exit_wave"]) < 1e-5


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="MSET_REFERENCE_ROOT does not name the reference checkout")
def test_matfile_reader_and_all_tilt_errors():
    """reader on every file of the example; the oracle's error pass of the
    stored final reconstruction against the stored errors of all 8 tilts"""
    from mset_b200 import physics
    from mset_b200.matfile import loadmat73
    from mset_b200.recon import load_example
    from oracle import oracle as O

    ref = loadmat73(os.path.join(REF, "MSET_recon.mat"))
    S = ref["STEM_data"]
    assert ref["rec_save"].shape == (24, 24, 24, 5)
    assert S["probe_wfn"].shape == (24, 24, 8) and S["probe_wfn"].dtype == np.complex64
    info = loadmat73(os.path.join(REF, "CuAu_s24_p72_Np_8_STEM_data_info.mat"))["STEM_data"]
    assert info["pot3D"].shape == (24, 24, 24)
    ex = load_example(REF, probe_from=os.path.join(REF, "MSET_recon.mat"))
    assert len(ex["tilts"]) == 8 and ex["tilts"][0].measured.shape == (576, 24, 24)
    rec = S["rec"].transpose(2, 1, 0)
    lam = physics.electron_wavelength(300e3)
    prop = physics.propagator(24, 0.4, lam, 1)
    assert rel_l2(prop, S["prop2D"].T) < 1e-7
    sigma = physics.interaction_constant(300e3)
    for j, t in enumerate(ex["tilts"]):
        V = O.rot3d(rec, ex["angles"][j], inverse=True).astype(np.float32)
        _, _, _, _, e = O.run_tilt(V, t.probe, prop, t.scan_x, t.scan_y, t.measured, sigma=sigma, dz=0.4,
                                   update=False)
        stored = float(S["error"].ravel()[j])
        assert abs(e / 576 / 576 - stored) <= TOL * stored, j


# ---- library (GPU) ---------------------------------------------------------------
@pytest.mark.gpu
def test_library_error_pass_reproduces_reference(gpu_available, fx):
    from mset_b200 import Session
    with Session() as s:
        s.upload(fx["RVol"], fx["probe"], fx["prop"], sigma=float(fx["sigma"]), potential_pixelsize=float(fx["dz"]),
                 scan_x=fx["scan_x"], scan_y=fx["scan_y"], measured=fx["measured"], n_scan_x=24, n_scan_y=24)
        e = s.error()
    assert abs(e - fx["error"]) <= TOL * fx["error"]


@pytest.mark.gpu
def test_library_batched_error_and_rotation_reproduce_reference(gpu_available, fx):
    from mset_b200 import Session
    from mset_b200.batch import BatchSession
    with Session() as s:
        V = s.rotate_volume(fx["rec"], fx["angles"], inverse=True)
    assert rel_l2(V, fx["RVol"]) < TOL
    bs = BatchSession(n=24, nz=24, npos=[576], prop=fx["prop"], sigma=float(fx["sigma"]),
                      potential_pixelsize=float(fx["dz"]))
    bs.set_tilt(0, probe=fx["probe"], scan_x=fx["scan_x"], scan_y=fx["scan_y"], measured=fx["measured"],
                volume=V)
    e = bs.error()[0] / 576 / 576
    bs.close()
    assert abs(e - fx["error"]) <= TOL * fx["error"]
