"""The per-position steps of the reference's CPU path (mset_forward_position /
mset_adjoint_position): STEP02_FORWARD_4D(_SSET) and STEP03_BACK(_SSET) for one
position (src/STEP02_FORWARD_4D.m:6-51, src/STEP03_BACK.m:6-39), checked
against the FP64 oracle of the same position (relative L2 <= 1e-4; the
scan-position step is cancellation-limited as in the sequential tests), and a
loop of STEP02 -> STEP03 -> STEP04 over every position against the fused
sequential pass (mset_run), which applies the same updates in one launch.

Spectra come back centred (fftshift of the oracle's standard order); real-space
arrays (waves, shifted probe, gradient) are the oracle's as they are.
"""
import numpy as np
import pytest

import mset_b200
from mset_b200 import MSET_ADJOINT_EXACT, MSET_ADJOINT_REF, MSET_MODE_MSET, MSET_MODE_SSET, Session
from tests.helpers import reasonable_steps, rel_l2, small_case
from tests.test_gpu_parity import STRENGTH, TOL, coord_tol

pytestmark = pytest.mark.gpu

CASES = [dict(n=24, nz=6, b=2), dict(n=64, nz=5, b=1), dict(n=128, nz=4, b=2), dict(n=256, nz=3, b=1)]
MODES = [(MSET_MODE_MSET, MSET_ADJOINT_REF), (MSET_MODE_MSET, MSET_ADJOINT_EXACT),
         (MSET_MODE_SSET, MSET_ADJOINT_REF)]


def _case(n, nz, b, npos=3, seed=0):
    return small_case(n=n, nz=nz, npos=npos, b=b, seed=seed + n + nz, defocus=20.0, jitter=4.0, strength=STRENGTH)


def _upload(s, c, step, npos):
    s.upload(c["V"], c["probe"], c["prop"], sigma=c["sigma"], potential_pixelsize=c["dz"], scan_x=c["sx"],
             scan_y=c["sy"], measured=c["meas"], step_size=step, slice_binning=c["b"], n_scan_x=npos, n_scan_y=1)


@pytest.mark.parametrize("method,admode", MODES, ids=["mset-ref", "mset-exact", "sset-ref"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c['n']}z{c['nz']}b{c['b']}")
def test_one_position_matches_oracle(gpu_available, case, method, admode):
    from oracle import oracle as O
    n, npos, k = case["n"], 3, 1
    c = _case(case["n"], case["nz"], case["b"], npos)
    step = reasonable_steps(c, method, admode)
    row, col = float(c["sx"][k]), float(c["sy"][k])
    o = O.position(c["V"], c["probe"], c["prop"], row, col, O.amp_std(c["meas"][k]), sigma=c["sigma"],
                   dz=c["dz"], binning=c["b"], method=method, adjoint=admode)
    with Session() as s:
        _upload(s, c, step, npos)
        f = s.step02(k, row, col, mode=method)
        g = s.step03(mode=method, adjoint=admode)
    # STEP02: |Psi|^2 and residual (centred), waves, shifted probe, error term
    far = o["far"]
    amp = O.amp_std(c["meas"][k])
    resi = far * (1.0 - amp / np.sqrt(np.abs(far) ** 2 + 1e-30))
    assert rel_l2(f["calc"], np.fft.fftshift(np.abs(far) ** 2)) < TOL
    assert rel_l2(f["resi"], np.fft.fftshift(resi)) < TOL
    assert rel_l2(f["psi0"], o["psi0"]) < TOL
    want_waves = o["waves"][:1] if method == MSET_MODE_SSET else o["waves"][1:]
    assert f["waves"].shape == want_waves.shape
    assert rel_l2(f["waves"], want_waves) < TOL
    assert abs(f["err"] - o["err"] / n ** 2 / npos) <= TOL * o["err"] / n ** 2 / npos
    # STEP03: complex gradient on every voxel of its slab, probe and scan steps
    nz = case["nz"]
    b = nz if method == MSET_MODE_SSET else case["b"]
    slab = np.minimum(np.arange(nz) // b, o["grad"].shape[0] - 1)
    assert rel_l2(g["grad"], o["grad"][slab]) < TOL
    assert rel_l2(g["probe"] - c["probe"], -step[1] * o["probe_dir"]) < TOL
    d = np.array([g["row"] - row, g["col"] - col])
    assert rel_l2(d, step[2] * o["pos_dir"]) < coord_tol(n, [row, col], step[2] * o["pos_dir"])


@pytest.mark.parametrize("method", [MSET_MODE_MSET, MSET_MODE_SSET], ids=["mset", "sset"])
def test_step_loop_equals_sequential_run(gpu_available, method):
    """STEP02 -> STEP03 -> STEP04 for every position in order, each starting at
    the scan coordinates and state the previous ones left (Run_MSET_recon.m:
    136-157), gives what the fused sequential pass gives"""
    npos = 5
    c = _case(64, 6, 2, npos, seed=7)
    step = reasonable_steps(c, method)
    with Session() as s:
        _upload(s, c, step, npos)
        rv, pr, sx, sy, err = s.run(method)
    V = c["V"].astype(np.float32).copy()
    rows, cols = c["sx"].astype(np.float32).copy(), c["sy"].astype(np.float32).copy()
    e = 0.0
    with Session() as s:
        _upload(s, c, step, npos)
        for k in range(npos):
            f = s.step02(k, rows[k], cols[k], mode=method)
            g = s.step03(mode=method, update_rvol=True)
            V += np.float32(step[0]) * g["grad"].real.astype(np.float32)
            rows[k], cols[k] = g["row"], g["col"]
            e += f["err"]
        probe = g["probe"]
        # the volume and probe the device holds after the loop
        rv_dev, pr_dev = s.read_state()
    assert rel_l2(rv_dev - c["V"], rv - c["V"]) < 1e-5
    assert rel_l2(pr_dev, probe) < 1e-6
    assert rel_l2(V - c["V"], rv - c["V"]) < 1e-5
    assert rel_l2(probe - c["probe"], pr - c["probe"]) < 1e-5
    assert rel_l2(np.r_[rows - c["sx"], cols - c["sy"]], np.r_[sx - c["sx"], sy - c["sy"]]) < 1e-5
    assert abs(e - err) <= 1e-5 * err


def test_adjoint_of_a_given_residual(gpu_available):
    """resi_in replaces the forward's residual: handing back the forward's own
    centred residual gives the same step; a scaled residual scales the
    gradient (the adjoint is linear in it)"""
    npos, k = 3, 2
    c = _case(96, 4, 1, npos, seed=3)
    step = reasonable_steps(c, MSET_MODE_MSET)
    with Session() as s:
        _upload(s, c, step, npos)
        f = s.step02(k, c["sx"][k], c["sy"][k])
        g0 = s.step03()
    with Session() as s:
        _upload(s, c, step, npos)
        s.step02(k, c["sx"][k], c["sy"][k])
        g1 = s.step03(resi=f["resi"])
    with Session() as s:
        _upload(s, c, step, npos)
        s.step02(k, c["sx"][k], c["sy"][k])
        g2 = s.step03(resi=2.0 * f["resi"])
    assert np.array_equal(g0["grad"], g1["grad"])
    assert np.array_equal(g0["probe"], g1["probe"])
    assert (g0["row"], g0["col"]) == (g1["row"], g1["col"])
    assert rel_l2(g2["grad"], 2.0 * g0["grad"]) < 1e-6


def test_step_errors(gpu_available):
    c = _case(24, 3, 1, 2)
    with Session() as s:
        with pytest.raises(mset_b200.MsetError, match="before upload"):
            s.step02(0, 12.0, 12.0)
        _upload(s, c, (0.0, 0.0, 0.0), 2)
        with pytest.raises(mset_b200.MsetError, match="preceding forward_position"):
            s.step03()
        with pytest.raises(mset_b200.MsetError, match="out of range"):
            s.step02(2, 12.0, 12.0)
        with pytest.raises(mset_b200.MsetError, match="non-finite"):
            s.step02(0, float("nan"), 12.0)
        s.step02(0, 12.0, 12.0, mode=MSET_MODE_SSET)
        with pytest.raises(mset_b200.MsetError, match="same mode"):
            s.step03(mode=MSET_MODE_MSET)
        s.step02(0, 12.0, 12.0)
        s.step03()
        with pytest.raises(mset_b200.MsetError, match="preceding forward_position"):
            s.step03()  # a forward is consumed by one adjoint
        # a sequential pass between STEP02 and STEP03 overwrites the saved
        # waves and the volume / probe / positions the forward used
        s.step02(0, 12.0, 12.0)
        s.run(MSET_MODE_MSET)
        with pytest.raises(mset_b200.MsetError, match="preceding forward_position") as ei:
            s.step03()
        assert ei.value.code == mset_b200.MSET_E_STATE


def test_per_position_backend_equals_fused_backend(gpu_available):
    """recon.LibraryBackend(per_position=True), the CPU device modes' loop of
    Run_MSET_recon.m:136-157 on the per-position entry points, updates a tilt
    as the fused sequential pass does"""
    from mset_b200 import recon
    npos = 4
    c = _case(64, 6, 2, npos, seed=11)
    step = reasonable_steps(c, MSET_MODE_MSET)
    t = recon.Tilt(c["probe"], c["sx"], c["sy"], c["meas"], (npos, 1))
    kw = dict(sigma=c["sigma"], dz=c["dz"], step=step, binning=c["b"], method=MSET_MODE_MSET)
    outs = []
    for per_position in (False, True):
        be = recon.LibraryBackend(per_position=per_position)
        outs.append(be.run_tilt(c["V"], t, c["prop"], **kw))
        be.close()
    (rv0, pr0, sx0, sy0), (rv1, pr1, sx1, sy1) = outs
    assert rel_l2(rv1 - c["V"], rv0 - c["V"]) < 1e-5
    assert rel_l2(pr1 - c["probe"], pr0 - c["probe"]) < 1e-5
    assert rel_l2(np.r_[sx1 - c["sx"], sy1 - c["sy"]], np.r_[sx0 - c["sx"], sy0 - c["sy"]]) < 1e-5
