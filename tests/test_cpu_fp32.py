"""The single-precision CPU port (oracle/cpu_fp32.c), the timed CPU baseline,
against the FP64 oracle on the same inputs: it computes what the batched pass
computes, to single-precision accuracy (relative L2 <= 2e-4 for the volume
gradient, probe direction and error; the scan-position directions, sums with
cancellation, to 5e-3)."""
import numpy as np

from oracle import oracle as O
from tests.helpers import rel_l2, small_case


def test_fp32_port_matches_fp64_oracle():
    c = small_case(n=64, nz=6, npos=5, b=2, seed=5, defocus=15.0, jitter=5.0, strength=20.0)
    kw = dict(sigma=c["sigma"], dz=c["dz"], binning=2)
    g, pa, pd, e = O.batched_tilt(c["V"], c["probe"], c["prop"], c["sx"], c["sy"], c["meas"], **kw)
    g32, pa32, pd32, e32 = O.batched_tilt_fp32(c["V"], c["probe"], c["prop"], c["sx"], c["sy"], c["meas"], **kw)
    assert rel_l2(g32, g) < 2e-4
    assert rel_l2(pa32, pa) < 2e-4
    assert abs(e32 - e) <= 2e-4 * e
    assert rel_l2(pd32, pd) < 5e-3


def test_fp32_port_rejects_non_power_of_two_windows():
    c = small_case(n=24, nz=2, npos=1)
    try:
        O.batched_tilt_fp32(c["V"], c["probe"], c["prop"], c["sx"], c["sy"], c["meas"], sigma=c["sigma"], dz=c["dz"])
    except ValueError as ex:
        assert "power of two" in str(ex)
    else:
        raise AssertionError("expected a ValueError")


def test_fp32_simulation_matches_fp64_far_field():
    c = small_case(n=64, nz=5, npos=3, b=1, seed=9, defocus=30.0, jitter=8.0)
    I32 = O.simulate_fp32(c["V"], c["probe"], c["prop"], c["sx"], c["sy"], sigma=c["sigma"], dz=c["dz"])
    for p in range(3):
        o = O.position(c["V"], c["probe"], c["prop"], c["sx"][p], c["sy"][p], O.amp_std(c["meas"][p]),
                       sigma=c["sigma"], dz=c["dz"])
        assert rel_l2(I32[p], np.fft.fftshift(np.abs(o["far"]) ** 2)) < 1e-4


def test_fp32_sequential_port_matches_fp64_sequential_pass():
    """The one-thread reference-semantics port (cpu32_sequential_tilt, the
    timed sequential CPU baseline) against the FP64 oracle's run_tilt: each
    position updates the volume, probe and its coordinates before the next
    starts (run_main_mset), so both carry the same chain of updates"""
    from tests.helpers import reasonable_steps
    c = small_case(n=64, nz=6, npos=5, b=2, seed=7, defocus=15.0, jitter=5.0, strength=20.0)
    step = reasonable_steps(c)
    kw = dict(sigma=c["sigma"], dz=c["dz"], step=step, binning=2)
    rv, pr, sx, sy, e = O.run_tilt(c["V"], c["probe"], c["prop"], c["sx"], c["sy"], c["meas"], **kw)
    rv32, pr32, sx32, sy32, e32 = O.sequential_tilt_fp32(c["V"], c["probe"], c["prop"], c["sx"], c["sy"],
                                                         c["meas"], **kw)
    assert rel_l2(rv32 - c["V"], rv - c["V"]) < 2e-4
    assert rel_l2(pr32 - c["probe"], pr - c["probe"]) < 2e-4
    assert abs(e32 - e) <= 2e-4 * e
    d, d32 = np.r_[sx - c["sx"], sy - c["sy"]], np.r_[sx32 - c["sx"], sy32 - c["sy"]]
    assert rel_l2(d32, d) < 5e-3
