"""The batched iteration (rotation -> pass -> rotation back -> update ->
positivity -> TV-FISTA, one CUDA graph) against its FP64 oracle
(tests/iteration_oracle.py), two iterations, with and without graph capture.
Tolerance: relative L2 1e-4 on the change of the volume, the probes, and the
errors; the scan positions at the cancellation-limited tolerance of the other
tests."""
import numpy as np
import pytest

from mset_b200 import physics
from mset_b200.batch import BatchSession
from oracle import oracle as O
from tests import iteration_oracle as IO
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _problem(seed=5):
    rng = np.random.default_rng(seed)
    nv, n, b, dz, E0 = 24, 32, 2, 0.4, 300e3
    lam = physics.electron_wavelength(E0)
    sigma = physics.interaction_constant(E0)
    z, y, x = np.meshgrid(*[np.arange(nv) - 12] * 3, indexing="ij")
    truth = np.zeros((nv,) * 3)
    for _ in range(12):
        p = rng.uniform(-7, 7, 3)
        truth += rng.uniform(20, 40) * np.exp(-((x - p[0]) ** 2 + (y - p[1]) ** 2 + (z - p[2]) ** 2) / 3.0)
    angles = [(0, -20, 0), (0, 0, 0), (0, 25, 0)]
    prop = physics.propagator(n, dz, lam, b)
    probe = physics.normalise_probe(physics.probe_wave(n, dz, lam, 20.0, C10=-20.0), 1e4).astype(np.complex64)
    c = np.floor((n + 1) / 2 + 0.5)
    tilts = []
    for j, a in enumerate(angles):
        sx = (c + rng.uniform(-5, 5, 4)).astype(np.float32)
        sy = (c + rng.uniform(-5, 5, 4)).astype(np.float32)
        Vt = IO.pad(O.rot3d(truth, a, inverse=True), n)
        meas = np.empty((4, n, n), np.float32)
        for p in range(4):
            o = O.position(Vt, probe, prop, sx[p] + 0.3, sy[p] - 0.2, np.zeros((n, n)), sigma=sigma, dz=dz, binning=b)
            meas[p] = rng.poisson(np.fft.fftshift(np.abs(o["far"]) ** 2))
        tilts.append(dict(probe=probe.copy(), sx=sx, sy=sy, meas=meas))
    rec0 = (0.6 * truth).astype(np.float32)
    return nv, n, b, dz, sigma, prop, angles, tilts, rec0


@pytest.mark.parametrize("use_graph", [True, False])
def test_iteration_matches_oracle(gpu_available, use_graph):
    nv, n, b, dz, sigma, prop, angles, tilts, rec0 = _problem()
    # step sizes from one oracle pass: ~5% volume change, ~1% probe change
    _, e0 = IO.iterate(rec0.astype(np.float64), [dict(t) for t in tilts], prop, angles, sigma=sigma, dz=dz,
                       binning=b, step=(0, 0, 0), positivity=False)
    V0 = IO.pad(O.rot3d(rec0, angles[1], inverse=True), n).astype(np.float32)
    g, pa, pd, _ = O.batched_tilt(V0, tilts[1]["probe"], prop, tilts[1]["sx"], tilts[1]["sy"], tilts[1]["meas"],
                                  sigma=sigma, dz=dz, binning=b)
    step = (0.05 * rec0.max() / np.abs(g).max(), 0.01 * np.abs(tilts[1]["probe"]).max() / np.abs(pa).max(),
            0.1 / np.abs(pd).max())
    kw = dict(positivity=True, tv_lambda=0.02, tv_iter=20, tv_fista=True)

    bs = BatchSession(n=n, nz=nv, npos=[4, 4, 4], prop=prop, sigma=sigma, potential_pixelsize=dz, slice_binning=b,
                      step_size=step)
    for j, t in enumerate(tilts):
        bs.set_tilt(j, probe=t["probe"], scan_x=t["sx"], scan_y=t["sy"], measured=t["meas"])
    bs.iteration_setup(nv, angles, positivity=True, tv_lambda=0.02, tv_iter=20, tv_fista=True)
    bs.set_rec(rec0)
    errs_g, _ = bs.iterate(2, use_graph=use_graph)
    rec_g = bs.get_rec()
    probes_g = [bs.get_tilt(j)[1] for j in range(3)]
    pos_g = [bs.get_tilt(j)[2:] for j in range(3)]
    bs.close()

    rec = rec0.astype(np.float64)
    tl = [dict(t) for t in tilts]
    errs_o = []
    for _ in range(2):
        rec, e = IO.iterate(rec, tl, prop, angles, sigma=sigma, dz=dz, binning=b, step=step, **kw)
        errs_o.append(e)
    assert rel_l2(rec_g - rec0, rec - rec0) < 1e-4
    for j in range(3):
        assert rel_l2(probes_g[j] - tilts[j]["probe"], tl[j]["probe"] - tilts[j]["probe"]) < 1e-4
        d_g = np.r_[pos_g[j][0] - tilts[j]["sx"], pos_g[j][1] - tilts[j]["sy"]]
        d_o = np.r_[tl[j]["sx"] - tilts[j]["sx"], tl[j]["sy"] - tilts[j]["sy"]]
        assert rel_l2(d_g, d_o) < 1e-4
    assert rel_l2(errs_g, np.array(errs_o)) < 1e-4


def test_phase_split_equals_full_iteration(gpu_available):
    """phase 1 + phase 2 (the tilt-sharding path, one rank) equals the fused
    iteration graph bit for bit in volume and probes"""
    from mset_b200.distributed import GpuBackend, sharded_iterate

    nv, n, b, dz, sigma, prop, angles, tilts, rec0 = _problem(seed=6)
    step = (1e-3, 1e-6, 1e-2)
    outs = []
    for mode in ("full", "phases"):
        bs = BatchSession(n=n, nz=nv, npos=[4, 4, 4], prop=prop, sigma=sigma, potential_pixelsize=dz,
                          slice_binning=b, step_size=step)
        for j, t in enumerate(tilts):
            bs.set_tilt(j, probe=t["probe"], scan_x=t["sx"], scan_y=t["sy"], measured=t["meas"])
        bs.iteration_setup(nv, angles, positivity=True, tv_lambda=0.02, tv_iter=10)
        bs.set_rec(rec0)
        if mode == "full":
            bs.iterate(2)
        else:
            sharded_iterate(GpuBackend(bs), 2, world=1)
        outs.append((bs.get_rec(), [bs.get_tilt(j)[1] for j in range(3)]))
        bs.close()
    # FP64 atomics make the gradient sums order-dependent at the last bit
    assert rel_l2(outs[1][0] - rec0, outs[0][0] - rec0) < 1e-6
    for a, c in zip(outs[0][1], outs[1][1]):
        assert rel_l2(a, c) < 1e-6


def test_line_search_matches_oracle(gpu_available):
    """the reference's backtracking line search (Run_MSET_recon.m:106-252) on
    the batched iteration: steps 4x too large, so the second iteration rejects
    two trials before it accepts; accepted errors, step sizes, volume, probes
    and positions against the FP64 oracle of the same rule"""
    nv, n, b, dz, sigma, prop, angles, tilts, rec0 = _problem()
    V0 = IO.pad(O.rot3d(rec0, angles[1], inverse=True), n).astype(np.float32)
    g, pa, pd, _ = O.batched_tilt(V0, tilts[1]["probe"], prop, tilts[1]["sx"], tilts[1]["sy"], tilts[1]["meas"],
                                  sigma=sigma, dz=dz, binning=b)
    step = 4.0 * np.array([0.05 * rec0.max() / np.abs(g).max(),
                           0.01 * np.abs(tilts[1]["probe"]).max() / np.abs(pa).max(), 0.1 / np.abs(pd).max()])
    step = step.astype(np.float32)
    rec_o, tl, e_o, st_o = IO.iterate_bls(rec0.astype(np.float64), [dict(t) for t in tilts], prop, angles,
                                          sigma=sigma, dz=dz, binning=b, step=step, bls=0.5, niter=4,
                                          tv_lambda=0.02, tv_iter=20)
    assert len(e_o) == 4 and st_o[-1][0] < step[0]  # the rule did reject

    bs = BatchSession(n=n, nz=nv, npos=[4, 4, 4], prop=prop, sigma=sigma, potential_pixelsize=dz, slice_binning=b,
                      step_size=step)
    for j, t in enumerate(tilts):
        bs.set_tilt(j, probe=t["probe"], scan_x=t["sx"], scan_y=t["sy"], measured=t["meas"])
    bs.iteration_setup(nv, angles, positivity=True, tv_lambda=0.02, tv_iter=20, tv_fista=True)
    bs.set_rec(rec0)
    e_g, st_g = bs.iterate_bls(4, 0.5)
    rec_g = bs.get_rec()
    probes_g = [bs.get_tilt(j)[1] for j in range(3)]
    pos_g = [bs.get_tilt(j)[2:] for j in range(3)]
    bs.close()
    np.testing.assert_array_equal(st_g, np.asarray(st_o, np.float32))
    assert rel_l2(e_g, e_o) < 1e-4
    assert rel_l2(rec_g - rec0, rec_o - rec0) < 1e-4
    for j in range(3):
        assert rel_l2(probes_g[j] - tilts[j]["probe"], tl[j]["probe"] - tilts[j]["probe"]) < 1e-4
        d_g = np.r_[pos_g[j][0] - tilts[j]["sx"], pos_g[j][1] - tilts[j]["sy"]]
        d_o = np.r_[tl[j]["sx"] - tilts[j]["sx"], tl[j]["sy"] - tilts[j]["sy"]]
        # four accepted iterations of cancellation-limited position sums
        assert rel_l2(d_g, d_o) < 3e-4
