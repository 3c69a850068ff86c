"""The gradient-validation configuration: the small 24^3 sample (0.4 A voxels,
24 slices) in a 128^2 window, 5 tilts x 12x12 positions, with joint probe and
scan-position refinement.  The truth has a probe with 5 nm defocus and
C3 = 1 mm and scan positions jittered by up to 0.5 px; the estimate has half
the potential, a probe 5 nm further from focus with C3 1 um larger, and the
nominal raster.  The library's EXACT gradients for V, probe and positions,
with the waves checkpointed every 8 slices and recomputed, against the FP64
oracle (itself pinned to central finite differences in test_oracle_fd.py):
relative L2 <= 1e-4 for V and the probe; the scan-position directions of this
weak sample are cancellation-limited (see the assertion)."""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_exact_gradients_of_the_validation_configuration(gpu_available):
    from mset_b200 import MSET_ADJOINT_EXACT, physics, synth
    from mset_b200.batch import BatchSession
    from oracle import oracle as O

    cfg = synth.CONFIGS["grad"]
    spec = synth.make_specimen(cfg)
    n, nz, J = cfg.window, cfg.vol[0], cfg.n_tilts
    P = spec.scan_x.size
    sx0, sy0 = synth.raster(synth.Config(**{**cfg.__dict__, "jitter_px": 0.0}))
    pr_est = physics.normalise_probe(
        physics.probe_wave(n, cfg.dx, spec.lam, cfg.alpha_mrad, C10=-(cfg.defocus_A + 50.0), C30=cfg.C30_A + 1e4),
        float(np.sum(np.abs(np.fft.fft2(spec.probe)) ** 2))).astype(np.complex64)

    def session():
        return BatchSession(n=n, nz=nz, npos=[P] * J, prop=spec.prop, sigma=spec.sigma,
                            potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning,
                            adjoint=MSET_ADJOINT_EXACT)

    # measured data: the truth through the library's forward model, seeded Poisson noise
    bs = session()
    for j, v in enumerate(spec.volumes):
        bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y, volume=v)
    meas = synth.poisson(bs.simulate(), seed=cfg.seed + 1)
    bs.close()

    bs = session()
    bs.set_checkpoint(8)
    for j, v in enumerate(spec.volumes):
        bs.set_tilt(j, probe=pr_est, scan_x=sx0, scan_y=sy0, measured=meas[j * P:(j + 1) * P], volume=0.5 * v)
    out = bs.gradient()
    bs.close()
    for j, v in enumerate(spec.volumes):
        g, pa, pd, e = O.batched_tilt(0.5 * v, pr_est, spec.prop, sx0, sy0, meas[j * P:(j + 1) * P],
                                      sigma=spec.sigma, dz=cfg.dx, binning=cfg.slice_binning,
                                      adjoint=MSET_ADJOINT_EXACT)
        assert rel_l2(out["grad"][j], g) < 1e-4, j
        assert rel_l2(np.fft.fft2(out["probe"][j]), pa) < 1e-4, j
        # the weak 24^3 sample makes each position direction a sum over
        # 128^2 pixels with a cancellation factor sum|t| / |sum t| of
        # 1.5e6 - 3e6 (measured with the oracle's FP64 terms), which FP32
        # propagation resolves to a few 1e-2: the directions agree to a
        # cosine of 0.999
        d = out["posdir"][j * P:(j + 1) * P].ravel()
        assert rel_l2(d, pd.ravel()) < 5e-2, j
        assert np.dot(d, pd.ravel()) / np.linalg.norm(d) / np.linalg.norm(pd) > 0.999, j
        assert abs(out["err"][j] - e) <= 1e-4 * e, j
