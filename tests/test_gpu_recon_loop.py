"""The reference's reconstruction loop (mset_b200.recon.reconstruct:
per tilt inverse rotation, run_mset with per-position updates, rotation back,
positivity; error pass and line search) on the small configuration (24^3
sample at 0.4 A centred in the 64^3 volume the loop rotates, 64^2 window,
12x12 scan, 5 tilts over +-30 deg), driven through the library (GPU) and through the FP64 oracle,
two iterations from half the true potential with probe and position steps
on: volume and mean errors relative L2 <= 1e-5 / 1e-4, the volume's change
5e-4 (FP32 rounding of the whole-volume rotations against a 5% change);
probe changes 3e-4 (coupled to the volume through 288 sequential updates);
positions at the cancellation-limited 3e-4."""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_reference_loop_library_vs_oracle(gpu_available):
    from mset_b200 import Session, recon, synth
    from mset_b200.batch import BatchSession
    from oracle import oracle as O
    from tests.recon_oracle import OracleBackend

    cfg = synth.CONFIGS["small"]
    spec = synth.make_specimen(cfg)
    P = spec.scan_x.size
    # the reference's loop rotates the reconstruction in the window's frame:
    # the 24^3 sample centred in a 64^3 volume (64 slices)
    n = cfg.window
    lab = np.zeros((n, n, n), np.float32)
    o0 = (n - cfg.vol[0]) // 2
    lab[o0:o0 + cfg.vol[0], o0:o0 + cfg.vol[1], o0:o0 + cfg.vol[2]] = spec.lab
    # measured data: the truth through the library's rotation and forward model, Poisson noise
    bs = BatchSession(n=n, nz=n, npos=[P] * cfg.n_tilts, prop=spec.prop, sigma=spec.sigma,
                      potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning)
    with Session() as rot:
        for j, a in enumerate(spec.angles):
            bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y,
                        volume=rot.rotate_volume(lab, a, inverse=True))
    meas = synth.poisson(bs.simulate(), seed=10)
    bs.close()
    # three of the five tilts (-30, 0, +30 deg): the FP64 oracle's 64^3
    # rotations take seconds each on the host
    keep = [0, 2, 4]
    tilts = [recon.Tilt(spec.probe, spec.scan_x, spec.scan_y, meas[j * P:(j + 1) * P], tuple(cfg.scan))
             for j in keep]
    angles = spec.angles[keep]
    rec0 = 0.5 * lab
    # steps that move the state by ~1e-2 (object), ~1e-3 (probe), ~0.05 px
    o = O.position(0.5 * O.rot3d(lab, spec.angles[2], inverse=True), spec.probe, spec.prop, spec.scan_x[0],
                   spec.scan_y[0], O.amp_std(tilts[2].measured[0]), sigma=spec.sigma, dz=cfg.dx)
    step = (1e-2 * rec0.max() / np.abs(o["grad"]).max(), 1e-3 * np.abs(spec.probe).max() / np.abs(o["probe_dir"]).max(),
            0.05 / np.abs(o["pos_dir"]).max())
    kw = dict(sigma=spec.sigma, dz=cfg.dx, step=step, n_iter=2, bls_parameter=0.5, positivity=True)
    lib = recon.LibraryBackend()
    r_g = recon.reconstruct(lib, rec0, tilts, spec.prop, angles, **kw)
    lib.close()
    r_o = recon.reconstruct(OracleBackend(), rec0, tilts, spec.prop, angles, **kw)
    assert len(r_g.mean_error) == len(r_o.mean_error) == 2
    assert np.allclose(r_g.step, r_o.step)
    assert rel_l2(r_g.rec, r_o.rec) < 1e-5
    # the change is ~5% of the volume and each of the 12 whole-volume
    # rotations adds FP32 rounding of ~1e-6 of the volume itself
    assert rel_l2(r_g.rec - rec0, r_o.rec - rec0) < 5e-4
    assert rel_l2(np.array(r_g.mean_error), np.array(r_o.mean_error)) < 1e-4
    for tg, to, t0 in zip(r_g.tilts, r_o.tilts, tilts):
        # 288 sequential probe updates, each on a volume that carries the
        # rotations' FP32 rounding (the per-pass probe direction itself is
        # checked at 1e-4 in test_gpu_parity.py)
        assert rel_l2(tg.probe - t0.probe, to.probe - t0.probe) < 3e-4
        d_g = np.r_[tg.scan_x - t0.scan_x, tg.scan_y - t0.scan_y]
        d_o = np.r_[to.scan_x - t0.scan_x, to.scan_y - t0.scan_y]
        assert rel_l2(d_g, d_o) < 3e-4
