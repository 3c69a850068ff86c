"""Size-independent properties at the full mid workload (128^3 volume, 128^2
window, 21 tilts x 1,024 positions, 64 slabs of 2 voxels).  The FP64 oracle
checks this geometry on sampled positions (tests/test_gpu_geometry.py, 16
positions in seconds); running it over all 21,504 positions would take about
an hour of host time, so the whole workload is checked through properties
that hold at any size:

* noise-free data simulated by the library at the true volumes: the error
  and every gradient at the truth vanish (the simulation and the loss share
  the forward model bit for bit; only the 1e-30 of nearly dark pixels is
  left);
* checkpointing every 8 slabs (the gradient-validation configuration) gives
  the full-storage gradients (relative L2 <= 1e-9; only the FP64 atomics'
  order differs);
* a small step along the batched volume gradient lowers the error of every
  tilt (the reference formula is a descent direction).
"""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mid(gpu_available):
    from mset_b200 import synth
    from mset_b200.batch import BatchSession

    cfg = synth.CONFIGS["mid"]
    spec = synth.make_specimen(cfg)
    npos = [spec.scan_x.size] * cfg.n_tilts
    bs = BatchSession(n=cfg.window, nz=cfg.vol[0], npos=npos, prop=spec.prop, sigma=spec.sigma,
                      potential_pixelsize=cfg.dx, slice_binning=cfg.slice_binning)
    for j, v in enumerate(spec.volumes):
        bs.set_tilt(j, probe=spec.probe, scan_x=spec.scan_x, scan_y=spec.scan_y, volume=v)
    inten = bs.simulate()
    off = 0
    for j in range(cfg.n_tilts):
        bs.set_tilt(j, measured=inten[off:off + npos[j]])
        off += npos[j]
    del inten
    yield cfg, spec, bs
    bs.close()


def _set_volumes(bs, vols):
    for j, v in enumerate(vols):
        bs.set_tilt(j, volume=v)


def test_noise_free_truth_has_zero_error_and_gradient(mid):
    cfg, spec, bs = mid
    _set_volumes(bs, [0.5 * v for v in spec.volumes])
    off = bs.gradient(want=("grad", "err"))
    _set_volumes(bs, spec.volumes)
    out = bs.gradient(want=("grad", "err"))
    # A = sqrt(|Psi|^2 + 1e-30) equals M = sqrt(I) to the bit wherever
    # |Psi|^2 >> 1e-30, so only the epsilon of nearly dark pixels is left
    assert np.all(out["err"] <= 1e-20 * off["err"])
    assert np.abs(out["grad"]).max() <= 1e-12 * np.abs(off["grad"]).max()


def test_checkpointing_every_8_slabs_at_full_size(mid):
    cfg, spec, bs = mid
    _set_volumes(bs, [0.5 * v for v in spec.volumes])
    bs.set_checkpoint(0)
    full = bs.gradient()
    bs.set_checkpoint(8)
    ck = bs.gradient()
    bs.set_checkpoint(0)
    for key in ("grad", "probe", "posdir", "err"):
        assert rel_l2(ck[key], full[key]) < 1e-9, key
    assert np.all(full["err"] > 0)


def test_step_along_gradient_lowers_every_tilt_error(mid):
    cfg, spec, bs = mid
    V = [0.5 * v for v in spec.volumes]
    _set_volumes(bs, V)
    out = bs.gradient(want=("grad", "err"))
    e0, G = out["err"], out["grad"]
    b = cfg.slice_binning
    # RVol += step0 * Re(grad), slab-replicated (the reference's update)
    alpha = 1e-3 * max(float(np.abs(v).max()) for v in V) / float(np.abs(G).max())
    V1 = [(v + alpha * np.repeat(G[j], b, axis=0)[:v.shape[0]]).astype(np.float32) for j, v in enumerate(V)]
    _set_volumes(bs, V1)
    e1 = bs.error()
    assert np.all(e1 < e0), (e0, e1)
