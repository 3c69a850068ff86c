"""The reference's reconstruction loop (Run_MSET_recon.m:106-287, CUDA
device mode) on this library: for every iteration, tilt after tilt,

    RVol = single(Func_inv_rot(rec, angles_j))            STEP01_ROTATION.m
    mset_cuda_kernel('upload' / 'run_mset')               Run_MSET_recon.m:160-172
    rec  = Func_rot(RVol, angles_j); rec(rec < 0) = 0     :178-185

then the error pass of the new state over all tilts (:189-237) and the
backtracking line search (:239-253): keep the iteration if the mean error fell
below the previous one, else restore rec / probes / positions, multiply the
step sizes by bls_parameter and retry; stop once the object step is below
bls_parameter^5 times its first value.  TV of rec / max(rec) after an accepted
iteration when enabled (:262-270).

The per-tilt work goes through a backend with the interface of
`LibraryBackend` (the library's MEX-compatible entry points, Fourier-shear
rotation and TV on the GPU); arrays are C views of the MATLAB arrays
(volumes [nz][ny][nx], probes and patterns [n][n] transposed from MATLAB).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from ._lib import MSET_MODE_MSET
from .session import Session


@dataclass
class Tilt:
    probe: np.ndarray   # [n][n] complex64
    scan_x: np.ndarray  # [P] float32, 1-based pixels
    scan_y: np.ndarray
    measured: np.ndarray  # [P][n][n] float32, centred patterns (cell order)
    n_scan: tuple = (0, 0)  # (N_scan_x, N_scan_y)


@dataclass
class Result:
    rec: np.ndarray
    rec_per_iter: list = field(default_factory=list)
    mean_error: list = field(default_factory=list)
    step: np.ndarray | None = None
    stopped_early: bool = False


class LibraryBackend:
    """Per-tilt work on the GPU through the C ABI.

    per_position=False: the CUDA device mode, one fused sequential pass per
    tilt (mset_run, Run_MSET_recon.m:160-172).  per_position=True: the CPU
    device modes' loop, STEP02 -> STEP03 -> STEP04 position by position
    (Run_MSET_recon.m:136-157) through mset_forward_position /
    mset_adjoint_position; the same updates, one launch per step."""

    def __init__(self, device: int = 0, vecs=((0, 0, 1), (0, 1, 0), (1, 0, 0)), per_position: bool = False):
        self.s = Session(device)
        self.vecs = vecs
        self.per_position = per_position

    def close(self):
        self.s.close()

    def rotate(self, vol, angles, inverse: bool):
        return self.s.rotate_volume(vol, angles, inverse=inverse, vec1=self.vecs[0], vec2=self.vecs[1],
                                    vec3=self.vecs[2])

    def run_tilt(self, V, t: Tilt, prop, *, sigma, dz, step, binning, method):
        nsx, nsy = t.n_scan if t.n_scan[0] else (t.scan_x.size, 1)
        self.s.upload(V, t.probe, prop, sigma=sigma, potential_pixelsize=dz, scan_x=t.scan_x, scan_y=t.scan_y,
                      measured=t.measured, step_size=step, slice_binning=binning, n_scan_x=nsx, n_scan_y=nsy)
        if not self.per_position:
            rv, pr, sx, sy, _ = self.s.run(method)
            return rv, pr, sx, sy
        sx = np.array(t.scan_x, dtype=np.float32, copy=True)
        sy = np.array(t.scan_y, dtype=np.float32, copy=True)
        for k in range(sx.size):
            self.s.step02(k, sx[k], sy[k], mode=method)
            # STEP03 and STEP04 (:155) on the device: RVol and the probe stay
            # there between positions, the scan coordinates come back
            g = self.s.step03(mode=method, update_rvol=True, want=())
            sx[k], sy[k] = g["row"], g["col"]
        rv, pr = self.s.read_state()
        return rv, pr, sx, sy

    def error_tilt(self, V, t: Tilt, prop, *, sigma, dz, binning, method) -> float:
        nsx, nsy = t.n_scan if t.n_scan[0] else (t.scan_x.size, 1)
        self.s.upload(V, t.probe, prop, sigma=sigma, potential_pixelsize=dz, scan_x=t.scan_x, scan_y=t.scan_y,
                      measured=t.measured, slice_binning=binning, n_scan_x=nsx, n_scan_y=nsy)
        return float(self.s.error(method))

    def tv(self, vol, lam: float, niter: int, fista: bool = False):
        return self.s.tv(vol, lam, niter, fista=fista)


def reconstruct(backend, rec: np.ndarray, tilts: Sequence[Tilt], prop: np.ndarray, angles, *, sigma: float,
                dz: float, step, n_iter: int, binning: int = 1, method: int = MSET_MODE_MSET,
                bls_parameter: float = 0.1, positivity: bool = True, use_tv: bool = False,
                tv_lambda: float = 0.005, tv_iter: int = 300) -> Result:
    rec = np.ascontiguousarray(rec, dtype=np.float32)
    tilts = [Tilt(t.probe.astype(np.complex64), t.scan_x.astype(np.float32), t.scan_y.astype(np.float32),
                  t.measured, t.n_scan) for t in tilts]
    step = np.asarray(step, dtype=np.float64).copy()
    step0 = step[0]
    old_mean = 1e31
    out = Result(rec=rec)
    for _ in range(n_iter):
        old = (rec.copy(), [(t.probe.copy(), t.scan_x.copy(), t.scan_y.copy()) for t in tilts])
        stop = False
        while True:
            for j, t in enumerate(tilts):
                V = backend.rotate(rec, angles[j], inverse=True).astype(np.float32)
                V, t.probe, t.scan_x, t.scan_y = backend.run_tilt(V, t, prop, sigma=sigma, dz=dz, step=step,
                                                                  binning=binning, method=method)
                rec = backend.rotate(V, angles[j], inverse=False).astype(np.float32)
                if positivity:
                    rec = np.maximum(rec, 0).astype(np.float32)
            err = []
            for j, t in enumerate(tilts):
                V = backend.rotate(rec, angles[j], inverse=True).astype(np.float32)
                err.append(backend.error_tilt(V, t, prop, sigma=sigma, dz=dz, binning=binning, method=method))
            mean = float(np.mean(err))
            if old_mean > mean:
                break
            rec = old[0].copy()
            for t, (p, x, y) in zip(tilts, old[1]):
                t.probe, t.scan_x, t.scan_y = p.copy(), x.copy(), y.copy()
            step = bls_parameter * step
            if step[0] < bls_parameter ** 5 * step0:
                stop = True
                break
        if stop:
            out.stopped_early = True
            break
        if use_tv and float(rec.max()) > 0:  # (an all-zero volume has nothing to regularise)
            m = float(rec.max())
            rec = (m * backend.tv(rec / m, tv_lambda, tv_iter)).astype(np.float32)
        out.rec_per_iter.append(rec.copy())
        out.mean_error.append(mean)
        old_mean = mean
    out.rec = rec
    out.step = step
    out.tilts = tilts
    return out


def load_example(folder: str, probe_from: str | None = None):
    """The reference's example tilt series (examples/CuAu_24size_dataset):
    8 files `*_4DSTEM_data_<j>.mat` (v7.3, cell Full_4D_STEM_data{x, y} of
    n x n patterns), `scan_pos.mat` ([P, 2] pixels), `tilt_angles.mat`
    ([J, 3] degrees).  Returns dict(tilts, angles) with patterns in cell
    (column-major) order and C views of the MATLAB arrays.  The probes are
    left None unless `probe_from` names a v7.3 file holding
    STEM_data.probe_wfn ([n, n, J] complex), e.g. the stored reconstruction."""
    import glob
    import os

    import scipy.io as sio

    from .matfile import loadmat73

    files = sorted(glob.glob(os.path.join(folder, "*_4DSTEM_data_*.mat")),
                   key=lambda f: int(f.rsplit("_", 1)[1].split(".")[0]))
    if not files:
        raise FileNotFoundError(f"no *_4DSTEM_data_*.mat files in {folder}")
    sp = sio.loadmat(os.path.join(folder, "scan_pos.mat"))["scan_pos"].astype(np.float32)
    ang = sio.loadmat(os.path.join(folder, "tilt_angles.mat"))
    angles = np.asarray(ang[[k for k in ang if not k.startswith("__")][0]], dtype=np.float64)
    probes = None
    if probe_from:
        probes = loadmat73(probe_from, names=["STEM_data"])["STEM_data"]["probe_wfn"]
    tilts = []
    for j, f in enumerate(files):
        cells = next(iter(loadmat73(f).values()))
        nsx, nsy = cells.shape
        P = nsx * nsy
        meas = np.stack([np.asarray(cells[k % nsx, k // nsx], np.float32).T for k in range(P)])
        pr = None if probes is None else np.ascontiguousarray(probes[:, :, j].T.astype(np.complex64))
        tilts.append(Tilt(pr, sp[:P, 0].copy(), sp[:P, 1].copy(), np.ascontiguousarray(meas), (nsx, nsy)))
    return {"tilts": tilts, "angles": angles}
