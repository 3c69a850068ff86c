"""Seeded synthetic tilt series (no public dataset is used).

A specimen is an fcc Cu/Au-like lattice of Gaussian atom blobs voxelised
directly in each tilt's beam frame (the atom coordinates are rotated, so no
interpolation enters the ground truth).  Probe, propagator and raster scan
follow the reference's set-up (STEP00_INIT.m:160-218, func_lib).  Measured
intensities are produced by a caller-supplied forward model plus seeded
Poisson noise, so the same generator serves CPU tests and GPU benchmarks.

All arrays are C order: volumes [nz][n][n] (x fastest), probes [n][n].
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import physics


@dataclass
class Config:
    name: str
    vol: tuple          # (nz, ny, nx) voxels of the specimen volume
    dx: float           # Angstrom per voxel
    window: int         # probe window n (volume zero-padded laterally to it)
    scan: tuple         # (N_scan_x, N_scan_y)
    scan_step: float    # pixels
    n_tilts: int
    tilt_max: float     # degrees, tilts evenly spaced over +-tilt_max
    slice_binning: int
    dose: float         # electrons per probe position
    E0_kV: float = 300.0
    alpha_mrad: float = 20.0
    defocus_A: float = 0.0
    C30_A: float = 0.0
    jitter_px: float = 0.0
    lattice: float = 3.8     # Angstrom, between Cu (3.615) and Au (4.078)
    blob_sigma: float = 0.3  # Angstrom
    peak_range: tuple = (1.0, 3.0)
    seed: int = 0
    extra: dict = field(default_factory=dict)


CONFIGS = {
    # small plain iteration: 24^3 at 0.4 A, 64^2 window, 12x12 scan at 2 px,
    # 24 slices of 1 voxel, 5 tilts over +-30 deg, 1e4 e-/probe
    "small": Config("small", (24, 24, 24), 0.4, 64, (12, 12), 2.0, 5, 30.0, 1, 1e4),
    # batched mid-size: 128^3 at 0.3 A, 128^2 window, 32x32 scan at 3 px,
    # 21 tilts over +-60 deg, 64 slices of 2 voxels
    "mid": Config("mid", (128, 128, 128), 0.3, 128, (32, 32), 3.0, 21, 60.0, 2, 1e4),
    # the mid-size geometry (128^2 window, 64 slabs of 2 voxels) on a small
    # position set: 2 tilts x 8x8 scan, for profiling captures
    "mid_s": Config("mid_s", (128, 128, 128), 0.3, 128, (8, 8), 3.0, 2, 60.0, 2, 1e4),
    # adjoint / gradient validation: the small sample in a 128^2 window with
    # +-5 nm defocus and C3 = 1 mm +- 1 um probe errors and +-0.5 px jitter
    "grad": Config("grad", (24, 24, 24), 0.4, 128, (12, 12), 2.0, 5, 30.0, 1, 1e4,
                   defocus_A=50.0, C30_A=1e7, jitter_px=0.5),
    # large single reconstruction: 256x256x192 at 0.25 A, 256^2 window (one
    # field over a 4-CTA cluster), 64x64 scan at 4 px, 41 tilts over +-70 deg,
    # 96 slices of 2 voxels
    "large": Config("large", (192, 256, 256), 0.25, 256, (64, 64), 4.0, 41, 70.0, 2, 1e4),
    # its geometry on 3 of the tilts (-70, 0, +70 deg), for timing samples
    "large_s": Config("large_s", (192, 256, 256), 0.25, 256, (64, 64), 4.0, 3, 70.0, 2, 1e4),
    # a cubic 256^3 reconstruction in the same window (the batched iteration
    # rotates cubic volumes), 128 slices of 2 voxels, on 3 tilts
    "large_cubic_s": Config("large_cubic_s", (256, 256, 256), 0.25, 256, (64, 64), 4.0, 3, 70.0, 2, 1e4),
    # its geometry on 1 tilt x 12x12 positions, for profiling captures
    "large_p": Config("large_p", (192, 256, 256), 0.25, 256, (12, 12), 4.0, 1, 0.0, 2, 1e4),
}

# uneven-size batch: 6 independent tilt series run as one pass, windows 64^2 to
# 160^2, scans 16x16 to 40x40, 11 to 31 tilts, 32 to 96 slabs, volume edges 64
# to 128 voxels, doses 1e3 to 1e5 e-/probe
UNEVEN = [
    Config("uneven_64a", (64, 64, 64), 0.3, 64, (16, 16), 2.0, 11, 50.0, 2, 1e3, seed=101),
    Config("uneven_96a", (96, 96, 96), 0.3, 96, (24, 24), 2.0, 15, 60.0, 2, 1e4, seed=102),
    Config("uneven_128", (128, 128, 128), 0.3, 128, (32, 32), 3.0, 21, 60.0, 2, 1e5, seed=103),
    Config("uneven_160", (96, 96, 96), 0.3, 160, (24, 24), 4.0, 31, 70.0, 1, 3e4, seed=104),
    Config("uneven_64b", (64, 64, 64), 0.3, 64, (40, 40), 1.0, 31, 70.0, 2, 3e3, seed=105),
    Config("uneven_96b", (96, 96, 96), 0.3, 96, (20, 20), 3.0, 11, 40.0, 1, 1e5, seed=106),
]


def tilt_angles(cfg: Config) -> np.ndarray:
    """[n_tilts, 3] (phi, theta, psi) in degrees; rotation about y only."""
    th = np.linspace(-cfg.tilt_max, cfg.tilt_max, cfg.n_tilts) if cfg.n_tilts > 1 else np.zeros(1)
    a = np.zeros((cfg.n_tilts, 3))
    a[:, 1] = th
    return a


def rot_y(theta_deg: float) -> np.ndarray:
    t = np.deg2rad(theta_deg)
    c, s = np.cos(t), np.sin(t)
    # acting on (x, y, z)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def atoms(cfg: Config, rng: np.random.Generator):
    """fcc lattice filling the specimen box; returns xyz (Angstrom, centred)
    and peak amplitudes."""
    nz, ny, nx = cfg.vol
    ext = np.array([nx, ny, nz]) * cfg.dx
    a = cfg.lattice
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    ncell = np.ceil(ext / a).astype(int) + 1
    g = np.stack(np.meshgrid(*[np.arange(-c, c + 1) for c in ncell // 2 + 1], indexing="ij"), -1).reshape(-1, 3)
    pos = (g[:, None, :] + basis[None]).reshape(-1, 3) * a
    pos = pos + rng.normal(0, 0.05, pos.shape)
    keep = np.all(np.abs(pos) < ext / 2 - 2 * cfg.blob_sigma, axis=1)
    pos = pos[keep]
    au = rng.random(len(pos)) < 0.5
    lo, hi = cfg.peak_range
    mid = 0.5 * (lo + hi)
    peak = np.where(au, rng.uniform(mid, hi, len(pos)), rng.uniform(lo, mid, len(pos)))
    return pos, peak


def voxelise(pos: np.ndarray, peak: np.ndarray, shape: tuple, dx: float, sigma: float) -> np.ndarray:
    """Sum of Gaussian blobs on a [nz][ny][nx] grid centred at index
    round((n+1)/2) - 1 (the reference's centre convention)."""
    nz, ny, nx = shape
    c = np.array([np.floor((nx + 1) / 2 + 0.5) - 1, np.floor((ny + 1) / 2 + 0.5) - 1,
                  np.floor((nz + 1) / 2 + 0.5) - 1])
    V = np.zeros(shape, np.float64)
    r = int(np.ceil(4 * sigma / dx))
    off = np.arange(-r, r + 1)
    for p, a in zip(pos, peak):
        ic = np.round(p / dx + c).astype(int)
        ix, iy, iz = ic[0] + off, ic[1] + off, ic[2] + off
        mx = (ix >= 0) & (ix < nx)
        my = (iy >= 0) & (iy < ny)
        mz = (iz >= 0) & (iz < nz)
        if not (mx.any() and my.any() and mz.any()):
            continue
        gx = np.exp(-(((ix[mx] - c[0]) * dx - p[0]) ** 2) / (2 * sigma ** 2))
        gy = np.exp(-(((iy[my] - c[1]) * dx - p[1]) ** 2) / (2 * sigma ** 2))
        gz = np.exp(-(((iz[mz] - c[2]) * dx - p[2]) ** 2) / (2 * sigma ** 2))
        V[np.ix_(iz[mz], iy[my], ix[mx])] += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return V


def pad_lateral(V: np.ndarray, n: int) -> np.ndarray:
    nz, ny, nx = V.shape
    if ny == n and nx == n:
        return V
    out = np.zeros((nz, n, n), V.dtype)
    oy, ox = (n - ny) // 2, (n - nx) // 2
    out[:, oy:oy + ny, ox:ox + nx] = V
    return out


def raster(cfg: Config, rng: np.random.Generator | None = None):
    """1-based scan coordinates, x fastest (ind2sub order, STEP00_INIT.m:173-178),
    centred on the window centre round((n+1)/2)."""
    nsx, nsy = cfg.scan
    c = np.floor((cfg.window + 1) / 2 + 0.5)
    xs = c + (np.arange(nsx) - (nsx - 1) / 2) * cfg.scan_step
    ys = c + (np.arange(nsy) - (nsy - 1) / 2) * cfg.scan_step
    X, Y = np.meshgrid(xs, ys, indexing="xy")  # Y rows, X fastest
    sx, sy = X.reshape(-1), Y.reshape(-1)
    if cfg.jitter_px and rng is not None:
        sx = sx + rng.uniform(-cfg.jitter_px, cfg.jitter_px, sx.shape)
        sy = sy + rng.uniform(-cfg.jitter_px, cfg.jitter_px, sy.shape)
    return sx.astype(np.float32), sy.astype(np.float32)


@dataclass
class Specimen:
    cfg: Config
    angles: np.ndarray        # [J, 3]
    volumes: list             # per tilt beam-frame volume [nz][n][n] float32 (ground truth)
    lab: np.ndarray | None    # lab-frame volume [nz][ny][nx] float32 (ground truth, unpadded)
    probe: np.ndarray         # [n][n] complex64, normalised to the dose
    prop: np.ndarray          # [n][n] complex64 centred
    scan_x: np.ndarray        # [P] float32
    scan_y: np.ndarray
    sigma: float
    lam: float
    natoms: int


def make_specimen(cfg: Config, with_volumes: bool = True, per_tilt: bool = True) -> Specimen:
    """per_tilt=False: only the lab-frame volume (tilts left to a rotation)"""
    rng = np.random.default_rng(cfg.seed)
    lam = physics.electron_wavelength(cfg.E0_kV * 1e3)
    sigma = physics.interaction_constant(cfg.E0_kV * 1e3)
    pos, peak = atoms(cfg, rng)
    angles = tilt_angles(cfg)
    vols = []
    lab = None
    if with_volumes:
        lab = voxelise(pos, peak, cfg.vol, cfg.dx, cfg.blob_sigma).astype(np.float32)
        for th in (angles[:, 1] if per_tilt else []):
            # beam frame of tilt th: the reference's Func_inv_rot_3Dvol_FourierShear
            # with (phi, theta, psi) = (0, th, 0) maps (x, 0, 0) to (x cos th, 0, x sin th)
            R = rot_y(-th)
            v = voxelise(pos @ R.T, peak, cfg.vol, cfg.dx, cfg.blob_sigma)
            vols.append(pad_lateral(v, cfg.window).astype(np.float32))
    n = cfg.window
    probe = physics.probe_wave(n, cfg.dx, lam, cfg.alpha_mrad, C10=-cfg.defocus_A, C30=cfg.C30_A)
    probe = physics.normalise_probe(probe, cfg.dose).astype(np.complex64)
    prop = physics.propagator(n, cfg.dx, lam, cfg.slice_binning)
    sx, sy = raster(cfg, rng)
    return Specimen(cfg, angles, vols, lab, probe, prop, sx, sy, float(sigma), float(lam), len(pos))


def poisson(intensities: np.ndarray, seed: int) -> np.ndarray:
    """Seeded Poisson counts of expected intensities (already scaled to the dose)."""
    rng = np.random.default_rng(seed)
    return rng.poisson(np.maximum(intensities, 0).astype(np.float64)).astype(np.float32)


def simulate(spec: Specimen, forward: Callable[[int, np.ndarray], np.ndarray], seed: int | None = None):
    """measured[j] = Poisson(forward(j, volume_j)) for every tilt; `forward`
    returns |Psi|^2 in the centred layout, [P][n][n]."""
    s = spec.cfg.seed + 1000 if seed is None else seed
    return [poisson(forward(j, v), s + j) for j, v in enumerate(spec.volumes)]
