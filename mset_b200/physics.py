"""Host-side physics set-up (once per run, FP64), restating the reference's
func_lib helpers.  Arrays are returned in C order: a MATLAB (dim1, dim2) array
is returned as [dim2][dim1], so x (MATLAB dim 1) is the fastest axis.
"""
from __future__ import annotations

import numpy as np

# constants as written in func_lib/electron_wavelength.m:3-6
_M = 9.109383e-31
_E = 1.602177e-19
_C = 299792458.0
_H = 6.62607e-34


def electron_wavelength(E0_eV: float) -> float:
    """Relativistic wavelength in Angstrom (func_lib/electron_wavelength.m:1-9)."""
    return _H / np.sqrt(2 * _M * _E * E0_eV) / np.sqrt(1 + _E * E0_eV / 2 / _M / _C ** 2) * 1e10


def interaction_constant(E0_eV: float) -> float:
    """sigma in rad/(V*Angstrom) (func_lib/interaction_constant.m:1-10)."""
    lam = electron_wavelength(E0_eV)
    return (2 * np.pi / lam / E0_eV) * (_M * _C ** 2 + _E * E0_eV) / (2 * _M * _C ** 2 + _E * E0_eV)


def _qgrid(n: int, dx: float):
    """q grid of Func_generate_propagator.m:17-26 (centre round((n+1)/2))."""
    k = np.arange(1, n + 1)
    cent = np.floor((n + 1) / 2 + 0.5)  # MATLAB round for positive values
    q = (k - cent) / (n * dx)
    # ndgrid(qx along dim1, qy along dim2) -> C order [dim2][dim1]
    qx = q[None, :]
    qy = q[:, None]
    return qx, qy


def propagator(n: int, dx: float, lam: float, slice_binning: int = 1) -> np.ndarray:
    """Fresnel propagator exp(-i pi lambda (dx*b) q^2), centred, complex64
    (Func_generate_propagator.m:14-39)."""
    qx, qy = _qgrid(n, dx)
    q2 = qx ** 2 + qy ** 2
    return np.exp(-1j * np.pi * lam * (dx * slice_binning) * q2).astype(np.complex64)


def probe_wave(n: int, dx: float, lam: float, alpha_mrad: float, C10: float = 0.0, C30: float = 0.0,
               C50: float = 0.0, C12: float = 0.0, Phi12: float = 0.0, C21: float = 0.0, Phi21: float = 0.0,
               C23: float = 0.0, Phi23: float = 0.0) -> np.ndarray:
    """Aberrated probe, real space, centred (Func_generate_probe_wave.m:20-53):
    fftshift(fft2(ifftshift(mask * exp(-i chi)))).  Aberrations in Angstrom,
    angles in rad.  Returns complex128 [n][n]."""
    qx, qy = _qgrid(n, dx)
    q2 = qx ** 2 + qy ** 2
    qa = lam * np.sqrt(q2)
    phi = np.arctan2(qy, qx)
    mask = q2 < (alpha_mrad / 1000 / lam) ** 2
    chi = (0.5 * qa ** 2 * C10 + 0.25 * qa ** 4 * C30 + (1 / 6) * qa ** 6 * C50
           + 0.5 * qa ** 2 * C12 * np.cos(2 * (phi - Phi12))
           + (1 / 3) * qa ** 3 * C21 * np.cos(phi - Phi21)
           + (1 / 3) * qa ** 3 * C23 * np.cos(3 * (phi - Phi23)))
    chi = 2 * np.pi / lam * chi
    return np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(mask * np.exp(-1j * chi))))


def normalise_probe(probe: np.ndarray, mean_intensity: float) -> np.ndarray:
    """Scale so that sum |fft2(probe)|^2 equals the mean measured pattern sum
    (STEP00_INIT.m:215-218)."""
    s = np.sum(np.abs(np.fft.fft2(probe)) ** 2)
    return probe * np.sqrt(mean_intensity / s)
