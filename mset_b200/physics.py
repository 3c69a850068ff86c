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


ABERRATIONS = ("C10", "C30", "C50", "C12", "Phi12", "C23", "Phi23", "C21", "Phi21")


def check_probe_wave_parameters(ntilts: int, alpha=None, aberration_paras: dict | None = None,
                                probeDefocus=None) -> dict:
    """Per-tilt aberration lists as Func_check_probe_wave_parameters.m:20-145
    makes them: without aberration_paras every coefficient is zero for every
    tilt; a coefficient given once is broadcast to all tilts, a list must
    have one entry per tilt (else ValueError, the reference's error), a
    missing one is zero; a scalar probeDefocus sets C10 = -probeDefocus for
    every tilt.  Two behaviours of the reference are kept as they are: a
    per-tilt probeDefocus list is accepted and leaves C10 unchanged (only the
    scalar case assigns, :136-142), and Phi21 is broadcast when Phi12 (not
    Phi21) has a single entry (:121); Phi12 is per tilt by then, so for more
    than one tilt a single Phi21 is an error and Phi21 must be given per tilt.
    Returns a dict of float64 arrays [ntilts]."""
    if alpha is None:
        raise ValueError('input error: put probe forming aperture value (convergence semi-angle) into "alpha".')
    out = {}
    if aberration_paras is None:
        for k in ABERRATIONS:
            out[k] = np.zeros(ntilts)
    else:
        for k in ABERRATIONS:
            if k not in aberration_paras:
                out[k] = np.zeros(ntilts)
                continue
            v = np.atleast_1d(np.asarray(aberration_paras[k], dtype=np.float64)).ravel()
            # Phi21 is tested on Phi12's size, as the reference does
            probe_size = out["Phi12"].size if k == "Phi21" else v.size
            if probe_size == 1:
                out[k] = np.ones(ntilts) * v  # broadcast (a per-tilt v passes through elementwise)
                if out[k].size != ntilts:
                    raise ValueError(f"input error: make {k} list size and # of tilt angle be same")
            elif v.size != ntilts:
                raise ValueError(f"input error: make {k} list size and # of tilt angle be same")
            else:
                out[k] = v.copy()
    if probeDefocus is not None:
        d = np.atleast_1d(np.asarray(probeDefocus, dtype=np.float64)).ravel()
        if d.size == 1:
            out["C10"] = -1.0 * np.ones(ntilts) * d
        elif d.size != ntilts:
            raise ValueError("input error: make probeDefocus list size and # of tilt angle be same")
    return out


def probe_waves(n: int, dx: float, lam: float, alpha_mrad: float, paras: dict) -> np.ndarray:
    """Func_generate_probe_wave.m:14-56 for every tilt of the per-tilt
    aberration lists `paras` (check_probe_wave_parameters): [ntilts][n][n]
    complex128, before the per-tilt normalisation of STEP00_INIT.m:215-218"""
    nt = paras["C10"].size
    return np.stack([probe_wave(n, dx, lam, alpha_mrad, **{k: float(paras[k][p]) for k in ABERRATIONS})
                     for p in range(nt)])
