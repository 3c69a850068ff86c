"""Gradient truth (parity ladder L3): the EXACT adjoint of the FP64 oracle
against central finite differences (step 1e-3, FP64).

Loss of one position: L = sum_px (sqrt(|Psi|^2 + 1e-30) - sqrt(I))^2.
  dL/dV_z      = -2 sigma dz N^2 Re(g_s)       for every voxel z of slab s
  dL/dRe(p) + i dL/dIm(p) = 2 N^2 probe_dir    (probe p)
  dL/ds_x      = -2 N^2 pos_dir_x,  dL/ds_y = -2 N^2 pos_dir_y
The REF formula (the reference's STEP03 gradient, mset.cu:248-251) is a
descent direction but not the gradient; its cosine to the exact one is
reported.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2, small_case

H = 1e-3


def _case(method):
    c = small_case(n=16, nz=5, b=2, seed=11, strength=40.0, defocus=30.0, dx=0.5, jitter=2.0, consistent=False)
    c["method"] = method
    c["amp"] = O.amp_std(c["meas"][0])
    return c


def _loss(c, V=None, probe=None, sx=None, sy=None):
    return O.position_loss(c["V"] if V is None else V, c["probe"] if probe is None else probe, c["prop"],
                           float(c["sx"][0] if sx is None else sx), float(c["sy"][0] if sy is None else sy),
                           c["amp"], sigma=c["sigma"], dz=c["dz"], binning=c["b"], method=c["method"])


@pytest.mark.parametrize("method", [1, 2])
def test_exact_gradients_match_finite_differences(method):
    c = _case(method)
    n = c["V"].shape[1]
    o = O.position(c["V"], c["probe"], c["prop"], c["sx"][0], c["sy"][0], c["amp"], sigma=c["sigma"],
                   dz=c["dz"], binning=c["b"], method=method, adjoint=1)
    rng = np.random.default_rng(5)
    V0 = c["V"].astype(np.float64)
    nz = V0.shape[0]
    bb = nz if method == 2 else c["b"]
    # volume
    idx = [(rng.integers(nz), rng.integers(n), rng.integers(n)) for _ in range(12)]
    fd, an = [], []
    for z, y, x in idx:
        Vp, Vm = V0.copy(), V0.copy()
        Vp[z, y, x] += H
        Vm[z, y, x] -= H
        fd.append((_loss(c, V=Vp) - _loss(c, V=Vm)) / (2 * H))
        an.append(-2 * c["sigma"] * c["dz"] * n * n * o["grad"][z // bb, y, x].real)
    assert rel_l2(an, fd) < 1e-4
    # probe (Wirtinger: dL/dRe + i dL/dIm = 2 N^2 probe_dir)
    P0 = c["probe"].astype(np.complex128)
    fdp, anp = [], []
    for _ in range(8):
        y, x = rng.integers(n), rng.integers(n)
        for d in (1.0, 1j):
            Pp, Pm = P0.copy(), P0.copy()
            h = H * np.abs(P0).max()
            Pp[y, x] += d * h
            Pm[y, x] -= d * h
            fdp.append((_loss(c, probe=Pp) - _loss(c, probe=Pm)) / (2 * h))
            g = 2 * n * n * o["probe_dir"][y, x]
            anp.append(g.real if d == 1.0 else g.imag)
    assert rel_l2(anp, fdp) < 1e-4
    # scan positions
    for k, (dx, dy) in enumerate(((H, 0.0), (0.0, H))):
        x0, y0 = float(c["sx"][0]), float(c["sy"][0])  # FP64 perturbation, not float32
        f = (_loss(c, sx=x0 + dx, sy=y0 + dy) - _loss(c, sx=x0 - dx, sy=y0 - dy)) / (2 * H)
        a = -2 * n * n * o["pos_dir"][k]
        assert abs(a - f) <= 1e-4 * abs(f) + 1e-9


def test_reference_formula_is_descent_not_gradient():
    c = _case(1)
    e = O.position(c["V"], c["probe"], c["prop"], c["sx"][0], c["sy"][0], c["amp"], sigma=c["sigma"],
                   dz=c["dz"], binning=c["b"], adjoint=1)
    r = O.position(c["V"], c["probe"], c["prop"], c["sx"][0], c["sy"][0], c["amp"], sigma=c["sigma"],
                   dz=c["dz"], binning=c["b"], adjoint=0)
    ge, gr = e["grad"].real.ravel(), r["grad"].real.ravel()
    cos = ge @ gr / np.linalg.norm(ge) / np.linalg.norm(gr)
    assert cos > 0.9          # still a descent direction
    assert rel_l2(gr, ge) > 1e-4  # but not the gradient of the loss
