"""FP64 oracle of one batched iteration, assembled from the oracle pieces
(oracle/oracle.py rotation and batched tilt pass, oracle/tv.py):

    V_j  = pad(Func_inv_rot(rec, angles_j))
    G_j  = sum_p Re g_{j,p}              (batched pass, slab-replicated)
    rec += step0 * sum_j crop(Func_rot(G_j))
    rec  = max(rec, 0)                   (if positivity)
    rec  = max(rec) * TV(rec / max(rec)) (if tv_lambda > 0)
    probe_j -= step1 * sum_p shift_{-s}(chi0);  positions += step2 * posdir
"""
import numpy as np

from oracle import oracle as O
from oracle import tv


def pad(v, n):
    nv = v.shape[0]
    o = (n - nv) // 2
    out = np.zeros((nv, n, n), v.dtype)
    out[:, o:o + nv, o:o + nv] = v
    return out


def crop(g, nv):
    n = g.shape[1]
    o = (n - nv) // 2
    return g[:, o:o + nv, o:o + nv]


def iterate(rec, tilts, prop, angles, *, sigma, dz, binning, step, positivity=True, tv_lambda=0.0, tv_iter=0,
            tv_fista=True, method=1, adjoint=0):
    """tilts: list of dicts with probe, sx, sy, meas (updated in place).
    Returns (rec, errs)."""
    nv = rec.shape[0]
    acc = np.zeros((nv, nv, nv))
    errs = []
    for j, t in enumerate(tilts):
        n = t["probe"].shape[0]
        V = pad(O.rot3d(rec, angles[j], inverse=True), n).astype(np.float32)
        g, pa, pd, e = O.batched_tilt(V, t["probe"], prop, t["sx"], t["sy"], t["meas"], sigma=sigma, dz=dz,
                                      binning=binning, method=method, adjoint=adjoint)
        errs.append(e)
        b = nv if method == 2 else binning
        gv = np.repeat(g, b, axis=0)[:nv]
        acc += O.rot3d(crop(gv, nv), angles[j])
        t["probe"] = (t["probe"] - step[1] * pa).astype(np.complex64)
        t["sx"] = (t["sx"] + step[2] * pd[:, 0]).astype(np.float32)
        t["sy"] = (t["sy"] + step[2] * pd[:, 1]).astype(np.float32)
    rec = rec + step[0] * acc
    if positivity:
        rec = np.maximum(rec, 0)
    if tv_lambda > 0:
        m = rec.max()
        out, _ = tv.tv_method(rec / m, tv_lambda, tv_iter, fista=tv_fista)
        rec = m * out
    return rec, np.array(errs)
