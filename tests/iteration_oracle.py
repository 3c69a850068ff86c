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
    """[nv3][nv2][nv1] volume centred laterally in the n x n window"""
    nv3, nv2, nv1 = v.shape
    o2, o1 = (n - nv2) // 2, (n - nv1) // 2
    out = np.zeros((nv3, n, n), v.dtype)
    out[:, o2:o2 + nv2, o1:o1 + nv1] = v
    return out


def crop(g, shape):
    """the [nv3][nv2][nv1] part of a window-sized [*][n][n] array; shape: the
    volume's shape, or its edge for a cubic one"""
    nv3, nv2, nv1 = (shape,) * 3 if np.isscalar(shape) else shape
    n = g.shape[1]
    o2, o1 = (n - nv2) // 2, (n - nv1) // 2
    return g[:nv3, o2:o2 + nv2, o1:o1 + nv1]


def iterate(rec, tilts, prop, angles, *, sigma, dz, binning, step, positivity=True, tv_lambda=0.0, tv_iter=0,
            tv_fista=True, method=1, adjoint=0):
    """tilts: list of dicts with probe, sx, sy, meas (updated in place).
    Returns (rec, errs)."""
    nv = rec.shape[0]
    acc = np.zeros(rec.shape)
    errs = []
    for j, t in enumerate(tilts):
        n = t["probe"].shape[0]
        V = pad(O.rot3d(rec, angles[j], inverse=True), n).astype(np.float32)
        g, pa, pd, e = O.batched_tilt(V, t["probe"], prop, t["sx"], t["sy"], t["meas"], sigma=sigma, dz=dz,
                                      binning=binning, method=method, adjoint=adjoint)
        errs.append(e)
        b = nv if method == 2 else binning
        gv = np.repeat(g, b, axis=0)[:nv]
        acc += O.rot3d(crop(gv, rec.shape), angles[j])
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


def tilt_errors(rec, tilts, prop, angles, *, sigma, dz, binning, method=1):
    """error pass of a state: per tilt the sum of (A - M)^2 over positions and
    pixels (run_error_mset, oracle forward)"""
    out = []
    for j, t in enumerate(tilts):
        n = t["probe"].shape[0]
        V = pad(O.rot3d(rec, angles[j], inverse=True), n).astype(np.float32)
        _, _, _, e = O.batched_tilt(V, t["probe"], prop, t["sx"], t["sy"], t["meas"], sigma=sigma, dz=dz,
                                    binning=binning, method=method)
        out.append(e)
    return np.array(out)


def iterate_bls(rec, tilts, prop, angles, *, sigma, dz, binning, step, bls, niter, positivity=True, tv_lambda=0.0,
                tv_iter=0, tv_fista=True, method=1, adjoint=0):
    """Iterations with the backtracking line search of Run_MSET_recon.m:106-252:
    an update (no TV) is kept only if the mean error of the new state is below
    the previous iteration's (1e31 at the start); else the state is restored
    and every step size multiplied by bls, until the object step falls below
    bls^5 times its starting value.  TV follows an accepted update.  Step
    sizes are float32 as in the library.  Returns (rec, tilts, mean errors,
    step sizes) of the accepted iterations."""
    step = [np.float32(x) for x in step]
    floor0 = bls ** 5 * float(step[0])
    old = 1e31
    errs, steps = [], []
    for _ in range(niter):
        stop = False
        while True:
            tl = [dict(t) for t in tilts]
            new, _ = iterate(rec, tl, prop, angles, sigma=sigma, dz=dz, binning=binning, step=step,
                             positivity=positivity, method=method, adjoint=adjoint)
            e = tilt_errors(new, tl, prop, angles, sigma=sigma, dz=dz, binning=binning, method=method)
            mean = float(np.mean([e[j] / t["meas"].shape[0] / t["meas"][0].size for j, t in enumerate(tl)]))
            if old > mean:
                rec, tilts = new, tl
                break
            step = [np.float32(bls * float(x)) for x in step]
            if float(step[0]) < floor0:
                stop = True
                break
        if stop:
            break
        if tv_lambda > 0:
            m = rec.max()
            out, _ = tv.tv_method(rec / m, tv_lambda, tv_iter, fista=tv_fista)
            rec = m * out
        errs.append(mean)
        steps.append([float(x) for x in step])
        old = mean
    return rec, tilts, np.array(errs), np.array(steps)
