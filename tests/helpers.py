"""Small seeded cases shared by the tests."""
import numpy as np

from mset_b200 import physics


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)


def small_case(n=24, nz=6, npos=4, b=1, seed=0, strength=1.0, defocus=0.0, dx=0.4, E0=300e3, jitter=1.5,
               consistent=True):
    """Random weak-phase volume V (the current estimate), aberrated probe,
    scan positions around the centre, and measured intensities.

    consistent=True: measured = Poisson(|Psi|^2) of a perturbed "true" volume
    (FP64 oracle forward model), as real data are; pixels the model predicts
    dark then measure ~0.  consistent=False: uniform random patterns, which
    make the residual phase at dark pixels ill-conditioned in FP32."""
    rng = np.random.default_rng(seed)
    lam = physics.electron_wavelength(E0)
    sigma = physics.interaction_constant(E0)
    V = (rng.random((nz, n, n)) * 3.0 * strength).astype(np.float32)
    probe = physics.probe_wave(n, dx, lam, 20.0, C10=defocus)
    probe = physics.normalise_probe(probe, 1e4).astype(np.complex64)
    prop = physics.propagator(n, dx, lam, b)
    c = np.floor((n + 1) / 2 + 0.5)
    sx = (c + rng.uniform(-jitter, jitter, npos)).astype(np.float32)
    sy = (c + rng.uniform(-jitter, jitter, npos)).astype(np.float32)
    if consistent:
        # the "true" specimen differs from the current estimate in all three
        # unknowns: volume (x U[0.5, 1.5]), probe (defocus + 30 A) and scan
        # positions (+-0.5 px), so every gradient carries signal
        from oracle import oracle as O
        Vt = V * rng.uniform(0.5, 1.5, V.shape).astype(np.float32)
        pt = physics.normalise_probe(physics.probe_wave(n, dx, lam, 20.0, C10=defocus + 30.0), 1e4)
        sxt = sx + rng.uniform(-0.5, 0.5, npos)
        syt = sy + rng.uniform(-0.5, 0.5, npos)
        meas = np.empty((npos, n, n), np.float32)
        for p in range(npos):
            o = O.position(Vt, pt, prop, sxt[p], syt[p], np.zeros((n, n)), sigma=sigma, dz=dx, binning=b)
            meas[p] = rng.poisson(np.fft.fftshift(np.abs(o["far"]) ** 2)).astype(np.float32)
    else:
        meas = (rng.random((npos, n, n)) * 50.0).astype(np.float32)
    return dict(V=V, probe=probe, prop=prop, sx=sx, sy=sy, meas=meas, sigma=float(sigma), dz=dx, b=b,
                lam=lam)


def reasonable_steps(c, method=1, admode=0, frac=(0.05, 0.01, 0.1)):
    """Step sizes (object, probe, position) that move the state by a given
    fraction per position, measured on the first position with the FP64
    oracle: ~5% of max|V|, ~1% of max|probe| and ~0.1 px.  Updates much
    smaller than the FP32 state they are added to would be lost to rounding
    (a probe step of 1e-4 |probe| is resolved to only ~1e-3 of itself)."""
    from oracle import oracle as O
    o = O.position(c["V"], c["probe"], c["prop"], c["sx"][0], c["sy"][0], O.amp_std(c["meas"][0]),
                   sigma=c["sigma"], dz=c["dz"], binning=c["b"], method=method, adjoint=admode)
    s0 = frac[0] * np.abs(c["V"]).max() / max(np.abs(o["grad"].real).max(), 1e-30)
    s1 = frac[1] * np.abs(c["probe"]).max() / max(np.abs(o["probe_dir"]).max(), 1e-30)
    s2 = frac[2] / max(np.abs(o["pos_dir"]).max(), 1e-30)
    return (float(s0), float(s1), float(s2))
