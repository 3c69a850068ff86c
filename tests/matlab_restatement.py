"""numpy restatement of the reference's MATLAB per-position code in its own
(centred, fftshift-wrapped) convention: STEP02_FORWARD_4D.m:6-51,
STEP03_BACK.m:6-39, Func_generate_probe_wave_scan_sub_pixel.m:4-27.

Used to check that the FP64 oracle (which follows the CUDA module's
unshifted convention) computes the same quantities.  Arrays are C order
[dim2][dim1] of the MATLAB arrays.
"""
import numpy as np

fftshift, ifftshift = np.fft.fftshift, np.fft.ifftshift


def sub_pixel_shift(p0, x1, y1, pi=np.pi):
    ny, nx = p0.shape[1], p0.shape[0]  # MATLAB size(p0,1) = dim1 = C columns
    cent = np.floor((np.array([p0.shape[1], p0.shape[0]]) + 1) / 2 + 0.5)
    dx, dy = x1 - cent[0], y1 - cent[1]
    X = (np.arange(p0.shape[1]) - ny / 2)[None, :]   # varies along dim1 (C columns)
    Y = (np.arange(p0.shape[0]) - nx / 2)[:, None]   # varies along dim2 (C rows)
    F = np.fft.fft2(p0)
    P = np.exp(-2j * pi * (dx * X / nx + dy * Y / ny))
    return np.fft.ifft2(F * ifftshift(P))


def step02_step03(V, probe, prop, row, col, meas_centred, sigma, dz, b, pi=np.pi):
    nz = V.shape[0]
    ns = -(-nz // b)
    potz = np.stack([V[s * b:min((s + 1) * b, nz)].sum(0) * dz for s in range(ns)])
    trans = np.exp(1j * sigma * potz)
    tmp_probe = sub_pixel_shift(probe, row, col, pi)
    w = tmp_probe
    save = []
    for s in range(ns):
        w = fftshift(np.fft.fft2(ifftshift(w * trans[s]))) * prop
        w = fftshift(np.fft.ifft2(ifftshift(w)))
        save.append(w)
    w = fftshift(np.fft.fft2(ifftshift(w)))
    calc = np.abs(w) ** 2
    resi = w * (1 - np.sqrt(meas_centred) / np.sqrt(calc + 1e-30))
    err = np.sum((np.sqrt(meas_centred) - np.sqrt(calc)) ** 2)
    back_prop = np.conj(prop)
    bw = resi
    grad = np.zeros((ns,) + V.shape[1:], complex)
    for s in range(ns - 1, -1, -1):
        bw = fftshift(np.fft.ifft2(ifftshift(bw * back_prop)))
        grad[s] = 1j * np.conj(trans[s]) * np.conj(save[s]) * bw
        bw = fftshift(np.fft.fft2(ifftshift(bw * np.conj(trans[s]))))
    bw = fftshift(np.fft.ifft2(ifftshift(bw)))
    cent = np.floor((np.array([probe.shape[1], probe.shape[0]]) + 1) / 2 + 0.5)
    shift = 2 * cent - np.array([row, col])
    probe_dir = sub_pixel_shift(bw, shift[0], shift[1], pi)
    cp = np.conj(tmp_probe)
    # MATLAB [FX, FY] = gradient(A): FX along dim2 (C rows), FY along dim1 (C columns)
    de_x = np.gradient(cp, axis=1)   # along dim1 -> "de_probex"
    de_y = np.gradient(cp, axis=0)   # along dim2 -> "de_probey"
    pos = np.array([np.real(np.sum(de_x * bw)), np.real(np.sum(de_y * bw))])
    return dict(calc=calc, err=err, grad=grad, chi0=bw, probe_dir=probe_dir, pos_dir=pos, psi0=tmp_probe,
                waves=np.stack(save))
