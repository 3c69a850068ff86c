"""numpy restatement of the reference's TV proximal operators, 3D case
(func_lib/TV_method.m:5-28, helpers :32-83; func_lib/TV_FISTA_method.m:5-38).

TEST INFRASTRUCTURE ONLY.  Arrays are C order [n3][n2][n1] = MATLAB
(n1, n2, n3); MATLAB circshift along dim 1 is np.roll along axis 2.
"""
import numpy as np

_AX = {1: 2, 2: 1, 3: 0}  # MATLAB dim -> numpy axis


def tv_div(P):
    """TV_div (TV_method.m:43-56): P1+P2+P3 - circshift(P1,[1 0 0]) - ..."""
    out = P[0] + P[1] + P[2]
    for k in range(3):
        out = out - np.roll(P[k], 1, axis=_AX[k + 1])
    return out


def tv_del(u):
    """TV_del (TV_method.m:58-69): -u + circshift(u, -e_k)"""
    return np.stack([np.roll(u, -1, axis=_AX[k + 1]) - u for k in range(3)])


def tv_project(P):
    return P / np.sqrt(np.maximum(1.0, P[0] ** 2 + P[1] ** 2 + P[2] ** 2))


def tv_error(u):
    d = tv_del(u)
    return float(np.sum(np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)))


def tv_method(inp, lam, niter, fista=True):
    """TV_FISTA_method (fista=True) or TV_method (fista=False); returns
    (output, error) in FP64."""
    inp = np.asarray(inp, dtype=np.float64)
    tau = 1.0 / 12
    P = np.zeros((3,) + inp.shape)
    Y = P.copy()
    t = 1.0
    for _ in range(niter):
        P0 = P
        t0 = t
        src = Y if fista else P
        temp = tau * tv_del(tv_div(src) - inp / lam)
        P = tv_project(src + temp)
        if fista:
            t = (1 + np.sqrt(1 + 4 * t0 ** 2)) / 2
            Y = P + ((t0 - 1) / t) * (P - P0)
    out = inp - lam * tv_div(P)
    return out, lam * tv_error(out)
