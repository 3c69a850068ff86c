"""TV / TV-FISTA proximal operator (func_lib/TV_method.m, TV_FISTA_method.m):
the GPU kernels against the numpy restatement (oracle/tv.py), relative
L2 <= 1e-4 on the output and 1e-4 on the TV error."""
import numpy as np
import pytest

from oracle import tv
from tests.helpers import rel_l2


def test_oracle_tv_reduces_total_variation():
    rng = np.random.default_rng(1)
    v = rng.random((12, 14, 16))
    out, err = tv.tv_method(v, 0.1, 100)
    assert tv.tv_error(out) < tv.tv_error(v)
    assert abs(err - 0.1 * tv.tv_error(out)) < 1e-12


def test_oracle_fista_converges_faster_than_plain():
    rng = np.random.default_rng(2)
    v = rng.random((10, 10, 10))
    ref, _ = tv.tv_method(v, 0.2, 2000, fista=True)
    f, _ = tv.tv_method(v, 0.2, 30, fista=True)
    p, _ = tv.tv_method(v, 0.2, 30, fista=False)
    assert rel_l2(f, ref) < rel_l2(p, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 20, 24), (32, 32, 32)])
@pytest.mark.parametrize("fista", [1, 0])
def test_gpu_tv_matches_oracle(gpu_available, shape, fista):
    from mset_b200 import Session
    from mset_b200._lib import check, dptr, fptr

    rng = np.random.default_rng(sum(shape) + fista)
    v = rng.random(shape).astype(np.float32)
    lam, niter = 0.05, 60
    ref, ref_err = tv.tv_method(v, lam, niter, fista=bool(fista))
    out = v.copy()
    err = np.zeros(1)
    with Session() as s:
        check("mset_tv", s._lib.mset_tv(s._h, fptr(out), shape[2], shape[1], shape[0], lam, niter, fista, dptr(err)))
    assert rel_l2(out, ref) < 1e-4
    assert abs(err[0] - ref_err) <= 1e-4 * ref_err
