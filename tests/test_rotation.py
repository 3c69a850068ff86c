"""Fourier-shear tilt rotation (func_lib/Func_rot_3Dvol_FourierShear.m,
Func_inv_rot_3Dvol_FourierShear.m, Func_rotate_3Dvol_ROTmat_FourierShear.m).

CPU: the FP64 oracle restatement moves a Gaussian blob as the rotation it
encodes (the reference's Func_rot with theta about vec2 = y maps (x,0,0) to
(x cos t, 0, -x sin t)), its inverse undoes it, and angles within 0.5 deg are
a no-op (Func_rot_3Dvol_FourierShear.m:14-18).
GPU: the library's shear kernels against the oracle, relative L2 <= 1e-4."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2


def _grid(n):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    c = int(np.floor((n + 1) / 2 + 0.5)) - 1
    return x - c, y - c, z - c


def _blob(n, p, s=1.5):
    x, y, z = _grid(n)
    return np.exp(-((x - p[0]) ** 2 + (y - p[1]) ** 2 + (z - p[2]) ** 2) / (2 * s * s))


def _centroid(v):
    x, y, z = _grid(v.shape[0])
    w = np.clip(v, 0, None)
    return np.array([(w * x).sum(), (w * y).sum(), (w * z).sum()]) / w.sum()


@pytest.mark.parametrize("angles,expect", [
    ((0, 30, 0), (6 * np.cos(np.pi / 6), 0, -6 * np.sin(np.pi / 6))),
    ((0, -50, 0), (6 * np.cos(np.pi * 50 / 180), 0, 6 * np.sin(np.pi * 50 / 180))),
    ((40, 0, 0), (6 * np.cos(np.pi * 40 / 180), 6 * np.sin(np.pi * 40 / 180), 0)),
])
def test_oracle_rotation_moves_blob(angles, expect):
    v = _blob(32, (6, 0, 0))
    r = O.rot3d(v, angles)
    assert np.allclose(_centroid(r), expect, atol=0.02)
    back = O.rot3d(r, angles, inverse=True)
    assert rel_l2(back, v) < 1e-3


def test_small_angles_are_identity():
    v = np.random.default_rng(0).random((24, 24, 24))
    assert np.array_equal(O.rot3d(v, (0.2, -0.4, 0.5)), v)


def test_rotation_plan_substeps():
    M, act = O.rotation_matrix((0, 60, 0), inverse=True)
    plan = O.rotation_plan(M)
    assert act and plan["num_step"] == 6  # floor(60 / 11) + 1


@pytest.mark.gpu
@pytest.mark.parametrize("n", [24, 32, 64])
@pytest.mark.parametrize("angles", [(0, 30, 0), (0, -60, 0), (10, -25, 40)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_gpu_rotation_matches_oracle(gpu_available, n, angles, inverse):
    import mset_b200
    from mset_b200 import Session
    from mset_b200._lib import check, fptr

    rng = np.random.default_rng(n)
    # smooth random volume (a few blobs) plus noise
    v = sum(_blob(n, rng.uniform(-n / 5, n / 5, 3), s=rng.uniform(1, 2)) for _ in range(5))
    v = (v + 0.05 * rng.random(v.shape)).astype(np.float32)
    ref = O.rot3d(v, angles, inverse=bool(inverse))
    out = np.empty_like(v)
    vecs = [np.asarray(x, np.float32) for x in (O.VEC1, O.VEC2, O.VEC3)]
    with Session() as s:
        check("mset_rotate_volume", s._lib.mset_rotate_volume(s._h, fptr(v), fptr(out), n, fptr(vecs[0]),
                                                               fptr(vecs[1]), fptr(vecs[2]), float(angles[0]),
                                                               float(angles[1]), float(angles[2]), inverse))
    assert rel_l2(out, ref) < 1e-4


@pytest.mark.gpu
def test_gpu_rotation_256_cluster_matches_oracle_samples(gpu_available):
    """256^3: every plane split over a 4-CTA cluster; checked on 8,192 seeded
    voxels of the FP64 oracle's result (tests/golden/make_rot256_fixture.py)"""
    import os

    from mset_b200 import Session
    from tests.golden.make_rot256_fixture import volume

    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "rot256.npz"))
    v = volume()
    with Session() as s:
        for i in range(2):
            out = s.rotate_volume(v, f[f"angles{i}"], inverse=bool(f[f"inverse{i}"]))
            vals = out.reshape(-1)[f["idx"]]
            assert rel_l2(vals, f[f"values{i}"]) < 1e-4
