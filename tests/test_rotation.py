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


def _grid3(shape):
    z, y, x = np.meshgrid(*[np.arange(k) for k in shape], indexing="ij")
    c = [int(np.floor((k + 1) / 2 + 0.5)) - 1 for k in shape]
    return x - c[2], y - c[1], z - c[0]


def _blob3(shape, p, s=1.5):
    x, y, z = _grid3(shape)
    return np.exp(-((x - p[0]) ** 2 + (y - p[1]) ** 2 + (z - p[2]) ** 2) / (2 * s * s))


@pytest.mark.parametrize("shape", [(32, 40, 48), (48, 40, 32)])
def test_oracle_rotation_of_a_non_cubic_volume_moves_blob(shape):
    """unequal sides: the reference's shear phase along x is
    exp(i 2 pi (a n_y + b n_z) n_x / N_x) (SheerTransforms_for3Drot.m:29-31),
    i.e. the shift of axis a per voxel of the shear axis d is scaled by
    N_a / N_d: the volume turns in coordinates normalised by each side, so a
    blob at x = 6 turned by 30 deg about y lands at x = 6 cos 30,
    z = -6 sin 30 N_z / N_x.  The FP64 restatement does that, and its inverse
    undoes it"""
    n3, n2, n1 = shape  # C order [n3][n2][n1]
    v = _blob3(shape, (6, 0, 0))
    r = O.rot3d(v, (0, 30, 0))
    x, y, z = _grid3(shape)
    w = np.clip(r, 0, None)
    cen = np.array([(w * x).sum(), (w * y).sum(), (w * z).sum()]) / w.sum()
    assert np.allclose(cen, (6 * np.cos(np.pi / 6), 0, -6 * np.sin(np.pi / 6) * n3 / n1), atol=0.02)
    assert rel_l2(O.rot3d(r, (0, 30, 0), inverse=True), v) < 1e-3


def _smooth(shape, seed):
    rng = np.random.default_rng(seed)
    v = sum(_blob3(shape, rng.uniform(-min(shape) / 5, min(shape) / 5, 3), s=rng.uniform(1, 2)) for _ in range(5))
    return (v + 0.05 * rng.random(shape)).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(48, 32, 24), (24, 32, 64), (32, 64, 64)], ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("angles", [(0, 30, 0), (10, -25, 40)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_gpu_rotation_of_non_cubic_volumes_matches_oracle(gpu_available, shape, angles, inverse):
    """volumes of unequal sides: every shear as batched line transforms on
    the GPU (mset_rotate_volume_nd) against the FP64 oracle"""
    from mset_b200 import Session
    v = _smooth(shape, sum(shape))
    ref = O.rot3d(v, angles, inverse=bool(inverse))
    with Session() as s:
        out = s.rotate_volume(v, angles, inverse=bool(inverse))
    assert rel_l2(out, ref) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("n", [24, 64, 160])
def test_gpu_line_rotation_of_a_cubic_volume_equals_plane_rotation(gpu_available, n):
    """the line kernels and the plane kernels compute the same rotation"""
    from mset_b200 import Session
    v = _smooth((n, n, n), n)
    with Session() as s:
        planes = s.rotate_volume(v, (10, -25, 40))
        lines = s.rotate_volume(v, (10, -25, 40), lines=True)
    assert rel_l2(lines, planes) < 1e-5


@pytest.mark.gpu
def test_gpu_rotation_256x256x192_matches_oracle_samples(gpu_available):
    """the large reconstruction's shape (MATLAB 256 x 256 x 192), line
    transforms of 256 and 192 points, against 8,192 seeded voxels of the FP64
    oracle's result (tests/golden/make_rot256x192_fixture.py)"""
    import os

    from mset_b200 import Session
    from tests.golden.make_rot256x192_fixture import volume

    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "rot256x192.npz"))
    v = volume()
    with Session() as s:
        for i in range(2):
            out = s.rotate_volume(v, f[f"angles{i}"], inverse=bool(f[f"inverse{i}"]))
            assert rel_l2(out.reshape(-1)[f["idx"]], f[f"values{i}"]) < 1e-4
            assert abs(np.linalg.norm(out) - f[f"norm{i}"]) <= 1e-4 * f[f"norm{i}"]
