"""Golden samples of the FP64 oracle's Fourier-shear rotation of a volume
of unequal sides, MATLAB 256 x 256 x 192 (C order [192][256][256], the large
reconstruction's shape), for the GPU test in tests/test_rotation.py.  A full
oracle rotation of it takes a few minutes on the CPU, so the fixture keeps
8,192 seeded voxel samples of each result and the result's L2 norm; the test
regenerates the input volume from the same seed.

    python tests/golden/make_rot256x192_fixture.py [outfile]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

CASES = [((0.0, -70.0, 0.0), 1), ((10.0, -25.0, 40.0), 0)]  # (angles, inverse)
SHAPE = (192, 256, 256)


def volume(shape=SHAPE, seed=2562):
    """smooth blobs plus 5% uniform noise, C order [n3][n2][n1] float32"""
    rng = np.random.default_rng(seed)
    axes = [np.arange(k, dtype=np.float32) - (int(np.floor((k + 1) / 2 + 0.5)) - 1) for k in shape]
    v = np.zeros(shape, np.float32)
    for _ in range(5):
        p = rng.uniform(-min(shape) / 5, min(shape) / 5, 3).astype(np.float32)
        s = np.float32(rng.uniform(3, 6))
        gz = np.exp(-(axes[0] - p[2]) ** 2 / (2 * s * s))
        gy = np.exp(-(axes[1] - p[1]) ** 2 / (2 * s * s))
        gx = np.exp(-(axes[2] - p[0]) ** 2 / (2 * s * s))
        v += gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    v += np.float32(0.05) * rng.random(shape, dtype=np.float32)
    return v


def sample_index(shape=SHAPE, k=8192, seed=2563):
    return np.random.default_rng(seed).integers(0, int(np.prod(shape)), k)


def main(out):
    v = volume()
    idx = sample_index()
    data = {"idx": idx}
    for i, (ang, inv) in enumerate(CASES):
        r = O.rot3d(v, ang, inverse=bool(inv))
        data[f"angles{i}"] = np.array(ang)
        data[f"inverse{i}"] = inv
        data[f"values{i}"] = r.reshape(-1)[idx].astype(np.float64)
        data[f"norm{i}"] = float(np.linalg.norm(r))
    np.savez_compressed(out, **data)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "rot256x192.npz"))
