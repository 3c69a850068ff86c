"""Golden samples of the FP64 oracle's Fourier-shear rotation of a 256^3
volume (the cluster-split shear kernels' size), for the GPU test in
tests/test_rotation.py.  A full 256^3 oracle rotation takes minutes on the
CPU, so the fixture keeps 8,192 seeded voxel samples of each result and the
result's L2 norm; the test regenerates the input volume from the same seed.

    python tests/golden/make_rot256_fixture.py [outfile]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

CASES = [((0.0, 30.0, 0.0), 1), ((10.0, -25.0, 40.0), 0)]  # (angles, inverse)
N = 256


def volume(n=N, seed=2560):
    """smooth blobs plus 5% uniform noise, C order [n][n][n] float32"""
    rng = np.random.default_rng(seed)
    c = int(np.floor((n + 1) / 2 + 0.5)) - 1
    ax = np.arange(n, dtype=np.float32) - c
    v = np.zeros((n, n, n), np.float32)
    for _ in range(5):
        p = rng.uniform(-n / 5, n / 5, 3).astype(np.float32)
        s = np.float32(rng.uniform(3, 6))
        gx = np.exp(-(ax - p[0]) ** 2 / (2 * s * s))
        gy = np.exp(-(ax - p[1]) ** 2 / (2 * s * s))
        gz = np.exp(-(ax - p[2]) ** 2 / (2 * s * s))
        v += gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    v += np.float32(0.05) * rng.random((n, n, n), dtype=np.float32)
    return v


def sample_index(n=N, k=8192, seed=2561):
    return np.random.default_rng(seed).integers(0, n ** 3, k)


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
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "rot256.npz"))
