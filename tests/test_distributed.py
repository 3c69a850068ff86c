"""Tilt sharding of the batched iteration (mset_b200/distributed.py) with
world size 2 on CPU (gloo): two ranks each run phase 1 on half of the tilts
with the FP64 oracle, all-reduce the lab-frame gradient, run phase 2 (update,
positivity and TV-FISTA of rec / max(rec), rescaled, as the device
iteration's phase 2), and end with the same volume, probes and positions as
one process over all tilts."""
import os

import numpy as np
import pytest

from mset_b200.distributed import sharded_iterate, tilt_shard


def test_tilt_shard_covers_and_balances():
    for n in (1, 5, 21, 64):
        for w in (1, 2, 3, 8):
            parts = [tilt_shard(n, w, r) for r in range(w)]
            assert sum(parts, []) == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


class OracleBackend:
    """phase 1 / phase 2 of tests/iteration_oracle.iterate, on CPU tensors"""

    def __init__(self, prob, tilt_ids, step):
        import torch

        from tests import iteration_oracle as IO  # noqa: F401
        self.p = prob
        self.ids = tilt_ids
        self.step = step
        self.rec = prob["rec0"].astype(np.float64).copy()
        self.tilts = {j: dict(prob["tilts"][j]) for j in tilt_ids}
        self.g = torch.zeros(self.rec.size, dtype=torch.float64)

    def phase1(self):
        from oracle import oracle as O
        from tests import iteration_oracle as IO
        p = self.p
        nv = self.rec.shape[0]
        acc = np.zeros_like(self.rec)
        self._pa, self._pd = {}, {}
        for j in self.ids:
            t = self.tilts[j]
            n = t["probe"].shape[0]
            V = IO.pad(O.rot3d(self.rec, p["angles"][j], inverse=True), n).astype(np.float32)
            g, pa, pd, _ = O.batched_tilt(V, t["probe"], p["prop"], t["sx"], t["sy"], t["meas"], sigma=p["sigma"],
                                          dz=p["dz"], binning=p["b"])
            gv = np.repeat(g, p["b"], axis=0)[:nv]
            acc += O.rot3d(IO.crop(gv, nv), p["angles"][j])
            self._pa[j], self._pd[j] = pa, pd
        self.g.copy_(__import__("torch").from_numpy(acc.ravel()))

    def gradient(self):
        return self.g

    def stream(self):
        import contextlib
        return contextlib.nullcontext()

    def phase2(self):
        from oracle import tv
        s = self.step
        self.rec = np.maximum(self.rec + s[0] * self.g.numpy().reshape(self.rec.shape), 0)
        if TV_LAMBDA > 0:
            m = self.rec.max()  # Run_MSET_recon.m:267-270
            out, _ = tv.tv_method(self.rec / m, TV_LAMBDA, TV_ITER, fista=True)
            self.rec = m * out
        for j in self.ids:
            t = self.tilts[j]
            t["probe"] = (t["probe"] - s[1] * self._pa[j]).astype(np.complex64)
            t["sx"] = (t["sx"] + s[2] * self._pd[j][:, 0]).astype(np.float32)
            t["sy"] = (t["sy"] + s[2] * self._pd[j][:, 1]).astype(np.float32)


def _problem():
    from tests.test_gpu_iteration import _problem as mk
    nv, n, b, dz, sigma, prop, angles, tilts, rec0 = mk(seed=9)
    return dict(nv=nv, n=n, b=b, dz=dz, sigma=sigma, prop=prop, angles=angles, tilts=tilts, rec0=rec0)


STEP = (1e-3, 1e-6, 1e-2)
TV_LAMBDA, TV_ITER = 1e-3, 20


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        prob = _problem()
        be = OracleBackend(prob, tilt_shard(len(prob["angles"]), world, rank), STEP)
        sharded_iterate(be, 2)
        np.save(os.path.join(out, f"rec{rank}.npy"), be.rec)
        for j, t in be.tilts.items():
            np.save(os.path.join(out, f"probe{j}.npy"), t["probe"])
            np.save(os.path.join(out, f"pos{j}.npy"), np.r_[t["sx"], t["sy"]])
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_iteration_equals_single_process(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    prob = _problem()
    single = OracleBackend(prob, list(range(len(prob["angles"]))), STEP)
    sharded_iterate(single, 2, world=1)
    for r in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"rec{r}.npy"), single.rec, rtol=1e-10, atol=1e-12)
    for j, t in single.tilts.items():
        np.testing.assert_allclose(np.load(tmp_path / f"probe{j}.npy"), t["probe"], rtol=1e-6, atol=1e-9)
        np.testing.assert_allclose(np.load(tmp_path / f"pos{j}.npy"), np.r_[t["sx"], t["sy"]], rtol=1e-6)
