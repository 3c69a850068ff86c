"""Uneven-size batches and the autotuner (``mset_group_*``, ``mset_batch_tune``).

A group runs several tilt series of different window sizes, slab counts, scan
counts and tilt counts as one pass.  Each member's results must equal the
member's own batched pass (relative L2 <= 1e-9: only the order of the FP64
atomics differs) and the FP64 oracle (<= 1e-4).  The tuner may change only the
batch shape (persistent CTAs, checkpoint interval), never the results.
"""
import numpy as np
import pytest

import mset_b200
from mset_b200 import MSET_ADJOINT_EXACT, MSET_ADJOINT_REF, MSET_MODE_MSET
from mset_b200._lib import MSET_GROUP_CONCURRENT, MSET_GROUP_SERIAL
from mset_b200.batch import BatchSession, SeriesGroup, split_ctas
from tests.helpers import rel_l2, small_case

TOL = 1e-4
KEYS = ("grad", "probe", "posdir", "err")


# ---- host logic (no GPU) ------------------------------------------------------
def test_split_ctas_shares_every_sm():
    work = [5.0, 1.0, 0.0, 12.5, 3.0]
    occ = [2, 1, 3, 1, 4]
    g = split_ctas(work, occ, 148)
    sms = g // np.asarray(occ)
    assert (g % np.asarray(occ) == 0).all()
    assert sms.sum() == 148 and (sms >= 1).all()
    share = (sms - 1) / 143.0
    assert np.allclose(share, np.asarray(work) / sum(work), atol=1.0 / 143)


def test_split_ctas_equal_when_no_work():
    g = split_ctas([0.0, 0.0, 0.0, 0.0], [1, 1, 1, 1], 148)
    assert g.sum() == 148 and g.max() - g.min() == 0


def test_split_ctas_rejects_more_members_than_sms():
    with pytest.raises(mset_b200.MsetError, match="more members"):
        split_ctas([1.0] * 5, [1] * 5, 4)
    with pytest.raises(mset_b200.MsetError, match="occupancy"):
        split_ctas([1.0, 1.0], [1, 0], 8)


# ---- GPU ------------------------------------------------------------------------
SERIES = [  # window, depth, binning, positions per tilt, tilts, adjoint
    dict(n=64, nz=6, b=1, npos=5, tilts=3, adjoint=MSET_ADJOINT_REF),
    dict(n=96, nz=4, b=2, npos=3, tilts=1, adjoint=MSET_ADJOINT_EXACT),
    dict(n=128, nz=5, b=1, npos=4, tilts=2, adjoint=MSET_ADJOINT_REF),
    dict(n=160, nz=3, b=1, npos=2, tilts=2, adjoint=MSET_ADJOINT_REF),
]


def _series(spec, seed):
    tilts = [small_case(n=spec["n"], nz=spec["nz"], npos=spec["npos"], b=spec["b"], seed=seed + j, defocus=15.0,
                        jitter=6.0, strength=20.0) for j in range(spec["tilts"])]
    c0 = tilts[0]
    bs = BatchSession(n=spec["n"], nz=spec["nz"], npos=[spec["npos"]] * spec["tilts"], prop=c0["prop"],
                      sigma=c0["sigma"], potential_pixelsize=c0["dz"], slice_binning=spec["b"],
                      method=MSET_MODE_MSET, adjoint=spec["adjoint"])
    for j, c in enumerate(tilts):
        bs.set_tilt(j, probe=c["probe"], scan_x=c["sx"], scan_y=c["sy"], measured=c["meas"], volume=c["V"])
    return bs, tilts


def _same(a, b, tol=1e-9):
    for k in KEYS:
        assert rel_l2(a[k], b[k]) < tol, k


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [MSET_GROUP_SERIAL, MSET_GROUP_CONCURRENT], ids=["serial", "concurrent"])
@pytest.mark.parametrize("use_graph", [False, True], ids=["stream", "graph"])
def test_group_pass_equals_each_member_alone(gpu_available, schedule, use_graph):
    members = [_series(s, 100 + 10 * i) for i, s in enumerate(SERIES)]
    alone = [bs.gradient() for bs, _ in members]
    grp = SeriesGroup([bs for bs, _ in members])
    grp.set_schedule(schedule)
    for rep in range(2):  # a replayed graph gives the same results
        grp.run(use_graph=use_graph)
        for (bs, _), ref in zip(members, alone):
            _same(bs.read_gradient(), ref)
    grp.close()
    for bs, _ in members:
        bs.close()


@pytest.mark.gpu
def test_group_members_match_oracle(gpu_available):
    from oracle import oracle as O
    members = [_series(s, 300 + 10 * i) for i, s in enumerate(SERIES[:3])]
    grp = SeriesGroup([bs for bs, _ in members])
    grp.set_schedule(MSET_GROUP_CONCURRENT)
    grp.run()
    for (bs, tilts), spec in zip(members, SERIES):
        out = bs.read_gradient()
        off = 0
        for j, c in enumerate(tilts):
            g, pa, pd, e = O.batched_tilt(c["V"], c["probe"], tilts[0]["prop"], c["sx"], c["sy"], c["meas"],
                                          sigma=c["sigma"], dz=c["dz"], binning=spec["b"], adjoint=spec["adjoint"])
            assert rel_l2(out["grad"][j], g) < TOL
            assert rel_l2(np.fft.fft2(out["probe"][j]), pa) < TOL
            # scan-position directions are sums over n^2 products with
            # cancellation factors of ~1e3, so FP32 propagation resolves them to
            # a few 1e-4 (the reference's own FP32 CUDA deviates more)
            assert rel_l2(out["posdir"][off:off + spec["npos"]], pd) < 3e-4
            assert abs(out["err"][j] - e) <= TOL * e
            off += spec["npos"]
    grp.close()
    for bs, _ in members:
        bs.close()


@pytest.mark.gpu
def test_tuner_respects_budget_and_keeps_results(gpu_available):
    spec = dict(n=64, nz=48, b=1, npos=40, tilts=2, adjoint=MSET_ADJOINT_REF)
    bs, _ = _series(spec, 500)
    ref = bs.gradient()
    free = bs.tune()  # no budget: any shape
    assert free["grid"] >= 1 and free["candidates"] >= 1 and free["us_per_position"] > 0
    _same(bs.gradient(), ref)
    # a budget of 40% of the storage of every wave (49 slots per position in
    # flight) leaves k = 4 (18 slots) and k = 8 (16 slots)
    full = free["grid"] * (48 + 1) * 64 * 64 * 8
    tight = bs.tune(mem_budget_bytes=0.4 * full)
    assert tight["save_bytes"] <= 0.4 * full
    assert tight["checkpoint"] in (4, 8)
    _same(bs.gradient(), ref)
    with pytest.raises(mset_b200.MsetError, match="memory budget"):
        bs.tune(mem_budget_bytes=1024.0)
    bs.close()


@pytest.mark.gpu
def test_group_tune_picks_a_schedule_and_keeps_results(gpu_available):
    members = [_series(s, 700 + 10 * i) for i, s in enumerate(SERIES)]
    alone = [bs.gradient() for bs, _ in members]
    grp = SeriesGroup([bs for bs, _ in members])
    sched = grp.tune(mem_budget_bytes=0)
    assert sched in (MSET_GROUP_SERIAL, MSET_GROUP_CONCURRENT)
    assert grp.time(2) > 0
    grp.run()
    for (bs, _), ref in zip(members, alone):
        _same(bs.read_gradient(), ref)
    grp.close()
    for bs, _ in members:
        bs.close()


@pytest.mark.gpu
def test_group_rejects_a_repeated_member(gpu_available):
    bs, _ = _series(SERIES[0], 900)
    grp = SeriesGroup([bs])
    with pytest.raises(mset_b200.MsetError, match="already in the group"):
        mset_b200._lib.check("mset_group_add", grp._lib.mset_group_add(grp._h, bs._h))
    grp.close()
    bs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 96, 128, 160, 256])
def test_every_kernel_shape_matches_default_and_oracle(gpu_available, n):
    """the alternative thread shapes of a window (the autotuner's choices)
    give the default shape's results and the oracle's"""
    from oracle import oracle as O
    spec = dict(n=n, nz=4, b=1, npos=3, tilts=1, adjoint=MSET_ADJOINT_REF)
    bs, tilts = _series(spec, 1000 + n)
    assert bs.variants() >= 2
    outs = []
    for v in range(bs.variants()):
        bs.set_variant(v)
        outs.append(bs.gradient())
        assert bs.shape()["threads"] > 0
    with pytest.raises(mset_b200.MsetError, match="kernel shapes"):
        bs.set_variant(len(outs))
    bs.close()
    for o in outs[1:]:
        _same(o, outs[0])
    c = tilts[0]
    g, pa, pd, e = O.batched_tilt(c["V"], c["probe"], c["prop"], c["sx"], c["sy"], c["meas"], sigma=c["sigma"],
                                  dz=c["dz"], binning=1)
    assert rel_l2(outs[1]["grad"][0], g) < TOL
    assert rel_l2(np.fft.fft2(outs[1]["probe"][0]), pa) < TOL
    assert abs(outs[1]["err"][0] - e) <= TOL * e
