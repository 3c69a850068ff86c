"""Host logic of the reconstruction loop (mset_b200.recon.reconstruct,
Run_MSET_recon.m:106-287) with a scripted backend: accept / reject decisions
of the backtracking line search, state restore, step reduction, early stop,
positivity and TV placement."""
import numpy as np

from mset_b200.recon import Tilt, reconstruct


class Scripted:
    """Each update adds `step0` to every voxel of a tilt's volume; the error
    pass returns the next value of a script (per tilt the same)."""

    def __init__(self, errors):
        self.errors = list(errors)
        self.calls = []

    def rotate(self, vol, angles, inverse):
        return np.array(vol, copy=True)

    def run_tilt(self, V, t, prop, *, sigma, dz, step, binning, method):
        self.calls.append(("run", float(step[0])))
        return V + np.float32(step[0]), t.probe, t.scan_x, t.scan_y

    def error_tilt(self, V, t, prop, *, sigma, dz, binning, method):
        self.calls.append(("err", None))
        return self.errors[0]

    def next_trial(self):
        self.errors.pop(0)

    def tv(self, vol, lam, niter, fista=False):
        self.calls.append(("tv", lam))
        return vol * 0.5


def _tilts(J=2):
    n = 4
    return [Tilt(np.ones((n, n), np.complex64), np.ones(1, np.float32), np.ones(1, np.float32),
                 np.zeros((1, n, n), np.float32)) for _ in range(J)]


class Stepper(Scripted):
    def error_tilt(self, V, t, prop, **kw):
        e = super().error_tilt(V, t, prop, **kw)
        self.k = getattr(self, "k", 0) + 1
        if self.k % 2 == 0:  # both tilts evaluated: the trial is over
            self.next_trial()
        return e


def test_line_search_accepts_rejects_and_restores():
    # trial errors: 5 (accept, first), 6 (reject), 7 (reject), 3 (accept)
    be = Stepper([5.0, 6.0, 7.0, 3.0])
    r = reconstruct(be, np.zeros((2, 2, 2), np.float32), _tilts(), None, [(0, 0, 0)] * 2, sigma=1.0, dz=1.0,
                    step=[1.0, 0, 0], n_iter=2, bls_parameter=0.5, positivity=False)
    assert r.mean_error == [5.0, 3.0]
    # iteration 1: +1 per tilt; iteration 2 accepted at step 0.25: +0.25 per tilt
    assert np.allclose(r.rec_per_iter[0], 2.0) and np.allclose(r.rec, 2.5)
    assert np.allclose(r.step, [0.25, 0, 0])
    steps = [s for k, s in be.calls if k == "run"]
    assert steps == [1.0, 1.0, 1.0, 1.0, 0.5, 0.5, 0.25, 0.25]


def test_line_search_stops_below_fifth_power():
    be = Stepper([5.0] + [9.0] * 10)
    r = reconstruct(be, np.zeros((2, 2, 2), np.float32), _tilts(), None, [(0, 0, 0)] * 2, sigma=1.0, dz=1.0,
                    step=[1.0, 0, 0], n_iter=3, bls_parameter=0.5, positivity=False)
    assert r.stopped_early and r.mean_error == [5.0]
    assert np.allclose(r.rec, 2.0)  # the rejected trials were undone
    assert np.isclose(r.step[0], 0.5 ** 6)


def test_positivity_and_tv_after_acceptance():
    be = Stepper([5.0, 4.0])
    r = reconstruct(be, np.full((2, 2, 2), -10.0, np.float32), _tilts(1), None, [(0, 0, 0)], sigma=1.0, dz=1.0,
                    step=[1.0, 0, 0], n_iter=1, bls_parameter=0.5, positivity=True)
    assert np.all(r.rec == 0)  # -10 + 1, then rec(rec < 0) = 0
    be = Stepper([5.0, 4.0])
    r = reconstruct(be, np.ones((2, 2, 2), np.float32), _tilts(1), None, [(0, 0, 0)], sigma=1.0, dz=1.0,
                    step=[1.0, 0, 0], n_iter=1, bls_parameter=0.5, use_tv=True, tv_lambda=0.1)
    # TV of rec / max(rec), rescaled by max(rec), once, after the accepted update
    assert [c for c in be.calls if c[0] == "tv"] == [("tv", 0.1)]
    assert np.allclose(r.rec, 1.0)
