"""The FP64 oracle as a backend of mset_b200.recon.reconstruct (test use)."""
from oracle import oracle as O


class OracleBackend:
    def rotate(self, vol, angles, inverse):
        return O.rot3d(vol, angles, inverse=inverse)

    def run_tilt(self, V, t, prop, *, sigma, dz, step, binning, method):
        rv, pr, sx, sy, _ = O.run_tilt(V, t.probe, prop, t.scan_x, t.scan_y, t.measured, sigma=sigma, dz=dz,
                                       step=step, binning=binning, method=method)
        return rv, pr, sx, sy

    def error_tilt(self, V, t, prop, *, sigma, dz, binning, method):
        _, _, _, _, e = O.run_tilt(V, t.probe, prop, t.scan_x, t.scan_y, t.measured, sigma=sigma, dz=dz,
                                   binning=binning, method=method, update=False)
        return e / t.measured.shape[0] / t.measured[0].size

    def tv(self, vol, lam, niter, fista=False):
        from oracle import tv
        out, _ = tv.tv_method(vol, lam, niter, fista=fista)
        return out
