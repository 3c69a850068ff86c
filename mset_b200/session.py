"""Host-side mirror of the reference's MEX interface (src/CUDA/mex_main.cu).

Two layers:

* :class:`Session` -- an explicit handle over the C ABI with C-order numpy
  arrays (volume ``[nz][n][n]`` float32, probe ``[n][n]`` complex64, measured
  ``[P][n][n]`` float32 in the reference's centred layout);
* :func:`mset_cuda_kernel` -- the reference's call signature
  ``mset_cuda_kernel(mode, STEM_data, measured_cells)`` with MATLAB-shaped
  arrays (``RVol`` of shape ``(n, n, nz)``, the measured cell array of shape
  ``(N_scan_x, N_scan_y)``), one implicit session per process as the MEX keeps
  one (mex_main.cu:13).

Errors raise :class:`mset_b200._lib.MsetError`; nothing aborts.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Mapping, Sequence

import numpy as np

from . import _lib
from ._lib import MSET_ADJOINT_EXACT, MSET_ADJOINT_REF, MSET_MODE_MSET, MSET_MODE_SSET, check, fptr

_MODES = {"mset": MSET_MODE_MSET, "sset": MSET_MODE_SSET}


def _c32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _cplx_f32(a) -> np.ndarray:
    """complex array -> float32 [..., 2] interleaved view"""
    z = np.ascontiguousarray(np.asarray(a, dtype=np.complex64))
    return z.view(np.float32).reshape(z.shape + (2,))


class Session:
    """One device session: the state the MEX keeps between 'upload' and
    'run_*' / 'error_*' calls, but with device buffers reused across uploads."""

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        check("mset_create", self._lib.mset_create(int(device), C.byref(h)))
        self._h = h
        self._keep: list = []
        self.n = self.nz = self.npos = 0
        self._binning = 1

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mset_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- volume operations of the reconstruction loop ----
    def rotate_volume(self, vol, angles, *, inverse: bool = False, vec1=(0, 0, 1), vec2=(0, 1, 0),
                      vec3=(1, 0, 0), lines: bool = False) -> np.ndarray:
        """Func_rot_3Dvol_FourierShear / Func_inv_rot_3Dvol_FourierShear of a
        [n3][n2][n1] volume by (phi, theta, psi) degrees: mset_rotate_volume
        (plane kernels) for a cubic volume, mset_rotate_volume_nd (line
        kernels) for any other shape, or for a cubic one with lines=True"""
        v = _c32(vol)
        if v.ndim != 3:
            raise ValueError(f"3D volume expected, got {v.shape}")
        n3, n2, n1 = v.shape
        out = np.empty_like(v)
        vecs = [np.ascontiguousarray(np.asarray(x, np.float32)) for x in (vec1, vec2, vec3)]
        a = [float(x) for x in angles]
        if n1 == n2 == n3 and not lines:
            check("mset_rotate_volume", self._lib.mset_rotate_volume(self._h, fptr(v), fptr(out), n1, fptr(vecs[0]),
                                                                     fptr(vecs[1]), fptr(vecs[2]), a[0], a[1], a[2],
                                                                     int(bool(inverse))))
        else:
            check("mset_rotate_volume_nd",
                  self._lib.mset_rotate_volume_nd(self._h, fptr(v), fptr(out), n1, n2, n3, fptr(vecs[0]),
                                                  fptr(vecs[1]), fptr(vecs[2]), a[0], a[1], a[2], int(bool(inverse))))
        return out

    def tv(self, vol, lam: float, niter: int, fista: bool = False):
        """TV_method (fista=False) / TV_FISTA_method of a [n3][n2][n1] volume
        (mset_tv); returns the regularised volume"""
        out = np.array(_c32(vol), dtype=np.float32, copy=True)
        n3, n2, n1 = out.shape
        err = np.zeros(1)
        check("mset_tv", self._lib.mset_tv(self._h, fptr(out), n1, n2, n3, float(lam), int(niter), int(bool(fista)),
                                           err.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    # ---- 'upload' (mex_main.cu:42-95) ----
    def upload(self, rvol, probe, prop, *, sigma: float, potential_pixelsize: float,
               scan_x, scan_y, measured, step_size=(0.0, 0.0, 0.0), slice_binning: int = 1,
               n_scan_x: int | None = None, n_scan_y: int | None = None) -> None:
        rvol = _c32(rvol)
        if rvol.ndim != 3:
            raise ValueError("rvol must be [nz][n][n]")
        nz, n1, n2 = rvol.shape
        if n1 != n2:
            raise ValueError("only square windows are supported (the reference uses one centre, mset.cu:83)")
        pr = _cplx_f32(probe)
        pp = _cplx_f32(prop)
        sx = _c32(scan_x).reshape(-1)
        sy = _c32(scan_y).reshape(-1)
        meas = _c32(measured).reshape(-1, n1, n1)
        npos = sx.size
        if sy.size != npos or meas.shape[0] != npos:
            raise ValueError("scan_x, scan_y and measured must have one entry per position")
        if pr.shape != (n1, n1, 2) or pp.shape != (n1, n1, 2):
            raise ValueError("probe and prop must be n x n complex")
        a = _lib.UploadArgs()
        a.n, a.nz, a.num_scan_pos = n1, nz, npos
        a.N_scan_x = int(n_scan_x if n_scan_x is not None else npos)
        a.N_scan_y = int(n_scan_y if n_scan_y is not None else 1)
        a.sigma = float(sigma)
        a.potential_pixelsize = float(potential_pixelsize)
        a.alpha = 0.0
        a.E0 = 0.0
        a.step_size[:] = [float(v) for v in step_size]
        a.slice_binning = int(slice_binning)
        a.RVol, a.init_wave2D, a.prop2D = fptr(rvol), fptr(pr), fptr(pp)
        a.scan_xlist, a.scan_ylist, a.measured = fptr(sx), fptr(sy), fptr(meas)
        self._keep = [rvol, pr, pp, sx, sy, meas]
        check("mset_upload", self._lib.mset_upload(self._h, C.byref(a)))
        self.n, self.nz, self.npos = n1, nz, npos
        self._binning = int(slice_binning)

    # ---- 'run_mset' / 'run_sset' (mex_main.cu:98-155) ----
    def run(self, mode: int = MSET_MODE_MSET, adjoint: int = MSET_ADJOINT_REF, with_error: bool = True):
        rv = np.empty((self.nz, self.n, self.n), np.float32)
        pr = np.empty((self.n, self.n, 2), np.float32)
        sx = np.empty(max(self.npos, 1), np.float32)
        sy = np.empty(max(self.npos, 1), np.float32)
        err = np.zeros(1, np.float32)
        check("mset_run_ex", self._lib.mset_run_ex(self._h, int(mode), int(adjoint), fptr(rv), fptr(pr),
                                                   fptr(sx), fptr(sy), fptr(err) if with_error else None))
        probe = pr.view(np.complex64).reshape(self.n, self.n)
        out = (rv, probe, sx[: self.npos].copy(), sy[: self.npos].copy())
        return out + ((float(err[0]),) if with_error else ())

    # ---- 'error_mset' / 'error_sset' (mex_main.cu:157-184) ----
    def error(self, mode: int = MSET_MODE_MSET) -> float:
        err = np.zeros(1, np.float32)
        check("mset_error", self._lib.mset_error(self._h, int(mode), fptr(err)))
        return float(err[0])

    # ---- per-position steps of the CPU path (Run_MSET_recon.m:136-157) ----
    def step02(self, k: int, row: float, col: float, mode: int = MSET_MODE_MSET) -> dict:
        """STEP02_FORWARD_4D(_SSET) of position k at scan coordinates (row, col):
        dict with calc (centred |Psi|^2), resi (centred residual), waves
        (save_wave_f: [ns][n][n], SSET [1][n][n]), psi0 (tmp_probe_wave) and
        err (this position's error term)"""
        n = self.n
        ns = 1 if mode == MSET_MODE_SSET else self._ns()
        calc = np.empty((n, n), np.float32)
        resi = np.empty((n, n, 2), np.float32)
        waves = np.empty((ns, n, n, 2), np.float32)
        psi0 = np.empty((n, n, 2), np.float32)
        err = np.zeros(1, np.float32)
        check("mset_forward_position",
              self._lib.mset_forward_position(self._h, int(mode), int(k), float(row), float(col), fptr(calc),
                                              fptr(resi), fptr(waves), fptr(psi0), fptr(err)))
        cplx = lambda a: a.view(np.complex64)[..., 0]
        return dict(calc=calc, resi=cplx(resi), waves=cplx(waves), psi0=cplx(psi0), err=float(err[0]))

    def step03(self, mode: int = MSET_MODE_MSET, adjoint: int = MSET_ADJOINT_REF, resi=None,
               update_rvol: bool = False, want=("grad", "probe")) -> dict:
        """STEP03_BACK(_SSET) after :meth:`step02` (and STEP04 with update_rvol):
        dict with grad ([nz][n][n] complex, slab-replicated), probe (updated)
        and row, col (updated scan coordinates); grad / probe only when named
        in `want` (each is a device-to-host copy)"""
        n = self.n
        ri = None if resi is None else _cplx_f32(resi)
        if ri is not None and ri.shape != (n, n, 2):
            raise ValueError("resi must be n x n complex")
        grad = np.empty((self.nz, n, n, 2), np.float32) if "grad" in want else None
        probe = np.empty((n, n, 2), np.float32) if "probe" in want else None
        rc = np.zeros(2, np.float32)
        check("mset_adjoint_position",
              self._lib.mset_adjoint_position(self._h, int(mode), int(adjoint), fptr(ri) if ri is not None else None,
                                              int(bool(update_rvol)), fptr(grad), fptr(probe), fptr(rc)))
        cplx = lambda a: None if a is None else a.view(np.complex64)[..., 0]
        return dict(grad=cplx(grad), probe=cplx(probe), row=float(rc[0]), col=float(rc[1]))

    def set_sequential_split(self, on: bool) -> None:
        """split one position's field over a thread-block cluster in run() and
        the per-position steps (default on where compiled, n = 128)"""
        check("mset_set_sequential_split", self._lib.mset_set_sequential_split(self._h, int(bool(on))))

    def sequential_split(self) -> int:
        """CTAs per field of the sequential modes after upload (1: one CTA)"""
        r = self._lib.mset_sequential_split(self._h)
        if r < 0:
            check("mset_sequential_split", r)
        return int(r)

    def read_state(self):
        """(rvol [nz][n][n] float32, probe [n][n] complex64): the session's
        volume and probe as the per-position steps left them on the device"""
        n = self.n
        rv = np.empty((self.nz, n, n), np.float32)
        probe = np.empty((n, n, 2), np.float32)
        check("mset_read_state", self._lib.mset_read_state(self._h, fptr(rv), fptr(probe)))
        return rv, probe.view(np.complex64)[..., 0]

    def _ns(self) -> int:
        b = max(1, min(self._binning, self.nz))
        return -(-self.nz // b)


# ---------------------------------------------------------------------------
# reference call signature
# ---------------------------------------------------------------------------
_default: Session | None = None


def _field(d: Mapping[str, Any], k: str):
    if k not in d:
        raise KeyError(f"STEM_data has no field '{k}'")
    return d[k]


def _scalar(v) -> float:
    return float(np.asarray(v).reshape(-1)[0])


def _cells_linear(cells) -> list:
    """measured cell array -> list in MATLAB linear (column-major) order"""
    if isinstance(cells, np.ndarray) and cells.dtype == object:
        return list(cells.reshape(-1, order="F"))
    if isinstance(cells, np.ndarray) and cells.ndim == 4:  # (nsx, nsy, n, n)
        return [cells[i, j] for j in range(cells.shape[1]) for i in range(cells.shape[0])]
    return list(cells)


def mset_cuda_kernel(mode: str, STEM_data: Mapping[str, Any], measured_cells=None):
    """Drop-in for the reference MEX function ``mset_cuda_kernel``
    (mex_main.cu:19-39).

    Arrays are MATLAB-shaped: ``RVol`` (n, n, nz), ``init_wave2D`` and
    ``prop2D`` (n, n) complex, ``scan_xlist``/``scan_ylist`` (P,), the measured
    cell array (N_scan_x, N_scan_y) of (n, n) patterns.  Returns what the MEX
    returns: nothing for 'upload'; ``(RVol, probe, scan_x, scan_y[, error])``
    for 'run_*' (the error is always returned here); ``error`` for 'error_*'.
    """
    global _default
    if mode == "upload":
        d = STEM_data
        rvol_m = np.asarray(_field(d, "RVol"), dtype=np.float32)
        rvol = np.ascontiguousarray(rvol_m.transpose(2, 1, 0))  # MATLAB (n,n,nz) -> C [nz][n][n]
        probe = np.ascontiguousarray(np.asarray(_field(d, "init_wave2D")).T)
        prop = np.ascontiguousarray(np.asarray(_field(d, "prop2D")).T)
        cells = _cells_linear(measured_cells)
        meas = np.stack([np.asarray(c, dtype=np.float32).T for c in cells]) if cells else \
            np.zeros((0, rvol.shape[1], rvol.shape[2]), np.float32)
        npos = int(_scalar(_field(d, "num_scan_pos")))
        if _default is None:
            _default = Session(0)
        _default.upload(rvol, probe, prop, sigma=_scalar(_field(d, "sigma")),
                        potential_pixelsize=_scalar(_field(d, "potential_pixelsize")),
                        scan_x=np.asarray(_field(d, "scan_xlist")).reshape(-1)[:npos],
                        scan_y=np.asarray(_field(d, "scan_ylist")).reshape(-1)[:npos],
                        measured=meas[:npos],
                        step_size=np.asarray(_field(d, "step_size"), dtype=np.float64).reshape(-1)[:3],
                        slice_binning=int(_scalar(_field(d, "slice_binning"))),
                        n_scan_x=int(_scalar(_field(d, "N_scan_x"))),
                        n_scan_y=int(_scalar(_field(d, "N_scan_y"))))
        return None
    if mode in ("run_mset", "run_sset"):
        if _default is None:
            raise RuntimeError("run called before upload")
        rv, pr, sx, sy, err = _default.run(_MODES[mode[4:]])
        return rv.transpose(2, 1, 0), pr.T, sx, sy, err
    if mode in ("error_mset", "error_sset"):
        if _default is None:
            raise RuntimeError("error called before upload")
        return _default.error(_MODES[mode[6:]])
    raise ValueError("The running mode is not correct (choose 'upload' or 'run_mset' or 'run_sset' "
                     "or 'error_mset' or 'error_sset')")


def clear() -> None:
    """``clear mset_cuda_kernel`` (Run_MSET_recon.m:174): drop the session."""
    global _default
    if _default is not None:
        _default.close()
        _default = None


__all__ = ["Session", "mset_cuda_kernel", "clear", "MSET_MODE_MSET", "MSET_MODE_SSET",
           "MSET_ADJOINT_REF", "MSET_ADJOINT_EXACT"]
